"""Builds libfiber.so (the sm_100a CUDA library behind include/fiber.h) in-tree.

The library is compiled with --fmad=false and IEEE division / square root so
that the integer-deciding stages (projection, clipping, depth quantisation,
DDA traversal) reproduce binary32 results operation by operation; the shading
file alone (compared within a tolerance) is compiled with contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
LIB_PATH = PKG_DIR / "libfiber.so"
SOURCES = ["fiber_prepass.cu", "fiber_raster.cu", "fiber_render.cu", "fiber_ctx.cu", "fiber_server.cu", "fiber_batch.cu", "fiber_noalloc.cu"]
HEADERS = ["fiber_device.cuh", "fiber_kernels.cuh", "fiber_internal.h"]

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "--fmad=false",
    "-prec-div=true",
    "-prec-sqrt=true",
    "-ftz=false",
    "-Xcompiler", "-fPIC",
    "-Xptxas", "-O3",
]


# Shading and composite are compared within a tolerance (they end in binary16),
# so their file is compiled with contraction and approximate division and
# square root. What selects a DOM texel and slice there (projection, depth
# normalisation, the slice quotient) is written with correctly rounded
# intrinsics and stays exact.
FAST_FP_SOURCES = {"fiber_render.cu"}
FAST_FP = {"--fmad=false": "--fmad=true", "-prec-div=true": "-prec-div=false", "-prec-sqrt=true": "-prec-sqrt=false"}


def flags_for(src: str) -> list[str]:
    """nvcc flags of one source file."""
    if src in FAST_FP_SOURCES:
        return [FAST_FP.get(f, f) for f in NVCC_FLAGS]
    return list(NVCC_FLAGS)


def _nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda_home) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def _stale(out: Path, inputs: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.stat().st_mtime > t for p in inputs)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    """Compiles the CUDA sources into libfiber.so next to this file."""
    include = PKG_DIR.parent / "include"
    inputs = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS] + [include / "fiber.h"]
    if not force and not ptxas_info and not _stale(LIB_PATH, inputs):
        return LIB_PATH
    obj_dir = PKG_DIR / "_build"
    obj_dir.mkdir(exist_ok=True)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in SOURCES:
        obj = obj_dir / (Path(src).stem + ".o")
        cmd = [_nvcc(), *flags_for(src), *extra, "-I", str(include), "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", str(tmp), "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas-info" in sys.argv)
