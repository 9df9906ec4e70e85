"""ctypes bridge from the tests to the oracle (oracle/_build/libfiber_ref.so).

Test infrastructure only: the oracle is the checker, never the thing measured.
It receives exactly the host arrays and matrices that the GPU path receives.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from bevy_strand_rasterizer_b200 import abi

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "_build" / "libfiber_ref.so"

FREF_COMPOSITE = 100
FREF_REF_KEYS = 101
FREF_STAGE_MS = 102
FREF_TELEMETRY = 103


class FrefInstance(C.Structure):
    _fields_ = [("vertices4", C.c_void_p), ("n_vertices", C.c_uint32), ("indices", C.c_void_p),
                ("n_indices", C.c_uint32), ("meta", C.c_void_p), ("n_meta", C.c_uint32),
                ("geo", abi.StrandGeo), ("materials", C.c_void_p), ("n_materials", C.c_uint32),
                ("world_from_local", C.c_float * 16)]


class FrefCaps(C.Structure):
    _fields_ = [("task_capacity", C.c_uint32), ("page_capacity", C.c_uint32), ("ref_capacity", C.c_uint32),
                ("work_capacity", C.c_uint32)]


_LIB = None


def build_oracle() -> Path:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return ORACLE_LIB


def oracle_lib():
    global _LIB
    if _LIB is None:
        if not ORACLE_LIB.exists():
            build_oracle()
        lib = C.CDLL(str(ORACLE_LIB))
        lib.fref_run.restype = C.c_void_p
        lib.fref_run.argtypes = [C.POINTER(FrefInstance), C.c_uint32, C.POINTER(abi.FroxelConfigC),
                                 C.POINTER(abi.Camera), C.POINTER(abi.FroxelConfigC), C.POINTER(abi.Light),
                                 C.c_uint32, C.POINTER(abi.Settings), C.POINTER(FrefCaps), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_int]
        lib.fref_run_opaque.restype = C.c_void_p
        lib.fref_run_opaque.argtypes = lib.fref_run.argtypes[:-1] + [C.c_void_p, C.c_uint32, C.c_int]
        lib.fref_get.restype = C.c_uint64
        lib.fref_get.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64]
        lib.fref_stats.restype = None
        lib.fref_stats.argtypes = [C.c_void_p, C.POINTER(abi.Stats)]
        lib.fref_free.restype = None
        lib.fref_free.argtypes = [C.c_void_p]
        lib.fref_wang_hash.restype = C.c_uint32
        lib.fref_wang_hash.argtypes = [C.c_uint32]
        lib.fref_hash_to_unit_float.restype = C.c_float
        lib.fref_hash_to_unit_float.argtypes = [C.c_uint32]
        lib.fref_pack2x16unorm.restype = C.c_uint32
        lib.fref_pack2x16unorm.argtypes = [C.c_float, C.c_float]
        lib.fref_quantize_depth01.restype = C.c_uint32
        lib.fref_quantize_depth01.argtypes = [C.c_float]
        lib.fref_normalize_depth01.restype = C.c_float
        lib.fref_normalize_depth01.argtypes = [C.c_float]
        lib.fref_clip_segment.restype = C.c_uint32
        lib.fref_clip_segment.argtypes = [C.POINTER(C.c_float)] * 5
        lib.fref_build_lut.restype = None
        lib.fref_build_lut.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_uint32, C.c_void_p]
        lib.fref_composite.restype = None
        lib.fref_composite.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        _LIB = lib
    return _LIB


def _next_pow2(x: int) -> int:
    p = 1
    while p < x:
        p <<= 1
    return p


def capacities(total_segments: int, total_strands: int, n_frusta: int, total_coarse_tiles: int,
               settings: abi.Settings) -> FrefCaps:
    """The capacities fiber_frame_begin derives from src/plugin.rs:483-576
    (kept identical so overflow behaviour matches)."""
    table = total_coarse_tiles * 16
    prepass = max(_next_pow2(total_strands), 2048)
    base = max(_next_pow2(total_segments), prepass)
    task = max(_next_pow2(base * n_frusta), base)
    page = max(1, table // settings.page_capacity_divisor)
    ref = max(_next_pow2(task * settings.ref_capacity_factor), max(task, 1024))
    work = max(1, min(ref, 256 * table))
    return FrefCaps(task, page, ref, work)


def coarse_tiles(cfgs) -> int:
    total = 0
    for c in cfgs:
        tx = (c.screen_width + c.froxel_size_x - 1) // c.froxel_size_x
        ty = (c.screen_height + c.froxel_size_y - 1) // c.froxel_size_y
        total += max(1, (tx + 3) // 4) * max(1, (ty + 3) // 4)
    return total


@dataclass
class OracleFrame:
    handle: int

    def get(self, what: int, dtype=None) -> np.ndarray:
        lib = oracle_lib()
        n = lib.fref_get(self.handle, what, None, 0)
        buf = np.empty(n, np.uint8)
        if n:
            lib.fref_get(self.handle, what, buf.ctypes.data_as(C.c_void_p), n)
        if dtype is None:
            dtype = abi.DUMP_DTYPES.get(what, np.dtype("<f4"))
        return buf.view(dtype)

    def stats(self) -> abi.Stats:
        s = abi.Stats()
        oracle_lib().fref_stats(self.handle, C.byref(s))
        return s

    def telemetry(self) -> abi.Telemetry:
        w = self.get(FREF_TELEMETRY, np.dtype("<u4"))
        return abi.Telemetry.from_buffer_copy(w.tobytes())

    def composite(self, scene_color: np.ndarray, scene_depth: np.ndarray | None = None,
                  dest: np.ndarray | None = None, half_out: bool = True) -> np.ndarray:
        """The frame's composite over scene_color (H, W, 4) float32, blended
        onto dest (the destination's contents before the pass; None = in
        place over the scene colour). Returns (H, W, 4) float32."""
        sc = np.ascontiguousarray(scene_color, np.float32)
        sd = None if scene_depth is None else np.ascontiguousarray(scene_depth, np.float32)
        dd = None if dest is None else np.ascontiguousarray(dest, np.float32)
        out = np.empty_like(sc)
        oracle_lib().fref_composite(self.handle, sc.ctypes.data, sd.ctypes.data if sd is not None else None,
                                    dd.ctypes.data if dd is not None else None, 1 if half_out else 0,
                                    out.ctypes.data)
        return out

    def stage_ms(self) -> np.ndarray:
        return self.get(FREF_STAGE_MS, np.dtype("<f4"))

    def free(self):
        if self.handle:
            oracle_lib().fref_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def run_oracle(assets, camera_cfg, cam: abi.Camera, light_cfgs, lights_c, settings: abi.Settings,
               history_prev: np.ndarray | None = None, scene_color: np.ndarray | None = None,
               scene_depth: np.ndarray | None = None, threads: int = 0, opaque_depth: np.ndarray | None = None,
               opaque_samples: int = 1) -> OracleFrame:
    """assets: list of (PackedStrandBuffers, StrandMaterial, world_from_local[16]).
    opaque_depth: the camera's opaque depth, (H, W, samples) or (H, W) float32."""
    lib = oracle_lib()
    n = len(assets)
    insts = (FrefInstance * max(1, n))()
    keep = []
    total_segments = 0
    total_strands = 0
    for i, (packed, material, w) in enumerate(assets):
        v = np.ascontiguousarray(packed.vertices, np.float32)
        idx = np.ascontiguousarray(packed.indices, np.uint32)
        meta = np.ascontiguousarray(packed.meta)
        mat = np.frombuffer(bytes(material.to_c()), np.uint8).copy()
        keep += [v, idx, meta, mat]
        it = insts[i]
        it.vertices4 = v.ctypes.data
        it.n_vertices = v.shape[0]
        it.indices = idx.ctypes.data
        it.n_indices = idx.shape[0]
        it.meta = meta.ctypes.data
        it.n_meta = meta.shape[0]
        it.geo = packed.geo()
        it.materials = mat.ctypes.data
        it.n_materials = 1
        it.world_from_local[:] = [float(x) for x in np.asarray(w, np.float32).reshape(16)]
        c = meta["count"].astype(np.int64)
        total_segments += int(np.maximum(c - 1, 0)[c >= 2].sum())
        total_strands += min(int(meta.shape[0]), int(packed.strand_count))
    nl = len(light_cfgs)
    cfgs = (abi.FroxelConfigC * max(1, nl))(*[c.to_c() for c in light_cfgs])
    caps = capacities(total_segments, total_strands, 1 + nl, coarse_tiles([camera_cfg.to_c()] + [c.to_c() for c in light_cfgs]),
                      settings)
    hp = None if history_prev is None else np.ascontiguousarray(history_prev.view(np.uint16))
    sc = None if scene_color is None else np.ascontiguousarray(scene_color, np.float32)
    sd = None if scene_depth is None else np.ascontiguousarray(scene_depth, np.float32)
    od = None if opaque_depth is None else np.ascontiguousarray(opaque_depth, np.float32)
    h = lib.fref_run_opaque(insts, n, C.byref(camera_cfg.to_c()), C.byref(cam), cfgs, lights_c, nl,
                            C.byref(settings), C.byref(caps), hp.ctypes.data if hp is not None else None,
                            sc.ctypes.data if sc is not None else None, sd.ctypes.data if sd is not None else None,
                            od.ctypes.data if od is not None else None, opaque_samples, threads)
    del keep
    return OracleFrame(h)
