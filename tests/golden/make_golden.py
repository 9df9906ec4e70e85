"""Regenerates the committed fixtures under tests/golden/.

strand_cache_kat.strands: the 3-vertex, 1-strand binary cache that the
reference's unit test builds by hand (src/strand_cache.rs:254-281).
curly_600.strands: a seeded asset in the binary `.strands` layout (600 curly
strands x 12 points) for the loader-to-GPU parity test: the vertices are
stored at twice their size with a scale of 0.5 and in a shuffled order that
the index buffer undoes, so the loader's scale and indexing both matter.
oracle_tiny.json: SHA-256 digests of the oracle's integer outputs for the
seeded "tiny" scene; they pin the oracle against unintended drift (the
reference cannot run here, so these are oracle-produced, not reference-produced).

Run: python tests/golden/make_golden.py
"""
import hashlib
import json
import struct
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))


def kat_bytes() -> bytes:
    b = bytearray(b"SSRSTRD\0")
    b += struct.pack("<I", 1) + struct.pack("<f", 1.0) + struct.pack("<QQQ", 3, 1, 3)
    for v in ([0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.0]):
        b += struct.pack("<3f", *v)
    b += struct.pack("<II", 3, 0) + struct.pack("<3I", 0, 1, 2)
    return bytes(b)


GOLDEN_DUMPS = ["DUMP_FRUSTA", "DUMP_RANGES", "DUMP_KEEP", "DUMP_LUT", "DUMP_TASKS", "DUMP_PROJECTED",
                "DUMP_PAGE_TABLE", "DUMP_PAGE_META", "DUMP_COUNTS", "DUMP_OFFSETS", "DUMP_REFS",
                "DUMP_ACTIVE_TILES", "DUMP_WORK", "DUMP_RUNS", "DUMP_DOM_DEPTH", "DUMP_DOM_OPACITY",
                "DUMP_SHADOW_MAP"]


def oracle_digests() -> dict:
    from bevy_strand_rasterizer_b200 import abi
    from common import build_scene, run_ref
    fr = run_ref(build_scene("tiny"), threads=1)
    out = {}
    for name in GOLDEN_DUMPS:
        out[name] = hashlib.sha256(fr.get(getattr(abi, name)).view("u1").tobytes()).hexdigest()
    out["stats"] = {k: v for k, v in fr.stats().as_dict().items() if not isinstance(v, list)}
    return out


def curly_asset_bytes() -> bytes:
    import numpy as np
    from bevy_strand_rasterizer_b200.scene import scalp_hair
    from bevy_strand_rasterizer_b200.strand_cache import StrandCacheFile, write_binary_cache
    sl = scalp_hair(600, 12, 2024, curly=True)
    pts = np.asarray(sl.vertices, np.float32)[np.asarray(sl.indices)]  # points in strand order
    perm = np.random.default_rng(2024).permutation(pts.shape[0])     # stored order
    stored = np.empty_like(pts)
    stored[perm] = pts * np.float32(2.0)                              # point k lives at row perm[k]
    cache = StrandCacheFile(1, None, 0.5, stored, np.asarray(sl.strand_counts, np.uint32),
                            np.asarray(sl.strand_offsets, np.uint32), perm.astype(np.uint32))
    return write_binary_cache(cache)


if __name__ == "__main__":
    (HERE / "curly_600.strands").write_bytes(curly_asset_bytes())
    (HERE / "strand_cache_kat.strands").write_bytes(kat_bytes())
    (HERE / "oracle_tiny.json").write_text(json.dumps(oracle_digests(), indent=1, sort_keys=True) + "\n")
    print("wrote", HERE / "strand_cache_kat.strands", HERE / "oracle_tiny.json")
