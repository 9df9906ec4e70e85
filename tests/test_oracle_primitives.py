"""Known-answer tests for the oracle's primitives, each checked against an
independent numpy / pure-Python statement of the WGSL builtin it restates
(src/shaders/common.wgsl:206-262, strand_prepass.wgsl:523-539,1356-1410,884-1014)."""
import ctypes as C

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from oracle_bridge import oracle_lib

F = np.float32


def py_wang_hash(x: int) -> int:
    m = 0xFFFFFFFF
    x = (x ^ 61) ^ (x >> 16)
    x = (x + (x << 3)) & m
    x = x ^ (x >> 4)
    x = (x * 0x27D4EB2D) & m
    return x ^ (x >> 15)


def test_wang_hash_known_answers():
    lib = oracle_lib()
    assert lib.fref_wang_hash(0) == py_wang_hash(0)
    rng = np.random.default_rng(3)
    for x in [1, 61, 12345, 0x7FFFFFFF, 0xFFFFFFFF] + rng.integers(0, 2**32, 500, dtype=np.uint64).tolist():
        assert lib.fref_wang_hash(int(x)) == py_wang_hash(int(x))
    # instance/strand seeding of broad_strand_prepass: wang_hash((inst * 16777619) ^ strand)
    assert lib.fref_wang_hash(((3 * 16777619) & 0xFFFFFFFF) ^ 42) == py_wang_hash(((3 * 16777619) & 0xFFFFFFFF) ^ 42)


def test_hash_to_unit_float():
    lib = oracle_lib()
    for x in [0, 1, 2**31, 2**32 - 1, 123456789]:
        want = F(F(x) / F(4294967296.0))
        assert np.float32(lib.fref_hash_to_unit_float(x)) == want
    assert lib.fref_hash_to_unit_float(2**32 - 1) == 1.0  # rounds up to 2^32


def py_unorm16(e):
    e = F(min(F(1.0), max(F(0.0), F(e))))
    return int(np.floor(F(0.5) + F(65535.0) * e))


def test_pack2x16unorm():
    lib = oracle_lib()
    assert lib.fref_pack2x16unorm(0.0, 1.0) == 0xFFFF0000
    assert lib.fref_pack2x16unorm(0.5, 0.25) == 0x40008000
    assert lib.fref_pack2x16unorm(-3.0, 7.0) == 0xFFFF0000
    rng = np.random.default_rng(5)
    for a, b in rng.uniform(-0.1, 1.1, (300, 2)).astype(np.float32):
        assert lib.fref_pack2x16unorm(float(a), float(b)) == py_unorm16(a) | (py_unorm16(b) << 16)


def test_quantize_depth01_round_half_even():
    lib = oracle_lib()
    assert lib.fref_quantize_depth01(0.5) == 8388608  # 8388607.5 rounds to even
    assert lib.fref_quantize_depth01(1.0) == 16777215
    assert lib.fref_quantize_depth01(-1.0) == 0
    rng = np.random.default_rng(9)
    for z in rng.uniform(0.0, 1.0, 500).astype(np.float32):
        want = int(np.rint(F(z) * F(16777215.0)))
        assert lib.fref_quantize_depth01(float(z)) == want


def test_normalize_depth01():
    lib = oracle_lib()
    assert lib.fref_normalize_depth01(0.25) == pytest.approx(0.25)
    assert lib.fref_normalize_depth01(-0.5) == pytest.approx(0.25)
    assert lib.fref_normalize_depth01(-1.0) == 0.0
    assert lib.fref_normalize_depth01(2.0) == 1.0


def _clip(p0, p1, lo, hi):
    arr = lambda v: (C.c_float * len(v))(*v)
    out = (C.c_float * 6)()
    ok = oracle_lib().fref_clip_segment(arr(p0), arr(p1), arr(lo), arr(hi), out)
    return ok, list(out)


def test_clip_segment_cases():
    ok, o = _clip([-10, 5, 0.5], [10, 5, 0.5], [0, 0, 0], [8, 8, 1])
    assert ok == 1 and o[0] == pytest.approx(0.0) and o[3] == pytest.approx(8.0) and o[1] == o[4] == 5.0
    ok, _ = _clip([-10, 9, 0.5], [10, 9, 0.5], [0, 0, 0], [8, 8, 1])  # y = 9 outside, degenerate axis
    assert ok == 0
    ok, _ = _clip([20, 1, 0.5], [30, 2, 0.5], [0, 0, 0], [8, 8, 1])
    assert ok == 0
    ok, o = _clip([1, 1, 0.2], [2, 2, 0.4], [0, 0, 0], [8, 8, 1])  # fully inside: untouched
    assert ok == 1 and o == pytest.approx([1, 1, 0.2, 2, 2, 0.4])


def _lut(intervals):
    mins = (C.c_uint32 * max(1, len(intervals)))(*[a for a, _ in intervals])
    maxs = (C.c_uint32 * max(1, len(intervals)))(*[b for _, b in intervals])
    out = np.zeros(16, abi.LUT_ENTRY)
    oracle_lib().fref_build_lut(mins, maxs, len(intervals), out.ctypes.data)
    return out


def test_depth_warp_lut_single_interval():
    lut = _lut([(100, 1699)])
    assert lut["z_min_q"].tolist() == [100 + 100 * i for i in range(16)]
    assert lut["z_max_q"].tolist() == [199 + 100 * i for i in range(16)]
    assert np.all(lut["virtual_count_q"] == 100)


def test_depth_warp_lut_two_intervals_sorted_and_split():
    lut = _lut([(1000, 1099), (0, 99)])  # inserted out of order
    # 8 slices per interval: start = z_min + (100 * s) // 8
    assert lut["z_min_q"][:8].tolist() == [0, 12, 25, 37, 50, 62, 75, 87]
    assert lut["z_max_q"][:8].tolist() == [11, 24, 36, 49, 61, 74, 86, 99]
    assert lut["z_min_q"][8] == 1000 and lut["z_max_q"][15] == 1099


def test_depth_warp_lut_merge_and_overflow():
    lut = _lut([(0, 10), (11, 20)])  # touching intervals merge
    assert lut["z_min_q"][0] == 0 and lut["z_max_q"][15] == 20
    assert _lut([])["virtual_count_q"].sum() == 0
    # 17 disjoint intervals: the 17th joins the nearest existing one
    iv = [(i * 1000, i * 1000 + 9) for i in range(16)] + [(15500, 15509)]
    lut = _lut(iv)
    assert lut["z_max_q"][15] == 15509 and lut["z_min_q"][15] == 15000
