"""`.strands` parser: mirrors the reference's only unit test,
strand_cache::tests::parses_binary_cache (src/strand_cache.rs:238-281), plus the
validation and JSON paths of parse_cache / validate_cache (:109-209)."""
import json
import struct
from pathlib import Path

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import strand_cache as sc
from bevy_strand_rasterizer_b200.plugin import pack_indexed_strands

GOLDEN = Path(__file__).parent / "golden" / "strand_cache_kat.strands"


def _kat_bytes() -> bytes:
    b = bytearray(sc.BINARY_MAGIC)
    b += struct.pack("<I", sc.BINARY_VERSION)
    b += struct.pack("<f", 1.0)
    b += struct.pack("<QQQ", 3, 1, 3)
    for v in ([0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.0]):
        b += struct.pack("<3f", *v)
    b += struct.pack("<II", 3, 0)
    b += struct.pack("<3I", 0, 1, 2)
    return bytes(b)


def test_parses_binary_cache():
    cache = sc.parse_binary_cache(_kat_bytes())
    sc.validate_cache(cache)
    assert cache.vertices.shape == (3, 3)
    assert cache.counts.tolist() == [3]
    assert cache.indices.tolist() == [0, 1, 2]
    assert cache.scale == 1.0


def test_golden_file_matches_kat():
    assert GOLDEN.read_bytes() == _kat_bytes()
    assert sc.parse_cache(GOLDEN.read_bytes()).indices.tolist() == [0, 1, 2]


def test_rejects_bad_magic_version_and_trailing_bytes():
    with pytest.raises(sc.StrandCacheError, match="magic"):
        sc.parse_binary_cache(b"NOTMAGIC" + _kat_bytes()[8:])
    bad_version = bytearray(_kat_bytes())
    bad_version[8:12] = struct.pack("<I", 2)
    with pytest.raises(sc.StrandCacheError, match="version"):
        sc.parse_binary_cache(bytes(bad_version))
    with pytest.raises(sc.StrandCacheError, match="trailing"):
        sc.parse_binary_cache(_kat_bytes() + b"\0")
    with pytest.raises(sc.StrandCacheError, match="end"):
        sc.parse_binary_cache(_kat_bytes()[:-2])


def test_validate_errors():
    c = sc.parse_binary_cache(_kat_bytes())
    c.counts = np.array([1], np.uint32)
    with pytest.raises(sc.StrandCacheError, match="fewer than two"):
        sc.validate_cache(c)
    c = sc.parse_binary_cache(_kat_bytes())
    c.offsets = np.array([1], np.uint32)
    with pytest.raises(sc.StrandCacheError, match="exceeds"):
        sc.validate_cache(c)
    c = sc.parse_binary_cache(_kat_bytes())
    c.indices = np.array([0, 1, 7], np.uint32)
    with pytest.raises(sc.StrandCacheError, match="references vertex 7"):
        sc.validate_cache(c)


def test_json_cache_and_roundtrip():
    j = {"version": 1, "source": "unit", "vertices": [[0, 0, 0], [0, 1, 0], [0, 2, 0], [1, 0, 0], [1, 1, 0]],
         "strands": [[0, 1, 2], [3, 4]]}
    c = sc.parse_cache(json.dumps(j).encode())
    sc.validate_cache(c)
    assert c.scale == 1.0 and c.counts.tolist() == [3, 2] and c.offsets.tolist() == [0, 3]
    again = sc.parse_cache(sc.write_binary_cache(c))
    assert np.array_equal(again.vertices, c.vertices) and np.array_equal(again.indices, c.indices)
    packed = pack_indexed_strands(c.vertices, c.counts, c.offsets, c.indices)
    assert packed.strand_count == 2 and packed.index_count == 5
    assert packed.vertices.shape == (5, 4) and np.all(packed.vertices[:, 3] == 1.0)


def test_committed_curly_asset_loads_to_the_seeded_strands():
    # tests/golden/curly_600.strands (tests/golden/make_golden.py): vertices
    # stored doubled with scale 0.5 in a shuffled order; the loader's scale and
    # index buffer give back the seeded strands point for point.
    from bevy_strand_rasterizer_b200.scene import scalp_hair
    from bevy_strand_rasterizer_b200.strand_cache import load, to_packed
    cache = load(str(Path(__file__).parent / "golden" / "curly_600.strands"))
    assert cache.scale == 0.5 and cache.counts.shape[0] == 600
    packed = to_packed(cache)
    sl = scalp_hair(600, 12, 2024, curly=True)
    want = np.asarray(sl.vertices, np.float32)[np.asarray(sl.indices)]
    got = packed.vertices[packed.indices][:, :3]
    assert np.array_equal(got, want)
    assert np.all(packed.vertices[:, 3] == 1.0)
    assert packed.meta["count"].tolist() == np.asarray(sl.strand_counts).tolist()
