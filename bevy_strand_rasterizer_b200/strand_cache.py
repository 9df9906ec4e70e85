"""`.strands` cache format (src/strand_cache.rs:7-209).

Binary layout (little endian): magic b"SSRSTRD\\0", u32 version (1), f32 scale,
u64 vertex count, u64 strand count, u64 index count, then xyz f32 per vertex,
(count, offset) u32 pairs per strand and u32 indices; no trailing bytes. The
JSON variant holds {version, source, scale (default 1), vertices: [[x,y,z]],
strands: [[indices]]}. `validate_cache` applies the reference's checks.
"""
from __future__ import annotations

import json
import struct
from dataclasses import dataclass

import numpy as np

BINARY_MAGIC = b"SSRSTRD\0"
BINARY_VERSION = 1


class StrandCacheError(ValueError):
    pass


@dataclass
class StrandCacheFile:
    version: int
    source: str | None
    scale: float
    vertices: np.ndarray      # (V, 3) float32
    counts: np.ndarray        # (S,) uint32
    offsets: np.ndarray       # (S,) uint32
    indices: np.ndarray       # (N,) uint32


def parse_binary_cache(data: bytes) -> StrandCacheFile:
    if len(data) < 8 or data[:8] != BINARY_MAGIC:
        raise StrandCacheError("invalid strand cache magic")
    off = 8

    def take(fmt):
        nonlocal off
        size = struct.calcsize(fmt)
        if off + size > len(data):
            raise StrandCacheError("unexpected end of strand cache")
        v = struct.unpack_from(fmt, data, off)
        off += size
        return v

    (version,) = take("<I")
    if version != BINARY_VERSION:
        raise StrandCacheError(f"unsupported strand cache version {version}")
    (scale,) = take("<f")
    nv, ns, ni = take("<QQQ")
    need = nv * 12 + ns * 8 + ni * 4
    if off + need > len(data):
        raise StrandCacheError("unexpected end of strand cache")
    verts = np.frombuffer(data, "<f4", nv * 3, off).reshape(nv, 3).astype(np.float32)
    off += nv * 12
    pairs = np.frombuffer(data, "<u4", ns * 2, off).reshape(ns, 2)
    off += ns * 8
    idx = np.frombuffer(data, "<u4", ni, off).astype(np.uint32)
    off += ni * 4
    if off != len(data):
        raise StrandCacheError(f"strand cache has {len(data) - off} trailing bytes after payload")
    return StrandCacheFile(version, None, float(scale), verts, pairs[:, 0].astype(np.uint32),
                           pairs[:, 1].astype(np.uint32), idx)


def parse_json_cache(data: bytes) -> StrandCacheFile:
    j = json.loads(data)
    counts, offsets, idx = [], [], []
    for s in j["strands"]:
        counts.append(len(s))
        offsets.append(len(idx))
        idx.extend(s)
    return StrandCacheFile(int(j["version"]), j.get("source"), float(j.get("scale", 1.0)),
                           np.asarray(j["vertices"], np.float32).reshape(-1, 3), np.asarray(counts, np.uint32),
                           np.asarray(offsets, np.uint32), np.asarray(idx, np.uint32))


def parse_cache(data: bytes) -> StrandCacheFile:
    return parse_binary_cache(data) if data.startswith(BINARY_MAGIC) else parse_json_cache(data)


def validate_cache(cache: StrandCacheFile) -> None:
    if cache.version != BINARY_VERSION:
        raise StrandCacheError(f"unsupported strand cache version {cache.version}")
    n_idx, n_vert = cache.indices.shape[0], cache.vertices.shape[0]
    for s, (count, offset) in enumerate(zip(cache.counts.tolist(), cache.offsets.tolist())):
        if count < 2:
            raise StrandCacheError(f"strand {s} has fewer than two vertices")
        end = offset + count
        if end > 0xFFFFFFFF:
            raise StrandCacheError(f"strand {s} index range overflows")
        if end > n_idx:
            raise StrandCacheError(f"strand {s} range {offset}..{end} exceeds {n_idx} cache indices")
        bad = cache.indices[offset:end] >= n_vert
        if bad.any():
            v = int(cache.indices[offset:end][bad][0])
            raise StrandCacheError(f"strand {s} references vertex {v}, but cache has {n_vert} vertices")


def write_binary_cache(cache: StrandCacheFile) -> bytes:
    out = bytearray(BINARY_MAGIC)
    out += struct.pack("<If", BINARY_VERSION, cache.scale)
    out += struct.pack("<QQQ", cache.vertices.shape[0], cache.counts.shape[0], cache.indices.shape[0])
    out += np.ascontiguousarray(cache.vertices, "<f4").tobytes()
    out += np.ascontiguousarray(np.stack([cache.counts, cache.offsets], 1), "<u4").tobytes()
    out += np.ascontiguousarray(cache.indices, "<u4").tobytes()
    return bytes(out)


def load(path: str) -> StrandCacheFile:
    with open(path, "rb") as f:
        cache = parse_cache(f.read())
    validate_cache(cache)
    return cache


def to_packed(cache: StrandCacheFile):
    """set_cached_strand_geometry (src/plugin.rs:1468-1497): the cache's vertices
    times its scale (one binary32 product per component), then
    pack_indexed_strands over its strands and shared index buffer. None when no
    strand has two points (the reference warns and skips the entity)."""
    from .plugin import pack_indexed_strands
    v = np.ascontiguousarray(cache.vertices, np.float32) * np.float32(cache.scale)
    return pack_indexed_strands(v, cache.counts, cache.offsets, cache.indices)
