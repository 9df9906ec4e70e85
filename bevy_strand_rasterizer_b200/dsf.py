"""DSF (DAZ Studio JSON) polyline hair import, as the reference's DSON example
reads it (load_dson_polyline_strands and pack_loaded_dson_strands,
examples/dson_scene.rs:15-81):

- strands come from the first geometry of `geometry_library` whose
  `polyline_list.values` yields any strand. Each polyline is an array whose two
  leading fields are skipped; it needs at least 4 entries. Its remaining
  entries that are non-negative integers are the vertex indices (cast to u32),
  and a strand needs at least 2 of them;
- vertices come from the library's first geometry (`vertices.values`),
  converted from inches to metres (x 0.0254).

The result is a StrandList for pack_strands, the reference's path from a
StrandList component to the strand slabs.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from .plugin import StrandList

INCH_TO_METRE = 0.0254


class DsfError(ValueError):
    pass


def _index(v) -> int | None:
    # serde_json's as_u64: only non-negative integers (not floats, not booleans).
    if isinstance(v, bool) or not isinstance(v, int) or v < 0 or v >= 1 << 64:
        return None
    return v & 0xFFFFFFFF  # `index as u32`


def _polyline_strands(geometry) -> list[np.ndarray] | None:
    values = geometry.get("polyline_list", {}).get("values") if isinstance(geometry, dict) else None
    if not isinstance(values, list):
        return None
    strands = []
    for strand in values:
        if not isinstance(strand, list) or len(strand) < 4:
            continue
        idx = [i for i in (_index(v) for v in strand[2:]) if i is not None]
        if len(idx) >= 2:
            strands.append(np.asarray(idx, np.uint32))
    return strands or None


def parse_dsf_polylines(data: bytes | str) -> StrandList:
    try:
        doc = json.loads(data)
    except (ValueError, UnicodeDecodeError) as e:
        raise DsfError(f"not a DSF JSON document: {e}") from e
    library = doc.get("geometry_library") if isinstance(doc, dict) else None
    if not isinstance(library, list) or not library:
        raise DsfError("geometry library not found")
    strands = None
    for geometry in library:
        strands = _polyline_strands(geometry)
        if strands:
            break
    if not strands:
        raise DsfError("polyline list not found")
    verts = library[0].get("vertices", {}).get("values") if isinstance(library[0], dict) else None
    if not isinstance(verts, list):
        raise DsfError("vertices not found in the first geometry")
    v = np.asarray(verts, np.float32).reshape(-1, 3) * np.float32(INCH_TO_METRE)
    return StrandList(vertices=v, strands=strands)


def load_dsf(path: str | Path) -> StrandList:
    return parse_dsf_polylines(Path(path).read_bytes())
