"""DSF polyline hair import (examples/dson_scene.rs:15-81): the field rules on
a synthetic document, and the real Pixie Cut asset of the reference tree
through pack_strands and the oracle when that asset is present."""
import json
from pathlib import Path

import numpy as np
import pytest

from bevy_strand_rasterizer_b200.dsf import DsfError, INCH_TO_METRE, load_dsf, parse_dsf_polylines
from bevy_strand_rasterizer_b200.plugin import pack_strands

import os

# The reference tree's Pixie Cut asset (assets/dForce Pixie Cut_708408.dsf of the
# reference project), given by path in FIBER_PIXIE_DSF; the test skips without it.
PIXIE = Path(os.environ.get("FIBER_PIXIE_DSF", "")) if os.environ.get("FIBER_PIXIE_DSF") else None


def _doc(geometries):
    return json.dumps({"file_version": "0.6.1.0", "geometry_library": geometries})


def test_polyline_rules():
    g0 = {"id": "mesh", "vertices": {"count": 4, "values": [[1, 2, 3], [4, 5, 6], [7, 8, 9], [10, 11, 12]]}}
    g1 = {"id": "hair", "vertices": {"values": [[0, 0, 0]]},
          "polyline_list": {"values": [
              [0, 0, 1, 2],          # two indices: kept
              [0, 1, 3],             # fewer than 4 entries: dropped
              [0, 2, 0, -1, 2.5],    # one non-negative integer index: dropped
              [0, 3, 3, 2, 1, 0],    # kept
              [0, 4, True, 1, 2],    # booleans are not indices
              "junk",
          ]}}
    sl = parse_dsf_polylines(_doc([g0, g1]))
    # strands from the first geometry with polylines, vertices from the first geometry
    assert [s.tolist() for s in sl.strands] == [[1, 2], [3, 2, 1, 0], [1, 2]]
    want = (np.array([[1, 2, 3], [4, 5, 6], [7, 8, 9], [10, 11, 12]], np.float32) * np.float32(INCH_TO_METRE))
    assert sl.vertices.dtype == np.float32 and np.array_equal(sl.vertices, want)
    packed = pack_strands(sl.vertices, sl.strands)
    assert packed.strand_count == 3 and packed.index_count == 8
    assert packed.meta["count"].tolist() == [2, 4, 2] and packed.meta["offset"].tolist() == [0, 2, 6]


def test_index_cast_and_errors():
    g = {"vertices": {"values": [[0, 0, 0]]}, "polyline_list": {"values": [[0, 0, 2**32 + 5, 7]]}}
    assert parse_dsf_polylines(_doc([g])).strands[0].tolist() == [5, 7]  # `as u32`
    with pytest.raises(DsfError):
        parse_dsf_polylines("{not json")
    with pytest.raises(DsfError):
        parse_dsf_polylines(_doc([]))
    with pytest.raises(DsfError):
        parse_dsf_polylines(_doc([{"vertices": {"values": [[0, 0, 0]]}, "polyline_list": {"values": [[0, 0, 1]]}}]))


@pytest.mark.skipif(PIXIE is None or not PIXIE.exists(), reason="FIBER_PIXIE_DSF does not name the Pixie Cut asset")
def test_pixie_cut_through_the_oracle():
    sl = load_dsf(PIXIE)
    assert sl.vertices.shape == (236136, 3)
    assert len(sl.strands) == 21755
    packed = pack_strands(sl.vertices, sl.strands)
    assert packed.strand_count == 21755
    assert int(packed.indices.max()) < sl.vertices.shape[0]
    # one frame of the oracle over the imported hair: a camera in front of the
    # head looking at the hair's centre, one light from above
    from bevy_strand_rasterizer_b200 import abi
    from bevy_strand_rasterizer_b200.plugin import FroxelConfig, StrandMaterial
    from bevy_strand_rasterizer_b200.scene import CameraSpec, LightSpec
    from oracle_bridge import run_oracle
    lo, hi = packed.aabb_min, packed.aabb_max
    center = 0.5 * (lo + hi)
    eye = center + np.array([0.0, 0.05, 0.6])
    cam_spec = CameraSpec(eye=tuple(float(x) for x in eye), target=tuple(float(x) for x in center), width=320,
                          height=240)
    cam = abi.Camera()
    cam.clip_from_world[:] = [float(x) for x in cam_spec.clip_from_world()]
    cam.world_position[:] = [float(x) for x in eye]
    light = LightSpec((0.3, 1.0, 0.4), size=256)
    lights = (abi.Light * 1)()
    lights[0].clip_from_world[:] = [float(x) for x in light.clip_from_world(lo, hi)]
    lights[0].direction_to_light[:] = [float(x) for x in light.direction()]
    lights[0].color[:] = [float(x) for x in light.color4()]
    st = abi.default_settings()
    st.dom_slices = 4
    material = StrandMaterial(min_radius_pixels=0.7, max_radius_pixels=2.0)
    ident = np.eye(4, dtype=np.float32).reshape(16)
    fr = run_oracle([(packed, material, ident)], FroxelConfig(320, 240, 8, 8, 64), cam,
                    [FroxelConfig(256, 256, 8, 8, 64)], lights, st)
    s = fr.stats()
    assert s.binning_tasks > 0 and s.fine_refs > 0 and s.camera_runs > 0 and s.shadow_runs > 0
    color = fr.get(abi.DUMP_COLOR).astype(np.float32).reshape(240, 320, 4)
    assert (color[..., 3] > 0).mean() > 0.05  # the hair covers a visible part of the frame
