"""A `.strands` asset through the loader and the plugin to the GPU, against the
oracle: the StrandCache path (src/plugin.rs:1468-1497) of the committed,
script-generated tests/golden/curly_600.strands (scaled, shuffled vertex
storage). Integer dumps must match bit for bit, colour within max-abs 2e-3 and
PSNR >= 50 dB."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from test_gpu_parity import EXACT, _close, _exact

pytestmark = pytest.mark.gpu

ASSET = Path(__file__).parent / "golden" / "curly_600.strands"


def test_strand_cache_asset_matches_oracle():
    from bevy_strand_rasterizer_b200.plugin import FroxelConfig, StrandMaterial, StrandRasterizerPlugin
    from bevy_strand_rasterizer_b200.scene import CameraSpec, LightSpec
    from bevy_strand_rasterizer_b200.strand_cache import load, to_packed
    from oracle_bridge import run_oracle

    cache = load(str(ASSET))
    packed = to_packed(cache)
    material = StrandMaterial(min_radius_pixels=0.6, max_radius_pixels=1.8)
    st = abi.default_settings()
    st.history_enabled = 0
    st.fragment_counts_enabled = 1
    st.dom_slices = 4
    plugin = StrandRasterizerPlugin()
    abi.check(plugin.lib.fiber_settings_set(plugin.ctx, C.byref(st)), "fiber_settings_set")
    plugin.add_strand_cache(ASSET, material)  # the plugin loads the file itself

    lo, hi = packed.aabb_min, packed.aabb_max
    center = 0.5 * (lo + hi)
    eye = center + np.array([0.15, 0.1, 0.45])
    spec = CameraSpec(eye=tuple(float(x) for x in eye), target=tuple(float(x) for x in center), width=256, height=192)
    cam = abi.Camera()
    cam.clip_from_world[:] = [float(x) for x in spec.clip_from_world()]
    cam.world_position[:] = [float(x) for x in eye]
    light = LightSpec((0.4, 1.0, 0.3), size=256)
    lights = (abi.Light * 1)()
    lights[0].clip_from_world[:] = [float(x) for x in light.clip_from_world(lo, hi)]
    lights[0].direction_to_light[:] = [float(x) for x in light.direction()]
    lights[0].color[:] = [float(x) for x in light.color4()]
    cfg, lcfg = FroxelConfig(256, 192, 8, 8, 32), [FroxelConfig(256, 256, 8, 8, 32)]
    plugin.frame_begin_raw(cfg, cam, lcfg, lights)
    plugin.render_nodes()
    ident = np.eye(4, dtype=np.float32).reshape(16)
    ref = run_oracle([(packed, material, ident)], cfg, cam, lcfg, lights, st)
    s, rs = plugin.stats(), ref.stats()
    assert s.binning_tasks == rs.binning_tasks > 0 and s.fine_refs == rs.fine_refs > 0
    for what in EXACT:
        _exact(plugin.dump(what), ref.get(what), what)
    _close(plugin.dump(abi.DUMP_COLOR), ref.get(abi.DUMP_COLOR), abi.DUMP_COLOR)
    assert (plugin.dump(abi.DUMP_COLOR).astype(np.float32).reshape(-1, 4)[:, 3] > 0).mean() > 0.05
    plugin.close()
