"""Parity on the full workload configurations, through the C ABI.

- the whole medium frame (100,000 strands x 32 points, 1920x1080 camera,
  2048^2 x 8 deep-opacity map), exact against the oracle: every integer dump
  bit for bit, colour, atlas, history and depth within max-abs 2e-3 and
  PSNR >= 50 dB;
- the large configuration's frame shape (curly strands, 3840x2160 camera, two
  4096^2 x 8 maps) on a subset of its strands, with the reference's reference
  capacity factor of 4: the overflow flags match the oracle's, and so does
  every dump the overflow leaves defined;
- the served configuration's request shapes (odd sizes, 0-2 lights, 128^2
  maps, cameras around the scene) rendered by the request server, against the
  oracle's composite of the same request;
- a 500,000-strand scene served at 1920x1080 from close cameras: no request
  returns EOVERFLOW, and a request whose references outgrew the slot's
  capacity matches the oracle run with room for all of them.
"""
import ctypes as C

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from common import build_scene, psnr, run_gpu, run_ref
from test_gpu_parity import EXACT, _close, _compare, _exact

pytestmark = pytest.mark.gpu

TOL_ABS = 2e-3
TOL_PSNR = 50.0


def test_parity_full_medium_frame():
    scene = build_scene("medium", settings_overrides={"fragment_counts_enabled": 1})
    s = _compare(scene)
    assert s.fine_refs > 20_000_000 and s.overflow_flags == 0 and s.shadow_runs > 10_000


def test_parity_large_frame_shape_subset():
    # Curly strands at 3840x2160 with two 4096^2 x 8 maps; 60,000 of the
    # configuration's 500,000 strands keep the oracle within seconds.
    scene = build_scene("large", strands=60_000, settings_overrides={"fragment_counts_enabled": 1})
    assert scene.settings.ref_capacity_factor == 4
    plugin = run_gpu(scene)
    ref = run_ref(scene)
    s = plugin.stats(allow_overflow=True)
    rs = ref.stats()
    for k in ("binning_tasks", "camera_tasks", "allocated_pages", "fine_refs", "active_tiles", "camera_runs",
              "shadow_runs", "work_items", "overflow_flags", "refs_requested"):
        assert getattr(s, k) == getattr(rs, k), f"stat {k}: gpu {getattr(s, k)} oracle {getattr(rs, k)}"
    assert list(s.frustum_refs)[:3] == list(rs.frustum_refs)[:3]
    if s.overflow_flags:
        # Pages that did not fit are flagged and dropped exactly where the
        # oracle drops them.
        for what in (abi.DUMP_PAGE_META, abi.DUMP_COUNTS, abi.DUMP_ACTIVE_TILES, abi.DUMP_RUNS, abi.DUMP_WORK,
                     abi.DUMP_TASKS, abi.DUMP_PROJECTED):
            _exact(plugin.dump(what), ref.get(what), what)
    else:
        for what in EXACT:
            _exact(plugin.dump(what), ref.get(what), what)
        _close(plugin.dump(abi.DUMP_COLOR), ref.get(abi.DUMP_COLOR), abi.DUMP_COLOR)
    plugin.close()


def _oracle_composite(packed, cfg, cam, lcfg, lights, bg, settings):
    from bevy_strand_rasterizer_b200.plugin import StrandMaterial
    from oracle_bridge import run_oracle
    ident = np.eye(4, dtype=np.float32).reshape(16)
    ref = run_oracle([(packed, StrandMaterial(), ident)], cfg, cam, lcfg, lights, settings,
                     scene_color=bg.astype(np.float32))
    h, w = bg.shape[:2]
    return ref, ref.get(100, np.dtype("<f4")).reshape(h, w, 4)


def _served_settings():
    st = abi.default_settings()
    st.history_enabled = 0
    return st


def _check_image(got, want, what):
    g, r = got.astype(np.float32).reshape(-1), want.reshape(-1)
    err = float(np.max(np.abs(g - r)))
    p = psnr(g, r)
    assert err <= TOL_ABS and p >= TOL_PSNR, f"{what}: max abs {err:.3g}, PSNR {p:.1f} dB"


def test_served_request_shapes_match_oracle():
    from bevy_strand_rasterizer_b200.plugin import StrandMaterial, pack_strand_set
    from bevy_strand_rasterizer_b200.scene import scalp_hair
    from bevy_strand_rasterizer_b200.server import FiberServer
    from test_server import _background, _request
    scenes = [pack_strand_set(scalp_hair(n, p, seed, curly=curly))
              for n, p, curly, seed in ((300, 8, False, 7), (1500, 16, True, 11), (4000, 32, False, 13))]
    srv = FiberServer(slots=3, max_width=320, max_height=256, max_lights=2, max_dom=128,
                      settings=_served_settings())
    ids = [srv.add_scene(p, StrandMaterial()) for p in scenes]
    srv.start()
    rng = np.random.default_rng(17)
    shapes = [(96, 128), (200, 152), (250, 170), (64, 64), (320, 256), (130, 98), (256, 200), (160, 120)]
    jobs = []
    for k, (w, h) in enumerate(shapes):
        si = k % len(scenes)
        n_lights = k % 3
        cfg, cam, lcfg, lights = _request(scenes[si], rng, w, h, n_lights)
        bg = _background(w, h)
        bg[: h // 2, :, 3] = np.float16(0.5)  # a scene alpha below 1 over the top half
        out = np.zeros_like(bg)
        jobs.append((srv.submit(ids[si], cfg, cam, lcfg, lights, out, scene_rgba16f=bg), si, cfg, cam, lcfg,
                     lights, bg, out))
    results = [(srv.wait(t, allow_overflow=False), rest) for t, *rest in jobs]
    srv.close()
    for res, (si, cfg, cam, lcfg, lights, bg, out) in results:
        assert res.status == abi.OK
        _, want = _oracle_composite(scenes[si], cfg, cam, lcfg, lights, bg, _served_settings())
        what = f"{cfg.screen_width}x{cfg.screen_height}, {len(lcfg)} light(s), scene {si}"
        _check_image(out, want, what)
        assert (out.astype(np.float32) != bg.astype(np.float32)).any(), f"{what}: no strand pixel"


def test_served_large_scene_never_overflows():
    # The configuration's largest resident scene at the largest resolution,
    # seen from close up: the slot grows its reference capacity and renders
    # again instead of returning a truncated image.
    from bevy_strand_rasterizer_b200.plugin import FroxelConfig, StrandMaterial, pack_strand_set
    from bevy_strand_rasterizer_b200.scene import CameraSpec, LightSpec, scalp_hair
    from bevy_strand_rasterizer_b200.server import FiberServer
    packed = pack_strand_set(scalp_hair(500_000, 32, 1007, curly=True))
    srv = FiberServer(slots=2, max_width=1920, max_height=1080, max_lights=1, max_dom=1024,
                      settings=_served_settings())
    sid = srv.add_scene(packed, StrandMaterial())
    srv.start()
    jobs = []
    for k, (eye, dist) in enumerate((((0.0, 0.5, 1.0), 0.4), ((1.0, 0.3, 0.2), 0.45), ((-0.6, 0.8, 0.3), 0.5),
                                     ((0.2, 0.1, -1.0), 0.4))):
        e = np.asarray(eye, np.float64)
        e = e / np.linalg.norm(e) * dist
        spec = CameraSpec(eye=tuple(float(x) for x in e), width=1920, height=1080)
        cam = abi.Camera()
        cam.clip_from_world[:] = [float(x) for x in spec.clip_from_world()]
        cam.world_position[:] = [float(x) for x in spec.eye]
        light = LightSpec((1.0, 1.0, 1.0), size=1024)
        lights = (abi.Light * 1)()
        lights[0].clip_from_world[:] = [float(x) for x in light.clip_from_world(packed.aabb_min, packed.aabb_max)]
        lights[0].direction_to_light[:] = [float(x) for x in light.direction()]
        lights[0].color[:] = [float(x) for x in light.color4()]
        cfg, lcfg = FroxelConfig(1920, 1080, 8, 8, 64), [FroxelConfig(1024, 1024, 8, 8, 64)]
        bg = np.zeros((1080, 1920, 4), np.float16)
        bg[...] = np.array([0.05, 0.1, 0.2, 1.0], np.float16)
        out = np.zeros_like(bg)
        jobs.append((srv.submit(sid, cfg, cam, lcfg, lights, out, scene_rgba16f=bg), cfg, cam, lcfg, lights, bg, out))
    results = [(srv.wait(t, allow_overflow=False), rest) for t, *rest in jobs]
    srv.close()
    assert all(res.status == abi.OK for res, _ in results)
    # The first request that had to grow its slot (else the first request)
    # against the oracle given room for every reference.
    res, (cfg, cam, lcfg, lights, bg, out) = next(((r, x) for r, x in results if r.renders > 1), results[0])
    st = _served_settings()
    st.ref_capacity_factor = 64
    ref, want = _oracle_composite(packed, cfg, cam, lcfg, lights, bg, st)
    assert ref.stats().overflow_flags == 0
    _check_image(out, want, f"500k strands at 1920x1080 ({res.renders} render(s))")
