"""The request server (served mode): requests of different scenes, resolutions
and light counts, submitted at once so they overlap on the GPU, must render the
same image as each request rendered alone by a single context. Also checks
admission under an HBM budget and the rejection of oversized requests."""
import ctypes as C

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from bevy_strand_rasterizer_b200.plugin import FroxelConfig, StrandMaterial, StrandRasterizerPlugin, pack_strand_set
from bevy_strand_rasterizer_b200.scene import CameraSpec, LightSpec, scalp_hair

pytestmark = pytest.mark.gpu

SCENES = [(300, 8, False, 7), (900, 12, True, 11), (2000, 16, False, 13)]
LIGHT_DIRS = [(1.0, 1.0, 1.0), (-1.0, 1.0, 0.5)]


def _scenes():
    return [pack_strand_set(scalp_hair(n, p, seed, curly=curly)) for n, p, curly, seed in SCENES]


def _request(packed, rng, width, height, n_lights, dom=128):
    az = float(rng.uniform(0.0, 2.0 * np.pi))
    cam_spec = CameraSpec(eye=(0.6 * np.sin(az), 0.15, 0.6 * np.cos(az)), width=width, height=height)
    cam = abi.Camera()
    cam.clip_from_world[:] = [float(x) for x in cam_spec.clip_from_world()]
    cam.world_position[:] = [float(x) for x in cam_spec.eye]
    cfg = FroxelConfig(width, height, 8, 8, 32)
    light_cfgs = [FroxelConfig(dom, dom, 8, 8, 32) for _ in range(n_lights)]
    lights = (abi.Light * max(1, n_lights))()
    for i in range(n_lights):
        spec = LightSpec(LIGHT_DIRS[i], illuminance=10_000.0, size=dom)
        lights[i].clip_from_world[:] = [float(x) for x in spec.clip_from_world(packed.aabb_min, packed.aabb_max)]
        lights[i].direction_to_light[:] = [float(x) for x in spec.direction()]
        lights[i].color[:] = [float(x) for x in spec.color4()]
    return cfg, cam, light_cfgs, lights


def _background(width, height):
    bg = np.empty((height, width, 4), np.float16)
    bg[...] = np.array([0.05, 0.1, 0.2, 1.0], np.float16)
    return bg


def _alone(packed, cfg, cam, light_cfgs, lights, bg):
    st = abi.default_settings()
    st.history_enabled = 0
    p = StrandRasterizerPlugin()
    abi.check(p.lib.fiber_settings_set(p.ctx, C.byref(st)), "fiber_settings_set")
    p.add_geometry(packed, StrandMaterial())
    p.frame_begin_raw(cfg, cam, light_cfgs, lights, None)
    out = np.zeros_like(bg)
    abi.check(p.lib.fiber_render_host(p.ctx, C.c_void_p(bg.ctypes.data), None, C.c_void_p(out.ctypes.data), None),
              "fiber_render_host")
    p.stats()  # synchronises the context's stream
    p.close()
    return out


def test_served_results_match_alone():
    from bevy_strand_rasterizer_b200.server import FiberServer
    scenes = _scenes()
    srv = FiberServer(slots=3, max_width=320, max_height=240, max_lights=2, max_dom=128)
    ids = [srv.add_scene(p, StrandMaterial()) for p in scenes]
    assert srv.start() == 3
    rng = np.random.default_rng(5)
    shapes = [(64, 64), (320, 240), (160, 120), (200, 152), (96, 256 // 2), (320, 240), (128, 128), (256, 200)]
    jobs = []
    for k, (w, h) in enumerate(shapes * 2):
        si = int(rng.integers(0, len(scenes)))
        n_lights = int(rng.integers(0, 3))
        cfg, cam, lcfg, lights = _request(scenes[si], rng, w, h, n_lights)
        bg = _background(w, h)
        out = np.zeros_like(bg)
        t = srv.submit(ids[si], cfg, cam, lcfg, lights, out, scene_rgba16f=bg)
        jobs.append((t, si, cfg, cam, lcfg, lights, bg, out))
    slots_used = set()
    for t, *_ in jobs:
        slots_used.add(srv.wait(t).slot)
    srv.close()
    assert len(slots_used) > 1, "requests should spread over the slots"
    for t, si, cfg, cam, lcfg, lights, bg, out in jobs:
        want = _alone(scenes[si], cfg, cam, lcfg, lights, bg)
        assert np.array_equal(out.view(np.uint16), want.view(np.uint16)), \
            f"request {t} ({cfg.screen_width}x{cfg.screen_height}, scene {si}) differs from its lone render"
        assert (out.astype(np.float32) != bg.astype(np.float32)).any(), "strands should cover some pixels"


def test_budget_limits_slots_and_rejects_oversized_requests():
    from bevy_strand_rasterizer_b200.server import FiberServer
    packed = _scenes()[0]
    srv = FiberServer(slots=4, max_width=160, max_height=120, max_lights=1, max_dom=128, hbm_budget=1)
    sid = srv.add_scene(packed, StrandMaterial())
    assert srv.start() == 1  # a budget below one sized slot still admits one
    rng = np.random.default_rng(1)
    cfg, cam, lcfg, lights = _request(packed, rng, 320, 240, 1)
    out = np.zeros((240, 320, 4), np.float16)
    with pytest.raises(abi.FiberError) as e:
        srv.submit(sid, cfg, cam, lcfg, lights, out)
    assert e.value.status == abi.EINVAL
    cfg, cam, lcfg, lights = _request(packed, rng, 160, 120, 1)
    out = np.zeros((120, 160, 4), np.float16)
    srv.wait(srv.submit(sid, cfg, cam, lcfg, lights, out))
    srv.close()


def test_render_host_back_to_back():
    # fiber_render_host uploads the scene image on a copy stream beside the
    # frame; two calls queued back to back with different images (and a scene
    # depth on the second) must each equal the same frame rendered alone.
    import torch
    scenes = _scenes()
    rng = np.random.default_rng(11)
    cfg, cam, lcfg, lights = _request(scenes[0], rng, 160, 120, 1)
    bg_a = _background(160, 120)
    bg_b = bg_a.copy()
    bg_b[...] = np.array([0.3, 0.2, 0.1, 1.0], np.float16)
    depth = np.zeros((120, 160), np.float32)
    depth[:, :80] = 1e-3  # a far opaque wall over the left half
    want_a = _alone(scenes[0], cfg, cam, lcfg, lights, bg_a)
    st = abi.default_settings()
    st.history_enabled = 0
    p = StrandRasterizerPlugin()
    abi.check(p.lib.fiber_settings_set(p.ctx, C.byref(st)), "fiber_settings_set")
    p.add_geometry(scenes[0], StrandMaterial())
    stream = torch.cuda.Stream()
    h = C.c_void_p(stream.cuda_stream)
    pinned = [torch.from_numpy(x).pin_memory() for x in (bg_a, bg_b, depth)]
    outs = [torch.zeros((120, 160, 4), dtype=torch.float16).pin_memory() for _ in range(2)]
    p.frame_begin_raw(cfg, cam, lcfg, lights, stream)
    abi.check(p.lib.fiber_render_host(p.ctx, C.c_void_p(pinned[0].data_ptr()), None, C.c_void_p(outs[0].data_ptr()), h),
              "fiber_render_host")
    p.frame_begin_raw(cfg, cam, lcfg, lights, stream)
    abi.check(p.lib.fiber_render_host(p.ctx, C.c_void_p(pinned[1].data_ptr()), C.c_void_p(pinned[2].data_ptr()),
                                      C.c_void_p(outs[1].data_ptr()), h), "fiber_render_host")
    stream.synchronize()
    assert np.array_equal(outs[0].numpy().view(np.uint16), want_a.view(np.uint16))
    # the second frame alone: the same scene image and depth through fresh calls
    q = StrandRasterizerPlugin()
    abi.check(q.lib.fiber_settings_set(q.ctx, C.byref(st)), "fiber_settings_set")
    q.add_geometry(scenes[0], StrandMaterial())
    q.frame_begin_raw(cfg, cam, lcfg, lights, None)
    want_b = np.zeros_like(bg_b)
    abi.check(q.lib.fiber_render_host(q.ctx, C.c_void_p(bg_b.ctypes.data), C.c_void_p(depth.ctypes.data),
                                      C.c_void_p(want_b.ctypes.data), None), "fiber_render_host")
    q.stats()
    assert np.array_equal(outs[1].numpy().view(np.uint16), want_b.view(np.uint16))
    assert not np.array_equal(outs[0].numpy().view(np.uint16), outs[1].numpy().view(np.uint16))
    p.close()
    q.close()
