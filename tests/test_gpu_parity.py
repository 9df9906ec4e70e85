"""CUDA path vs the oracle on identical seeded inputs, through the C ABI.

Integer and index outputs (frustum table, coarse ranges, keep probabilities,
depth-warp LUT, binning tasks, projected segments, page table and metadata,
froxel counts, prefix offsets, canonical fine refs, active tiles, raster work
items, tile runs, per-pixel fragment counts) must match bit for bit. Shaded
colour, shading atlas and deep-shadow opacity must agree within max-abs 2e-3
and PSNR >= 50 dB in FP32 (the DOM stages use no transcendental functions and
are compared exactly).
"""
import ctypes as C

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from common import build_scene, psnr, run_gpu, run_ref

pytestmark = pytest.mark.gpu

TOL_ABS = 2e-3
TOL_PSNR = 50.0

EXACT = [
    abi.DUMP_FRUSTA, abi.DUMP_RANGES, abi.DUMP_KEEP, abi.DUMP_LUT, abi.DUMP_TASKS, abi.DUMP_PROJECTED,
    abi.DUMP_PAGE_TABLE, abi.DUMP_PAGE_META, abi.DUMP_COUNTS, abi.DUMP_OFFSETS, abi.DUMP_REFS,
    abi.DUMP_ACTIVE_TILES, abi.DUMP_WORK, abi.DUMP_RUNS, abi.DUMP_DOM_DEPTH, abi.DUMP_DOM_OPACITY,
    abi.DUMP_SHADOW_MAP, abi.DUMP_FRAGMENTS, abi.DUMP_OPAQUE_TILES,
]
NAMES = {v: k for k, v in vars(abi).items() if k.startswith("DUMP_") and isinstance(v, int)}


def _exact(gpu, ref, what):
    g = gpu.view(np.uint8)
    r = ref.view(np.uint8)
    assert g.shape == r.shape, f"{NAMES[what]}: size {g.shape} vs oracle {r.shape}"
    if not np.array_equal(g, r):
        gv, rv = gpu.reshape(-1), ref.reshape(-1)
        bad = np.nonzero(gv != rv)[0]
        raise AssertionError(f"{NAMES[what]}: {bad.size} of {gv.size} records differ; first {bad[:5]}: "
                             f"gpu {gv[bad[:3]]} oracle {rv[bad[:3]]}")


def _close(gpu, ref, what, mask=None):
    g = gpu.astype(np.float32).reshape(-1)
    r = ref.astype(np.float32).reshape(-1)
    assert g.shape == r.shape
    if mask is not None:
        g, r = g[mask], r[mask]
    assert np.array_equal(np.isnan(g), np.isnan(r)), f"{NAMES[what]}: NaN pattern differs"
    ok = ~np.isnan(g)
    err = float(np.max(np.abs(g[ok] - r[ok]))) if ok.any() else 0.0
    p = psnr(g[ok], r[ok]) if ok.any() else float("inf")
    assert err <= TOL_ABS and p >= TOL_PSNR, f"{NAMES[what]}: max abs {err:.3g}, PSNR {p:.1f} dB"
    return err, p


def _compare(scene, fused=False, gpu_kw=None, ref_kw=None):
    plugin = run_gpu(scene, fused=fused, **(gpu_kw or {}))
    ref = run_ref(scene, **(ref_kw or {}))
    s = plugin.stats()
    rs = ref.stats()
    for k in ("binning_tasks", "camera_tasks", "allocated_pages", "fine_refs", "active_tiles", "camera_runs",
              "shadow_runs", "work_items", "overflow_flags"):
        assert getattr(s, k) == getattr(rs, k), f"stat {k}: gpu {getattr(s, k)} oracle {getattr(rs, k)}"
    for what in EXACT:
        if what == abi.DUMP_FRAGMENTS and not scene.settings.fragment_counts_enabled:
            continue
        _exact(plugin.dump(what), ref.get(what), what)
    # Shading atlas / history: compare the texels this frame wrote.
    ga, ra = plugin.dump(abi.DUMP_ATLAS).reshape(-1, 4), ref.get(abi.DUMP_ATLAS).reshape(-1, 4)
    written = ra.astype(np.float32)[:, 3] > 0
    _close(ga[written], ra[written], abi.DUMP_ATLAS)
    gh, rh = plugin.dump(abi.DUMP_HISTORY).reshape(-1, 2), ref.get(abi.DUMP_HISTORY).reshape(-1, 2)
    _close(gh[written], rh[written], abi.DUMP_HISTORY)
    _close(plugin.dump(abi.DUMP_COLOR), ref.get(abi.DUMP_COLOR), abi.DUMP_COLOR)
    _close(plugin.dump(abi.DUMP_DEPTH), ref.get(abi.DUMP_DEPTH), abi.DUMP_DEPTH)
    plugin.close()
    return s


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_parity_default(name):
    scene = build_scene(name, settings_overrides={"fragment_counts_enabled": 1})
    s = _compare(scene)
    assert s.binning_tasks > 0 and s.fine_refs > 0 and s.camera_runs > 0 and s.shadow_runs > 0


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_parity_page_csr_backend(name):
    # FineBinningBackend::PageCsr: visits grouped by page, cells built per page;
    # the same canonical counts, offsets, refs and images as the default.
    scene = build_scene(name, settings_overrides={"fragment_counts_enabled": 1, "fine_binning_backend": 1})
    s = _compare(scene)
    assert s.fine_refs > 0 and s.camera_runs > 0 and s.shadow_runs > 0


def test_parity_page_csr_fused_and_overflow():
    # The page CSR inside the captured frame graph, then with a reference
    # budget too small for the visit records (the walking fallback).
    _compare(build_scene("tiny", frame=5, settings_overrides={"fine_binning_backend": 1}), fused=True)
    scene = build_scene("tiny", settings_overrides={"ref_capacity_factor": 1, "fine_binning_backend": 1})
    plugin = run_gpu(scene)
    ref = run_ref(scene)
    s = plugin.stats(allow_overflow=True)
    assert s.overflow_flags & 4 and ref.stats().overflow_flags & 4
    for what in (abi.DUMP_PAGE_META, abi.DUMP_COUNTS, abi.DUMP_OFFSETS, abi.DUMP_ACTIVE_TILES, abi.DUMP_RUNS,
                 abi.DUMP_WORK):
        _exact(plugin.dump(what), ref.get(what), what)
    plugin.close()


@pytest.mark.parametrize("backend", [0, 1])
def test_telemetry_matches_oracle(backend):
    # PrepassTelemetrySettings on: the telemetry image matches the oracle's word
    # for word on both binning backends, and the frame itself is unchanged.
    scene = build_scene("small", settings_overrides={"telemetry_enabled": 1, "fine_binning_backend": backend,
                                                      "fragment_counts_enabled": 1})
    plugin = run_gpu(scene)
    ref = run_ref(scene)
    got, want = bytes(plugin.telemetry()), bytes(ref.telemetry())
    gw, rw = np.frombuffer(got, np.uint32), np.frombuffer(want, np.uint32)
    bad = np.nonzero(gw != rw)[0]
    assert bad.size == 0, f"telemetry words differ at {bad[:8]}: gpu {gw[bad[:8]]} oracle {rw[bad[:8]]}"
    assert gw[2] > 0 and gw[4] > 0
    for what in (abi.DUMP_COUNTS, abi.DUMP_REFS, abi.DUMP_RUNS, abi.DUMP_FRAGMENTS, abi.DUMP_DOM_OPACITY):
        _exact(plugin.dump(what), ref.get(what), what)
    plugin.close()


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_parity_sparse_dom(name):
    # Sparse DOM residency with a pool that holds every requested page: the
    # same DOM, shadow map and images as the dense layers.
    scene = build_scene(name, settings_overrides={"dom_page_pool": 64, "fragment_counts_enabled": 1})
    s = _compare(scene)
    assert s.overflow_flags == 0 and s.shadow_runs > 0


def test_sparse_dom_pool_overflow():
    # A pool of half the light's 16 pages: the frame flags the DOM pool
    # overflow (bit 4); the resident pages (the first requested ones in
    # page-table order) match the dense DOM texel for texel, the rest is empty.
    scene = build_scene("small", settings_overrides={"dom_page_pool": 8})
    plugin = run_gpu(scene)
    ref = run_ref(scene)
    s = plugin.stats(allow_overflow=True)
    assert s.overflow_flags & 16
    gd, rd = plugin.dump(abi.DUMP_DOM_DEPTH), ref.get(abi.DUMP_DOM_DEPTH)
    stored = gd != 0.0
    assert 0 < int(stored.sum()) < int((rd != 0.0).sum())
    assert np.array_equal(gd[stored], rd[stored])
    go = plugin.dump(abi.DUMP_DOM_OPACITY).reshape(-1, gd.size)
    ro = ref.get(abi.DUMP_DOM_OPACITY).reshape(-1, gd.size)
    assert np.array_equal(go[:, stored], ro[:, stored])
    plugin.close()


def test_parity_fused_graph():
    scene = build_scene("tiny", settings_overrides={"fragment_counts_enabled": 1})
    _compare(scene, fused=True)


def test_parity_unsaturated_shading():
    # A dim light keeps the shaded colour inside (0, 1) so the Marschner terms
    # are compared before the unorm clamp.
    scene = build_scene("tiny", illuminance=0.02)
    _compare(scene)


def _materials():
    from bevy_strand_rasterizer_b200.plugin import StrandMaterial
    return {
        # Narrow lobes: a sharp longitudinal term and a tight azimuthal detector.
        "narrow": StrandMaterial(absorption_color=(0.2, 0.5, 0.9, 0.6), specular_color=(0.9, 0.8, 0.7, 0.5),
                                 ambient_factor=0.2, ao_factor=0.3, eta=1.3, beta=0.15, alpha=0.12, shift=-0.05),
        # Wide lobes, a dense medium and thicker strands.
        "wide": StrandMaterial(absorption_color=(0.95, 0.1, 0.3, 0.25), specular_color=(0.4, 1.0, 0.6, 1.0),
                               ambient_factor=0.02, ao_factor=0.05, eta=2.1, beta=1.0, alpha=0.6, shift=0.12,
                               min_radius_pixels=0.8, max_radius_pixels=3.0),
    }


@pytest.mark.parametrize("name,illuminance", [("narrow", 100.0), ("wide", 400.0)])
def test_parity_materials(name, illuminance):
    # Non-default BCSDF parameters and radii, lit so that the shaded texels
    # spread over (0, 1) with the narrow highlight reaching 1: the shading's
    # lobes and the rasters' coverage on other inputs.
    scene = build_scene("tiny", illuminance=illuminance, material=_materials()[name])
    _compare(scene)


def test_parity_two_instances():
    # A second instance of the same strands, rotated 30 degrees about y, scaled
    # by 0.8 and moved, with its own material: per-instance transforms,
    # materials and keep probabilities.
    scene = build_scene("tiny", illuminance=100.0)
    packed, _, _ = scene.assets[0]
    a, s = np.radians(30.0), 0.8
    m = np.zeros(16, np.float32)  # column-major world_from_local
    m[0], m[2], m[8], m[10] = s * np.cos(a), -s * np.sin(a), s * np.sin(a), s * np.cos(a)
    m[5], m[15] = s, 1.0
    m[12], m[13], m[14] = 0.04, 0.02, -0.03
    scene.assets.append((packed, _materials()["narrow"], m))
    s_ = _compare(scene)
    assert s_.binning_tasks > 0


def test_parity_no_cull_two_lights_orbit():
    scene = build_scene("tiny", frame=37, cull=False, lights=[(1.0, 1.0, 1.0), (-1.0, 1.0, 0.5)])
    _compare(scene)


def test_parity_ref_overflow():
    # A tiny reference budget overflows pages exactly like the oracle's.
    scene = build_scene("tiny", settings_overrides={"ref_capacity_factor": 1})
    plugin = run_gpu(scene)
    ref = run_ref(scene)
    s = plugin.stats(allow_overflow=True)
    assert s.overflow_flags & 4 and ref.stats().overflow_flags & 4
    for what in (abi.DUMP_PAGE_META, abi.DUMP_COUNTS, abi.DUMP_ACTIVE_TILES, abi.DUMP_RUNS, abi.DUMP_WORK):
        _exact(plugin.dump(what), ref.get(what), what)
    plugin.close()


def _depth_image(depth: np.ndarray):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(depth, np.float32)).cuda()
    h, w = depth.shape[:2]
    img = abi.Image(C.c_void_p(t.data_ptr()), w, h, t[0].numel() * 4, abi.FMT_R32F)
    return t, img


@pytest.mark.parametrize("samples", [1, 4])
def test_parity_opaque_depth(samples):
    # K0 + the prepass cull: an opaque wall at the strands' median depth over
    # part of the screen (and, at 4 samples, holes that leave tiles uncovered).
    from common import opaque_plane
    scene = build_scene("tiny", settings_overrides={"fragment_counts_enabled": 1})
    cfg = scene.camera_cfg
    depth = opaque_plane(cfg.screen_width, cfg.screen_height, 0.2, samples, seed=3)
    keep, img = _depth_image(depth)
    s = _compare(scene, gpu_kw=dict(opaque_depth=img, opaque_samples=samples),
                 ref_kw=dict(opaque_depth=depth, opaque_samples=samples))
    base = run_ref(scene).stats()
    assert 0 < s.fine_refs < base.fine_refs
    del keep


def test_parity_opaque_depth_fused():
    # fiber_frame_fused reduces its scene_depth (1 sample) ahead of the
    # prepass; the next frame without a depth must cull nothing again.
    from common import opaque_plane
    scene = build_scene("tiny", settings_overrides={"fragment_counts_enabled": 1, "history_enabled": 0})
    cfg = scene.camera_cfg
    depth = opaque_plane(cfg.screen_width, cfg.screen_height, 0.2, 1, seed=5)[:, :, 0]
    keep, img = _depth_image(depth)
    _compare(scene, fused=True, gpu_kw=dict(scene_depth=img), ref_kw=dict(opaque_depth=depth))
    p = run_gpu(scene, fused=True, scene_depth=img)
    culled = p.stats().fine_refs
    run_gpu(scene, plugin=p, fused=True)
    ref = run_ref(scene)
    assert p.stats().fine_refs == ref.stats().fine_refs > culled
    _exact(p.dump(abi.DUMP_REFS), ref.get(abi.DUMP_REFS), abi.DUMP_REFS)
    _exact(p.dump(abi.DUMP_OPAQUE_TILES), ref.get(abi.DUMP_OPAQUE_TILES), abi.DUMP_OPAQUE_TILES)
    p.close()
    del keep


def test_fused_graph_follows_frame_shape():
    # One context replays its captured frame graph on a stream while the frame
    # shape changes (resolution, light count) and the composite keeps writing
    # into the same backing buffers. Every frame must match a fresh context
    # that renders it with the plain node sequence.
    import torch
    from bevy_strand_rasterizer_b200.plugin import StrandRasterizerPlugin  # noqa: F401

    stream = torch.cuda.Stream()
    scene_buf = torch.empty((240 * 320 * 4,), dtype=torch.float16, device="cuda")
    out_buf = torch.empty_like(scene_buf)

    def images(w, h):
        scene_buf.zero_()
        scene_buf[: w * h * 4].view(h, w, 4)[...] = torch.tensor([0.1, 0.2, 0.3, 1.0], dtype=torch.float16)
        out_buf.zero_()
        torch.cuda.synchronize()
        return (abi.Image(C.c_void_p(scene_buf.data_ptr()), w, h, w * 8, abi.FMT_RGBA16F),
                abi.Image(C.c_void_p(out_buf.data_ptr()), w, h, w * 8, abi.FMT_RGBA16F))

    shapes = [dict(width=320, height=240), dict(width=160, height=120),
              dict(width=200, height=152, lights=[(1.0, 1.0, 1.0), (-1.0, 1.0, 0.5)]), dict(width=320, height=240)]
    p = None
    for kw in shapes:
        scene = build_scene("tiny", settings_overrides={"history_enabled": 0, "fragment_counts_enabled": 1}, **kw)
        w, h = kw["width"], kw["height"]
        sc, out = images(w, h)
        with torch.cuda.stream(stream):
            p = run_gpu(scene, plugin=p, fused=True, stream=stream, scene_color=sc, out=out)
        stream.synchronize()
        got = out_buf[: w * h * 4].cpu().numpy().copy()
        dumps = {what: p.dump(what).copy() for what in (abi.DUMP_COLOR, abi.DUMP_FRAGMENTS, abi.DUMP_DOM_OPACITY)}
        sc, out = images(w, h)
        fresh = run_gpu(scene, scene_color=sc, out=out)
        torch.cuda.synchronize()
        want = out_buf[: w * h * 4].cpu().numpy()
        assert np.array_equal(got.view(np.uint16), want.view(np.uint16)), f"composite differs at {w}x{h}"
        for what, v in dumps.items():
            assert np.array_equal(v.view(np.uint8), fresh.dump(what).view(np.uint8)), f"{NAMES[what]} at {w}x{h}"
        fresh.close()
    p.close()


def test_deterministic_repeat():
    # History off: with it on, frame 2 legitimately blends frame 1's visibility.
    scene = build_scene("small", settings_overrides={"history_enabled": 0})
    p = run_gpu(scene)
    first = {w: p.dump(w).copy() for w in (abi.DUMP_REFS, abi.DUMP_WORK, abi.DUMP_COLOR, abi.DUMP_DOM_OPACITY)}
    for _ in range(2):
        run_gpu(scene, plugin=p)
        for w, v in first.items():
            assert np.array_equal(p.dump(w).view(np.uint8), v.view(np.uint8)), NAMES[w]
    p.close()
