"""The composite (K20) against the oracle, through the C ABI.

composition_pass (src/nodes/composite.rs:19-131) runs strand_composite.wgsl:12-33
and blends its output with BlendState::ALPHA_BLENDING onto the destination
image loaded with LoadOp::Load. The destination is an image of its own
(post_process_write().destination), so the rule both implementations follow
is: out = frag * frag.a + dst * (1 - frag.a), dst = what `out` held before the
pass; compositing in place (out == scene colour) makes dst the scene colour.

The cases cover a scene alpha below 1, scene depths in front of and behind
the strands and none at all, RGBA16F and RGBA32F colour images and an R32F
depth image, all with padded row pitches, a destination distinct from the
scene image, the in-place form, the fused frame graph and the host-buffer
entry point. Colour is compared within max-abs 2e-3 and PSNR >= 50 dB.
"""
import ctypes as C

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from common import build_scene, psnr, run_gpu, run_ref

pytestmark = pytest.mark.gpu

TOL_ABS = 2e-3
TOL_PSNR = 50.0
PAD = 48  # bytes of padding per row: a multiple of every pixel size


def _row_bytes(w, fmt):
    return w * {abi.FMT_RGBA16F: 8, abi.FMT_RGBA32F: 16, abi.FMT_R32F: 4}[fmt]


def _encode(arr, fmt):
    h, w = arr.shape[:2]
    if fmt == abi.FMT_RGBA16F:
        return np.ascontiguousarray(arr, np.float16).reshape(h, -1).view(np.uint8)
    return np.ascontiguousarray(arr, np.float32).reshape(h, -1).view(np.uint8)


def _decode(rows, w, fmt):
    h = rows.shape[0]
    if fmt == abi.FMT_RGBA16F:
        return rows.copy().view(np.float16).astype(np.float32).reshape(h, w, 4)
    if fmt == abi.FMT_RGBA32F:
        return rows.copy().view(np.float32).reshape(h, w, 4)
    return rows.copy().view(np.float32).reshape(h, w)


class DeviceImage:
    """A padded-pitch device image; the padding holds 0xA5 and must survive."""

    def __init__(self, arr, fmt):
        import torch
        h, w = arr.shape[:2]
        self.h, self.w, self.fmt = h, w, fmt
        self.row = _row_bytes(w, fmt)
        self.pitch = self.row + PAD
        host = np.full((h, self.pitch), 0xA5, np.uint8)
        host[:, : self.row] = _encode(arr, fmt)
        self.t = torch.from_numpy(host).cuda()
        self.img = abi.Image(C.c_void_p(self.t.data_ptr()), w, h, self.pitch, fmt)

    def read(self):
        host = self.t.cpu().numpy()
        assert np.all(host[:, self.row:] == 0xA5), "the composite wrote into the row padding"
        return _decode(host[:, : self.row], self.w, self.fmt)


def _as_stored(arr, fmt):
    """The values an image of `fmt` holds for arr (binary16 rounding for RGBA16F)."""
    return arr.astype(np.float16).astype(np.float32) if fmt == abi.FMT_RGBA16F else arr.astype(np.float32)


def _scene_images(strand_depth, seed):
    """Seeded scene colour (alpha in [0.2, 1], a quarter exactly 1), scene depth
    and destination. Over strand pixels the scene depth is half (behind the
    strands, reversed-Z) or 1.5x (in front) the strand depth, or 0; over empty
    pixels it is 0 or in (0, 1)."""
    rng = np.random.default_rng(seed)
    h, w = strand_depth.shape
    color = rng.uniform(0.0, 1.0, (h, w, 4)).astype(np.float32)
    color[..., 3] = rng.uniform(0.2, 1.0, (h, w))
    color[rng.random((h, w)) < 0.25, 3] = 1.0
    pick = rng.integers(0, 3, (h, w))
    depth = np.where(pick == 0, strand_depth * np.float32(0.5),
                     np.where(pick == 1, strand_depth * np.float32(1.5), np.float32(0.0))).astype(np.float32)
    empty = strand_depth == 0.0
    depth[empty] = np.where(rng.random(int(empty.sum())) < 0.5, 0.0, rng.uniform(0.01, 1.0, int(empty.sum())))
    dest = rng.uniform(0.0, 1.0, (h, w, 4)).astype(np.float32)
    return color, depth.astype(np.float32), dest


def _check(got, want, what):
    g, r = got.reshape(-1), want.reshape(-1)
    assert np.all(np.isfinite(g)), f"{what}: non-finite output"
    err = float(np.max(np.abs(g - r)))
    p = psnr(g, r)
    assert err <= TOL_ABS and p >= TOL_PSNR, f"{what}: max abs {err:.3g}, PSNR {p:.1f} dB"


def _frame(name="tiny", **kw):
    scene = build_scene(name, settings_overrides={"history_enabled": 0}, **kw)
    plugin = run_gpu(scene)
    ref = run_ref(scene)
    h, w = scene.camera_cfg.screen_height, scene.camera_cfg.screen_width
    strand_depth = plugin.dump(abi.DUMP_DEPTH).reshape(h, w).astype(np.float32)
    assert (strand_depth > 0).sum() > 100, "the frame must cover pixels for the depth test to mean anything"
    return scene, plugin, ref, strand_depth


@pytest.mark.parametrize("fmt", [abi.FMT_RGBA16F, abi.FMT_RGBA32F])
def test_composite_matches_oracle(fmt):
    import torch
    scene, plugin, ref, strand_depth = _frame()
    color, depth, dest = _scene_images(strand_depth, seed=21 + fmt)
    color, dest = _as_stored(color, fmt), _as_stored(dest, fmt)
    half = fmt == abi.FMT_RGBA16F
    sc, sd, out = DeviceImage(color, fmt), DeviceImage(depth, abi.FMT_R32F), DeviceImage(dest, fmt)
    plugin.composition_pass(sc.img, sd.img, out.img)
    torch.cuda.synchronize()
    _check(out.read(), ref.composite(color, depth, dest, half_out=half), "composite onto a distinct destination")
    # Both sides of the depth test and the alpha blend were exercised.
    front = depth > strand_depth
    covered = (strand_depth > 0) & ~front
    assert front.sum() > 100 and covered.sum() > 100 and (color[..., 3] < 1).sum() > 100

    # No scene depth: every strand pixel blends.
    out2 = DeviceImage(dest, fmt)
    plugin.composition_pass(sc.img, None, out2.img)
    torch.cuda.synchronize()
    _check(out2.read(), ref.composite(color, None, dest, half_out=half), "composite without a scene depth")

    # In place: the destination is the scene colour itself.
    plugin.composition_pass(sc.img, sd.img, sc.img)
    torch.cuda.synchronize()
    _check(sc.read(), ref.composite(color, depth, None, half_out=half), "composite in place")
    assert np.array_equal(sd.read(), depth), "the scene depth must not change"
    plugin.close()


def test_composite_fused_frame_matches_oracle():
    # fiber_frame_fused: the scene depth also drives the opaque-tile cull, and
    # the composite blends onto a destination distinct from the scene image.
    import torch
    scene, plugin, _, strand_depth = _frame()
    color, depth, dest = _scene_images(strand_depth, seed=5)
    color, dest = _as_stored(color, abi.FMT_RGBA16F), _as_stored(dest, abi.FMT_RGBA16F)
    sc, sd = DeviceImage(color, abi.FMT_RGBA16F), DeviceImage(depth, abi.FMT_R32F)
    out = DeviceImage(dest, abi.FMT_RGBA16F)
    run_gpu(scene, plugin=plugin, fused=True, scene_color=sc.img, scene_depth=sd.img, out=out.img)
    torch.cuda.synchronize()
    ref = run_ref(scene, opaque_depth=depth)
    s, rs = plugin.stats(), ref.stats()
    assert s.fine_refs == rs.fine_refs
    _check(out.read(), ref.composite(color, depth, dest), "fused frame composite")
    plugin.close()


def test_render_host_matches_oracle():
    # fiber_render_host composites in place over the uploaded scene image.
    scene, plugin, _, strand_depth = _frame(width=200, height=152)
    h, w = strand_depth.shape
    color, depth, _ = _scene_images(strand_depth, seed=9)
    color = _as_stored(color, abi.FMT_RGBA16F)
    host_in = np.ascontiguousarray(color.astype(np.float16))
    host_depth = np.ascontiguousarray(depth)
    host_out = np.zeros_like(host_in)
    plugin.frame_begin_raw(scene.camera_cfg, scene.cam, scene.light_cfgs, scene.lights_c)
    abi.check(plugin.lib.fiber_render_host(plugin.ctx, C.c_void_p(host_in.ctypes.data),
                                           C.c_void_p(host_depth.ctypes.data), C.c_void_p(host_out.ctypes.data),
                                           None), "fiber_render_host")
    import torch
    torch.cuda.synchronize()
    ref = run_ref(scene, scene_color=color, scene_depth=depth, opaque_depth=depth)
    want = ref.get(100, np.dtype("<f4")).reshape(h, w, 4)
    _check(host_out.astype(np.float32), want, "fiber_render_host")
    _check(host_out.astype(np.float32), ref.composite(color, depth, None), "fiber_render_host (in place)")
    plugin.close()
