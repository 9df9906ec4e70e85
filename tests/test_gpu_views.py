"""Multi-view frames (fiber_frame_begin_views): several independent views —
each its own strand set, camera, resolution and lights — rendered by one frame
whose kernels cover every view at once, with each view's work at offsets from
the frame's single prefix sums. Every view's colour, depth, fragment counts,
deep-opacity layers, shadow map and shading atlas must equal, bit for bit, the
same view rendered alone by its own context (node sequence and fused graph,
two frames in a row)."""
import ctypes as C

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi

pytestmark = pytest.mark.gpu

SCENES = [(300, 8, False, 7), (900, 12, True, 11), (1500, 16, False, 13), (600, 10, True, 5)]
SHAPES = [(320, 240, 1, 128), (200, 152, 2, 256), (256, 256, 0, 128), (160, 120, 1, 64)]


def _settings():
    st = abi.default_settings()
    st.history_enabled = 0
    st.fragment_counts_enabled = 1
    st.dom_slices = 4
    return st


def _plugin():
    from bevy_strand_rasterizer_b200.plugin import StrandRasterizerPlugin
    p = StrandRasterizerPlugin()
    abi.check(p.lib.fiber_settings_set(p.ctx, C.byref(_settings())), "fiber_settings_set")
    return p


def _views():
    from bevy_strand_rasterizer_b200.plugin import pack_strand_set
    from bevy_strand_rasterizer_b200.scene import scalp_hair
    from test_server import _request
    rng = np.random.default_rng(23)
    out = []
    for (n, pts, curly, seed), (w, h, nl, dom) in zip(SCENES, SHAPES):
        packed = pack_strand_set(scalp_hair(n, pts, seed, curly=curly))
        cfg, cam, lcfg, lights = _request(packed, rng, w, h, nl, dom=dom)
        out.append((packed, cfg, cam, lcfg, lights, dom))
    return out


DUMPS = (abi.DUMP_COLOR, abi.DUMP_DEPTH, abi.DUMP_FRAGMENTS, abi.DUMP_DOM_DEPTH, abi.DUMP_DOM_OPACITY,
         abi.DUMP_SHADOW_MAP, abi.DUMP_ATLAS)


def _alone(view, fused):
    packed, cfg, cam, lcfg, lights, _ = view
    p = _plugin()
    p.add_geometry(packed)
    out = []
    for _ in range(2):
        p.frame_begin_raw(cfg, cam, lcfg, lights)
        if fused:
            p.frame_fused()
        else:
            p.render_nodes()
        out.append({w: p.dump(w).copy() for w in DUMPS})
    p.close()
    return out


@pytest.mark.parametrize("fused", [False, True])
def test_views_in_one_frame_match_views_alone(fused):
    views = _views()
    alone = [_alone(v, fused) for v in views]
    p = _plugin()
    for packed, *_ in views:
        p.add_geometry(packed)
    spec = [(cfg, cam, lcfg, lights, k, 1) for k, (_, cfg, cam, lcfg, lights, _) in enumerate(views)]
    K = 4
    D = max(v[5] for v in views if v[3])
    for frame in range(2):
        bases = p.frame_begin_views(spec)
        if fused:
            p.frame_fused()
        else:
            p.render_nodes()
        s = p.stats()
        assert s.frustum_count == sum(1 + len(v[3]) for v in views) and s.overflow_flags == 0
        color, depth, frags = p.dump(abi.DUMP_COLOR), p.dump(abi.DUMP_DEPTH), p.dump(abi.DUMP_FRAGMENTS)
        dom_d = p.dump(abi.DUMP_DOM_DEPTH).reshape(-1, D, D)
        dom_o = p.dump(abi.DUMP_DOM_OPACITY).reshape(-1, K, D, D)
        smap = p.dump(abi.DUMP_SHADOW_MAP).reshape(-1, D, D)
        atlas = p.dump(abi.DUMP_ATLAS).reshape(len(views), -1, 4)
        layer = 0
        for k, ((packed, cfg, _, lcfg, _, dom), ref) in enumerate(zip(views, alone)):
            want = ref[frame]
            n = cfg.screen_width * cfg.screen_height
            tag = f"frame {frame}, view {k} ({cfg.screen_width}x{cfg.screen_height}, {len(lcfg)} light(s))"
            b = bases[k]
            assert np.array_equal(color[4 * b: 4 * (b + n)].view(np.uint16), want[abi.DUMP_COLOR].view(np.uint16)), tag
            assert np.array_equal(depth[b: b + n].view(np.uint32), want[abi.DUMP_DEPTH].view(np.uint32)), tag
            assert np.array_equal(frags[b: b + n], want[abi.DUMP_FRAGMENTS]), tag
            assert int(want[abi.DUMP_FRAGMENTS].sum()) > 0, f"{tag}: no fragment"
            nl = len(lcfg)
            if nl:
                wd = want[abi.DUMP_DOM_DEPTH].reshape(nl, dom, dom)
                wo = want[abi.DUMP_DOM_OPACITY].reshape(nl, K, dom, dom)
                ws = want[abi.DUMP_SHADOW_MAP].reshape(nl, dom, dom)
                assert np.array_equal(dom_d[layer: layer + nl, :dom, :dom].view(np.uint32), wd.view(np.uint32)), tag
                assert np.array_equal(dom_o[layer: layer + nl, :, :dom, :dom].view(np.uint32), wo.view(np.uint32)), tag
                assert np.array_equal(smap[layer: layer + nl, :dom, :dom].view(np.uint32), ws.view(np.uint32)), tag
                layer += nl
            texels = int(packed.indices.shape[0])
            wa = want[abi.DUMP_ATLAS].reshape(-1, 4)[:texels]
            assert np.array_equal(atlas[k, :texels].view(np.uint16), wa.view(np.uint16)), tag
    p.close()


def test_frame_begin_views_rejects_bad_views():
    views = _views()
    p = _plugin()
    for packed, *_ in views[:2]:
        p.add_geometry(packed)
    (_, c0, m0, l0, s0, _), (_, c1, m1, l1, s1, _) = views[0], views[1]
    with pytest.raises(abi.FiberError):  # instance ranges must follow one another
        p.frame_begin_views([(c0, m0, l0, s0, 0, 1), (c1, m1, l1, s1, 0, 1)])
    with pytest.raises(abi.FiberError):  # and cover the instance table
        p.frame_begin_views([(c0, m0, l0, s0, 0, 1)] * 1 + [(c1, m1, l1, s1, 1, 0)])
    p.close()


def test_view_groups_match_one_multi_view_frame():
    """The views split into two multi-view frames on concurrent streams
    (batched.MultiViewGroups) render each view as one multi-view frame of all
    of them does, bit for bit."""
    import torch

    from bevy_strand_rasterizer_b200 import batched
    specs = batched.batched_views(6, seed=77, strand_range=(500, 3000))
    packed = [batched.view_strands(v) for v in specs]
    stream = torch.cuda.Stream()
    one = batched.MultiViewFrame(specs, packed)
    bases = one.launch(stream)
    stream.synchronize()
    want = {w: one.plugin.dump(w).copy() for w in (abi.DUMP_COLOR, abi.DUMP_FRAGMENTS)}
    one.close()
    two = batched.MultiViewGroups(specs, packed, 2)
    assert len(two.frames) == 2
    two.launch(stream)
    stream.synchronize()
    for g, f in zip(two.sets, two.frames):
        gb = f.launch(stream)
        stream.synchronize()
        color, frags = f.plugin.dump(abi.DUMP_COLOR), f.plugin.dump(abi.DUMP_FRAGMENTS)
        for j, k in enumerate(g):
            n = specs[k].camera_cfg.screen_width * specs[k].camera_cfg.screen_height
            a, b = bases[k], gb[j]
            assert np.array_equal(color[4 * b: 4 * (b + n)].view(np.uint16),
                                  want[abi.DUMP_COLOR][4 * a: 4 * (a + n)].view(np.uint16)), f"view {k}"
            assert np.array_equal(frags[b: b + n], want[abi.DUMP_FRAGMENTS][a: a + n]), f"view {k}"
    two.close()
