"""The batched configuration: many independent views, each with its own strand
set, camera, light and resolution, rendered either by one multi-view frame
(MultiViewFrame: every kernel covers all views) or by one CUDA graph launch of
the views' own frames over concurrent branches (fiber_batch_*), and the same
views as a loop of plain frames for comparison.

Views: strand counts log-uniform in [1k, 200k] at 16 or 32 points per strand
(straight scalp hair), a resolution from {256^2, 512^2, 1280x720, 1920x1080},
a camera on a sphere of radius 0.4-1.0 m (upper hemisphere) looking at the
origin, and one directional light from the upper hemisphere with a 512^2,
1024^2 or 2048^2 deep-opacity map. The temporal shadow history is off, so a
view's image is the same alone, in the plain loop and in the batch.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import abi
from .plugin import FroxelConfig, PackedStrandBuffers, StrandRasterizerPlugin, _stream_handle, pack_strand_set
from .scene import CameraSpec, LightSpec, scalp_hair
from .served import DOM_SIZES, RESOLUTIONS, _hemisphere

STRAND_RANGE = (1_000, 200_000)
POINTS = (16, 32)


@dataclass
class ViewSpec:
    strands: int
    points: int
    seed: int
    camera: CameraSpec
    camera_cfg: FroxelConfig
    light: LightSpec
    light_cfg: FroxelConfig


def batched_views(n: int = 64, seed: int = 2000, strand_range=STRAND_RANGE) -> list[ViewSpec]:
    rng = np.random.default_rng(seed)
    lo, hi = math.log(strand_range[0]), math.log(strand_range[1])
    views = []
    for v in range(n):
        strands = int(round(math.exp(rng.uniform(lo, hi))))
        points = POINTS[int(rng.integers(0, len(POINTS)))]
        w, h = RESOLUTIONS[int(rng.integers(0, len(RESOLUTIONS)))]
        dom = DOM_SIZES[int(rng.integers(0, len(DOM_SIZES)))]
        eye = _hemisphere(rng) * rng.uniform(0.4, 1.0)
        cam = CameraSpec(eye=tuple(float(x) for x in eye), width=w, height=h)
        light = LightSpec(tuple(float(x) for x in _hemisphere(rng)), size=dom)
        views.append(ViewSpec(strands, points, seed + 1 + v, cam, FroxelConfig(w, h, 8, 8, 64), light,
                              FroxelConfig(dom, dom, 8, 8, 64)))
    return views


def view_strands(spec: ViewSpec) -> PackedStrandBuffers:
    return pack_strand_set(scalp_hair(spec.strands, spec.points, spec.seed))


def view_plugin(spec: ViewSpec, packed: PackedStrandBuffers, device: int = 0, **kw) -> StrandRasterizerPlugin:
    """A context holding the view's strand set with its frame tables uploaded."""
    kw.setdefault("history", False)
    kw.setdefault("dom_slices", 8)
    p = StrandRasterizerPlugin(device=device, **kw)
    p.add_geometry(packed)
    p.frame_begin(spec.camera_cfg, spec.camera, [(spec.light_cfg, spec.light)])
    return p


def plain_frame(plugin: StrandRasterizerPlugin, spec: ViewSpec, stream=None):
    """The plain per-view frame the batch is compared with: frame tables, then
    the frame's nodes replayed from the context's own graph."""
    plugin.frame_begin(spec.camera_cfg, spec.camera, [(spec.light_cfg, spec.light)], stream)
    plugin.frame_fused(None, None, None, stream)


class MultiViewFrame:
    """Every view rendered by one multi-view frame (fiber_frame_begin_views):
    one context holds each view's strand set as an instance, every kernel of the
    frame covers all views (each view's tasks, pages and runs at offsets from the
    frame's single prefix sums), and the frame is replayed from one CUDA graph.
    Each view's image is the one it renders alone (tests/test_gpu_views.py)."""

    def __init__(self, specs: list[ViewSpec], packed: list[PackedStrandBuffers], device: int = 0, **kw):
        kw.setdefault("history", False)
        kw.setdefault("dom_slices", 8)
        self.plugin = StrandRasterizerPlugin(device=device, **kw)
        for p in packed:
            self.plugin.add_geometry(p)
        self.views = []
        self._keep = []
        for k, (s, p) in enumerate(zip(specs, packed)):
            cam = abi.Camera()
            cam.clip_from_world[:] = [float(x) for x in s.camera.clip_from_world()]
            cam.world_position[:] = [float(x) for x in s.camera.eye]
            lights = (abi.Light * 1)()
            lights[0].clip_from_world[:] = [float(x) for x in s.light.clip_from_world(p.aabb_min, p.aabb_max)]
            lights[0].direction_to_light[:] = [float(x) for x in s.light.direction()]
            lights[0].color[:] = [float(x) for x in s.light.color4()]
            self._keep.append((cam, lights))
            self.views.append((s.camera_cfg, cam, [s.light_cfg], lights, k, 1))

    def launch(self, stream=None) -> list:
        """One frame of every view; returns each view's first pixel in the
        concatenated colour / depth / fragment images."""
        bases = self.plugin.frame_begin_views(self.views, stream)
        self.plugin.frame_fused(None, None, None, stream)
        return bases

    def close(self):
        self.plugin.close()


def view_cost(spec: ViewSpec, packed: PackedStrandBuffers) -> float:
    """A view's work estimate for grouping: its segments plus its camera and
    deep-opacity pixels."""
    segs = float(np.maximum(packed.meta["count"].astype(np.int64) - 1, 0).sum())
    return segs + spec.camera_cfg.screen_width * spec.camera_cfg.screen_height + spec.light_cfg.screen_width ** 2


def group_views(costs, groups: int) -> list[list[int]]:
    """Views split into `groups` sets of near-equal cost: longest first, each to
    the set with the least cost so far; each set keeps increasing view order."""
    sets = [[] for _ in range(max(1, groups))]
    load = [0.0] * len(sets)
    for k in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        j = min(range(len(sets)), key=lambda i: (load[i], i))
        sets[j].append(k)
        load[j] += costs[k]
    return [sorted(g) for g in sets if g]


class MultiViewGroups:
    """The views as `groups` multi-view frames on concurrent streams (one
    context and one stream each), launched together from `stream`: the work of
    one group's small launches overlaps another's large ones. groups = 1 is one
    MultiViewFrame. Each view's image is the one it renders alone."""

    def __init__(self, specs: list[ViewSpec], packed: list[PackedStrandBuffers], groups: int, device: int = 0,
                 **kw):
        import torch
        self.sets = group_views([view_cost(s, p) for s, p in zip(specs, packed)], groups)
        self.frames = [MultiViewFrame([specs[k] for k in g], [packed[k] for k in g], device, **kw) for g in self.sets]
        self.streams = [torch.cuda.Stream(device) for _ in self.frames]

    def launch(self, stream):
        import torch
        start = torch.cuda.Event()
        start.record(stream)
        for f, s in zip(self.frames, self.streams):
            s.wait_event(start)
            f.launch(s)
        for s in self.streams:
            done = torch.cuda.Event()
            done.record(s)
            stream.wait_event(done)

    def close(self):
        for f in self.frames:
            f.close()


class FiberBatch:
    """fiber_batch over the contexts of `plugins` (which must outlive it)."""

    def __init__(self, plugins: list[StrandRasterizerPlugin]):
        self.lib = abi.load_library()
        self.plugins = list(plugins)
        arr = (C.c_void_p * len(plugins))(*[p.ctx.value for p in plugins])
        self.handle = C.c_void_p()
        abi.check(self.lib.fiber_batch_create(arr, len(plugins), C.byref(self.handle)), "fiber_batch_create")

    def launch(self, stream):
        abi.check(self.lib.fiber_batch_launch(self.handle, _stream_handle(stream)), "fiber_batch_launch")

    def tune(self, stream) -> abi.BatchTuning:
        best = abi.BatchTuning()
        abi.check(self.lib.fiber_batch_tune(self.handle, _stream_handle(stream), C.byref(best)), "fiber_batch_tune")
        return best

    @property
    def tuning(self) -> abi.BatchTuning:
        t = abi.BatchTuning()
        abi.check(self.lib.fiber_batch_get_tuning(self.handle, C.byref(t)), "fiber_batch_get_tuning")
        return t

    def set_tuning(self, branches: int, order: int = abi.BATCH_ORDER_INDEX):
        t = abi.BatchTuning(branches, order, 0.0, 0)
        abi.check(self.lib.fiber_batch_set_tuning(self.handle, C.byref(t)), "fiber_batch_set_tuning")

    def close(self):
        if self.handle:
            self.lib.fiber_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plan(costs, branches: int, order: int = abi.BATCH_ORDER_LPT) -> np.ndarray:
    """fiber_batch_plan: the branch of each view (host only)."""
    lib = abi.load_library()
    c = np.ascontiguousarray(costs, np.float32)
    out = np.zeros(len(c), np.uint32)
    abi.check(lib.fiber_batch_plan(c.ctypes.data_as(C.POINTER(C.c_float)), len(c), branches, order,
                                   out.ctypes.data_as(C.POINTER(C.c_uint32))), "fiber_batch_plan")
    return out
