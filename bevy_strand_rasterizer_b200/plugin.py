"""Host-side mirror of the reference's plugin API for the strand raster path.

Names, defaults and argument meaning follow RostigerDagmer/bevy_strand_rasterizer:
StrandMaterial / FroxelConfig (src/components.rs:61-123), StochasticCullSettings /
PrepassTelemetrySettings / FineBinningBackend (src/resources.rs:70-104),
StrandList packing (pack_strands, src/plugin.rs:1315-1355) and the render-graph
nodes (work_preparation_pass, strand_shadow_rasterizer_pass, strand_shading_pass,
strand_rasterizer_pass, composition_pass). Every node runs in libfiber.so on
the GPU; this module only owns host bookkeeping and the ctypes calls.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .scene import CameraSpec, LightSpec, StrandSet


@dataclass
class StrandMaterial:
    """StrandMaterial with the reference defaults (src/components.rs:74-89)."""
    absorption_color: tuple = (0.7, 0.7, 0.7, 0.4)
    specular_color: tuple = (1.0, 1.0, 1.0, 1.0)
    ambient_factor: float = 0.05
    ao_factor: float = 0.1
    eta: float = 1.55
    beta: float = 0.5
    alpha: float = 0.3
    shift: float = 0.01
    min_radius_pixels: float = 0.4
    max_radius_pixels: float = 2.0

    def to_c(self) -> abi.StrandMaterialC:
        m = abi.StrandMaterialC()
        m.absorption_color[:] = self.absorption_color
        m.specular_color[:] = self.specular_color
        for name in ("ambient_factor", "ao_factor", "eta", "beta", "alpha", "shift", "min_radius_pixels",
                     "max_radius_pixels"):
            setattr(m, name, getattr(self, name))
        return m


@dataclass
class FroxelConfig:
    """FroxelConfig (src/components.rs:93-110)."""
    screen_width: int = 1920
    screen_height: int = 1080
    froxel_size_x: int = 8
    froxel_size_y: int = 8
    depth_slices: int = 64

    def get_num_tiles(self) -> tuple[int, int, int]:
        tx = (self.screen_width + self.froxel_size_x - 1) // self.froxel_size_x
        ty = (self.screen_height + self.froxel_size_y - 1) // self.froxel_size_y
        return tx, ty, tx * ty * self.depth_slices

    def to_c(self) -> abi.FroxelConfigC:
        return abi.FroxelConfigC(self.screen_width, self.screen_height, self.froxel_size_x, self.froxel_size_y,
                                 self.depth_slices)


@dataclass
class StochasticCullSettings:
    """StochasticCullSettings (src/resources.rs:70-104); enabled by default."""
    enabled: bool = True
    target_strands_per_pixel: float = 2.0
    min_keep_probability: float = 0.02
    shadow_keep_probability: float = 1.0


@dataclass
class PrepassTelemetrySettings:
    enabled: bool = False


class FineBinningBackend(enum.IntEnum):
    SegmentScatter = 0
    PageCsr = 1


@dataclass
class StrandList:
    """StrandList (src/components.rs:11-20): vertices plus per-strand index lists."""
    vertices: np.ndarray
    strands: list


@dataclass
class PackedStrandBuffers:
    """The five slabs of one strand asset (insert_packed_strand_geometry, src/plugin.rs:1395-1440)."""
    vertices: np.ndarray      # (P, 4) float32, w = 1
    indices: np.ndarray       # (N,) uint32
    meta: np.ndarray          # abi.STRAND_META records
    strand_count: int
    index_count: int
    max_segments_in_strand: int
    aabb_min: np.ndarray
    aabb_max: np.ndarray

    def geo(self) -> abi.StrandGeo:
        g = abi.StrandGeo()
        g.strand_count = self.strand_count
        g.max_segments_in_strand = self.max_segments_in_strand
        g.offset = 0
        g.aabb.min[:] = [float(x) for x in self.aabb_min]
        g.aabb.max[:] = [float(x) for x in self.aabb_max]
        return g


def _vertices4(vertices: np.ndarray) -> np.ndarray:
    v = np.asarray(vertices, np.float32).reshape(-1, 3)
    out = np.ones((v.shape[0], 4), np.float32)
    out[:, :3] = v
    return out


def pack_strands(vertices: np.ndarray, strands) -> PackedStrandBuffers | None:
    """pack_strands (src/plugin.rs:1315-1355): vertices -> float4 (w = 1); strands
    with fewer than two points are dropped; meta = (count, offset, 0, 0)."""
    v4 = _vertices4(vertices)
    if v4.shape[0] == 0:
        return None
    indices, metas, max_count = [], [], 0
    offset = 0
    for s in strands:
        s = np.asarray(s, np.uint32)
        if s.shape[0] < 2:
            continue
        metas.append((s.shape[0], offset, 0, 0))
        indices.append(s)
        offset += s.shape[0]
        max_count = max(max_count, s.shape[0])
    if not metas:
        return None
    meta = np.array(metas, dtype=abi.STRAND_META)
    idx = np.concatenate(indices).astype(np.uint32)
    return PackedStrandBuffers(v4, idx, meta, len(metas), int(idx.shape[0]), max_count,
                               v4[:, :3].min(axis=0), v4[:, :3].max(axis=0))


def pack_indexed_strands(vertices: np.ndarray, counts: np.ndarray, offsets: np.ndarray,
                         indices: np.ndarray) -> PackedStrandBuffers | None:
    """pack_indexed_strands (src/plugin.rs:1357-1393): cache strands reference a
    shared index buffer; strands with count < 2 are dropped."""
    v4 = _vertices4(vertices)
    counts = np.asarray(counts, np.uint32)
    offsets = np.asarray(offsets, np.uint32)
    keep = counts >= 2
    if v4.shape[0] == 0 or not keep.any():
        return None
    meta = np.zeros(int(keep.sum()), dtype=abi.STRAND_META)
    meta["count"] = counts[keep]
    meta["offset"] = offsets[keep]
    idx = np.asarray(indices, np.uint32)
    return PackedStrandBuffers(v4, idx, meta, int(keep.sum()), int(idx.shape[0]), int(counts[keep].max()),
                               v4[:, :3].min(axis=0), v4[:, :3].max(axis=0))


def pack_strand_set(s: StrandSet) -> PackedStrandBuffers:
    return pack_indexed_strands(s.vertices, s.strand_counts, s.strand_offsets, s.indices)


IDENTITY = np.eye(4, dtype=np.float32).reshape(16)


@dataclass
class _Asset:
    packed: PackedStrandBuffers
    material: StrandMaterial
    world_from_local: np.ndarray
    ids: dict = field(default_factory=dict)


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(int(stream.cuda_stream))


class StrandRasterizerPlugin:
    """StrandRasterizerPlugin (src/plugin.rs:162-262) over libfiber.so.

    `add_geometry` registers a strand asset (the StrandGeometry component),
    `frame_begin` is use_prepass_buffers for one camera + directional lights,
    and `prepass / shadows / shading / raster / composite` are the render-graph
    nodes in their reference order. Raises abi.FiberError on any failure.
    """

    def __init__(self, device: int = 0, hbm_budget: int = 0,
                 cull: StochasticCullSettings | None = None,
                 telemetry: PrepassTelemetrySettings | None = None,
                 backend: FineBinningBackend = FineBinningBackend.SegmentScatter,
                 dom_slices: int = 12, shadow_map_size: int = 0, ambient=(80.0, 80.0, 80.0, 80.0),
                 history: bool = True, fragment_counts: bool = False, ref_capacity_factor: int = 4,
                 page_capacity_divisor: int = 1, dom_page_pool: int = 0):
        self.lib = abi.load_library()
        self.ctx = C.c_void_p()
        abi.check(self.lib.fiber_ctx_create(device, hbm_budget, C.byref(self.ctx)), "fiber_ctx_create")
        self.device = device
        self.assets: list[_Asset] = []
        s = abi.default_settings()
        cull = cull or StochasticCullSettings()
        s.stochastic_cull_enabled = 1 if cull.enabled else 0
        s.target_strands_per_pixel = cull.target_strands_per_pixel
        s.min_keep_probability = cull.min_keep_probability
        s.shadow_keep_probability = cull.shadow_keep_probability
        s.telemetry_enabled = 1 if (telemetry and telemetry.enabled) else 0
        s.fine_binning_backend = int(backend)
        s.dom_slices = dom_slices
        s.shadow_map_size = shadow_map_size
        s.ambient_color[:] = ambient
        s.history_enabled = 1 if history else 0
        s.fragment_counts_enabled = 1 if fragment_counts else 0
        s.ref_capacity_factor = ref_capacity_factor
        s.page_capacity_divisor = page_capacity_divisor
        s.dom_page_pool = dom_page_pool  # 0: dense DOM layers; N: sparse residency in N pages of 256^2
        self.settings = s
        abi.check(self.lib.fiber_settings_set(self.ctx, C.byref(s)), "fiber_settings_set")
        self.camera_cfg = None
        self.light_cfgs = []

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self.ctx:
            self.lib.fiber_ctx_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- slabs / geometry ---------------------------------------------------
    def _slab(self, kind: int, data: np.ndarray) -> int:
        data = np.ascontiguousarray(data)
        aid = C.c_uint32()
        ptr = abi.DevicePtr()
        abi.check(self.lib.fiber_slab_alloc(self.ctx, kind, data.nbytes, C.byref(aid), C.byref(ptr)),
                  "fiber_slab_alloc")
        abi.check(self.lib.fiber_slab_upload(self.ctx, kind, aid.value, 0, data.ctypes.data_as(C.c_void_p),
                                             data.nbytes, None), "fiber_slab_upload")
        return aid.value

    def add_geometry(self, packed: PackedStrandBuffers, material: StrandMaterial | None = None,
                     world_from_local: np.ndarray | None = None) -> int:
        material = material or StrandMaterial()
        w = IDENTITY if world_from_local is None else np.asarray(world_from_local, np.float32).reshape(16)
        a = _Asset(packed, material, w)
        geo = packed.geo()
        mat = material.to_c()
        a.ids["vertex"] = self._slab(abi.SLAB_VERT, packed.vertices)
        a.ids["index"] = self._slab(abi.SLAB_INDEX, packed.indices)
        a.ids["meta"] = self._slab(abi.SLAB_META, packed.meta)
        a.ids["geo"] = self._slab(abi.SLAB_GEO, np.frombuffer(bytes(geo), np.uint8))
        a.ids["material"] = self._slab(abi.SLAB_MATERIAL, np.frombuffer(bytes(mat), np.uint8))
        self.assets.append(a)
        self._register()
        return len(self.assets) - 1

    def add_strand_cache(self, cache, material: StrandMaterial | None = None,
                         world_from_local: np.ndarray | None = None) -> int:
        """A StrandCache component (src/components.rs:17, loaded by
        set_cached_strand_geometry, src/plugin.rs:1468-1497): `cache` is a
        `.strands` path or a parsed strand_cache.StrandCacheFile."""
        from . import strand_cache
        if not isinstance(cache, strand_cache.StrandCacheFile):
            cache = strand_cache.load(str(cache))
        packed = strand_cache.to_packed(cache)
        if packed is None:
            raise abi.FiberError(abi.EINVAL, "strand cache: no strand with two points")
        return self.add_geometry(packed, material, world_from_local)

    def _register(self):
        rows = (abi.StrandInstance * max(1, len(self.assets)))()
        for i, a in enumerate(self.assets):
            r = rows[i]
            r.vertex_id, r.index_id, r.meta_id = a.ids["vertex"], a.ids["index"], a.ids["meta"]
            r.geo_id, r.material_id = a.ids["geo"], a.ids["material"]
            r.world_from_local[:] = [float(x) for x in a.world_from_local]
            inv = np.linalg.inv(a.world_from_local.reshape(4, 4).T.astype(np.float64)).T.reshape(16)
            r.local_from_world[:] = [float(x) for x in inv]
        abi.check(self.lib.fiber_instance_set(self.ctx, rows, len(self.assets)), "fiber_instance_set")

    def scene_aabb(self) -> tuple[np.ndarray, np.ndarray]:
        lo = np.full(3, np.inf)
        hi = np.full(3, -np.inf)
        for a in self.assets:
            w = a.world_from_local.reshape(4, 4).T.astype(np.float64)
            for x in (a.packed.aabb_min[0], a.packed.aabb_max[0]):
                for y in (a.packed.aabb_min[1], a.packed.aabb_max[1]):
                    for z in (a.packed.aabb_min[2], a.packed.aabb_max[2]):
                        p = w @ np.array([x, y, z, 1.0])
                        lo = np.minimum(lo, p[:3])
                        hi = np.maximum(hi, p[:3])
        return lo, hi

    # -- frame ---------------------------------------------------------------
    def frame_begin(self, camera_cfg: FroxelConfig, camera: CameraSpec, lights: list, stream=None):
        """lights: list of (FroxelConfig, LightSpec)."""
        lo, hi = self.scene_aabb()
        cam = abi.Camera()
        cam.clip_from_world[:] = [float(x) for x in camera.clip_from_world()]
        cam.world_position[:] = [float(x) for x in camera.eye]
        n = len(lights)
        cfgs = (abi.FroxelConfigC * max(1, n))()
        ls = (abi.Light * max(1, n))()
        for i, (cfg, spec) in enumerate(lights):
            cfgs[i] = cfg.to_c()
            ls[i].clip_from_world[:] = [float(x) for x in spec.clip_from_world(lo, hi)]
            ls[i].direction_to_light[:] = [float(x) for x in spec.direction()]
            ls[i].color[:] = [float(x) for x in spec.color4()]
        self.camera_cfg = camera_cfg
        self.light_cfgs = [c for c, _ in lights]
        self._cam_c, self._lights_c, self._cfgs_c = cam, ls, cfgs
        abi.check(self.lib.fiber_frame_begin(self.ctx, C.byref(camera_cfg.to_c()), C.byref(cam), cfgs, ls, n,
                                             _stream_handle(stream)), "fiber_frame_begin")

    def frame_begin_raw(self, camera_cfg: FroxelConfig, cam: abi.Camera, light_cfgs: list, lights_c, stream=None):
        n = len(light_cfgs)
        cfgs = (abi.FroxelConfigC * max(1, n))(*[c.to_c() for c in light_cfgs])
        self.camera_cfg = camera_cfg
        self.light_cfgs = list(light_cfgs)
        abi.check(self.lib.fiber_frame_begin(self.ctx, C.byref(camera_cfg.to_c()), C.byref(cam), cfgs, lights_c, n,
                                             _stream_handle(stream)), "fiber_frame_begin")

    def frame_begin_views(self, views: list, stream=None):
        """One frame of several independent views (fiber_frame_begin_views).
        views: list of (camera_cfg: FroxelConfig, cam: abi.Camera, light_cfgs:
        list[FroxelConfig], lights_c: abi.Light array, instance_first,
        instance_count); a view's instances follow the previous view's. Returns
        the first pixel of each view's colour / depth / fragment image."""
        arr = (abi.View * len(views))()
        keep = []
        bases, px = [], 0
        for k, (cfg, cam, lcfgs, lights_c, first, count) in enumerate(views):
            v = arr[k]
            v.camera_cfg = cfg.to_c()
            v.camera = cam
            n = len(lcfgs)
            lc = (abi.FroxelConfigC * max(1, n))(*[c.to_c() for c in lcfgs])
            keep += [lc, lights_c]
            v.light_cfgs = C.cast(lc, C.POINTER(abi.FroxelConfigC))
            v.lights = C.cast(lights_c, C.POINTER(abi.Light))
            v.n_lights = n
            v.instance_first = first
            v.instance_count = count
            bases.append(px)
            px += cfg.screen_width * cfg.screen_height
        self.camera_cfg = views[0][0]
        self.light_cfgs = [c for view in views for c in view[2]]
        abi.check(self.lib.fiber_frame_begin_views(self.ctx, arr, len(views), _stream_handle(stream)),
                  "fiber_frame_begin_views")
        del keep
        return bases

    # Render-graph nodes ------------------------------------------------------
    def depth_reduce(self, opaque_depth: abi.Image, samples: int = 1, stream=None):
        """reduce_opaque_depth (src/pipelines/prepass.rs:780-815): the camera's
        opaque depth (R32F, reversed-Z, `samples` floats per pixel) to the
        per-fine-tile pairs the prepass culls against. Call after frame_begin,
        before work_preparation_pass."""
        abi.check(self.lib.fiber_opaque_depth(self.ctx, C.byref(opaque_depth), samples, _stream_handle(stream)),
                  "fiber_opaque_depth")

    def work_preparation_pass(self, stream=None):
        abi.check(self.lib.fiber_prepass(self.ctx, _stream_handle(stream)), "fiber_prepass")

    def strand_shadow_rasterizer_pass(self, stream=None):
        abi.check(self.lib.fiber_shadows(self.ctx, _stream_handle(stream)), "fiber_shadows")

    def strand_shading_pass(self, stream=None):
        abi.check(self.lib.fiber_shading(self.ctx, _stream_handle(stream)), "fiber_shading")

    def strand_rasterizer_pass(self, stream=None):
        abi.check(self.lib.fiber_raster(self.ctx, 0, _stream_handle(stream)), "fiber_raster")

    def composition_pass(self, scene_color: abi.Image, scene_depth: abi.Image | None, out: abi.Image, stream=None):
        abi.check(self.lib.fiber_composite(self.ctx, 0, C.byref(scene_color),
                                           C.byref(scene_depth) if scene_depth is not None else None,
                                           C.byref(out), _stream_handle(stream)), "fiber_composite")

    def render_nodes(self, scene_color=None, scene_depth=None, out=None, stream=None, opaque_samples: int = 1,
                     opaque_depth=None):
        """Every node in order. The opaque-tile reduce reads opaque_depth
        (`opaque_samples` per pixel) when given, else scene_depth at 1 sample,
        as the reference's prepass node reads the view's depth prepass."""
        if opaque_depth is not None:
            self.depth_reduce(opaque_depth, opaque_samples, stream)
        elif scene_depth is not None:
            self.depth_reduce(scene_depth, 1, stream)
        self.work_preparation_pass(stream)
        self.strand_shadow_rasterizer_pass(stream)
        self.strand_shading_pass(stream)
        self.strand_rasterizer_pass(stream)
        if scene_color is not None and out is not None:
            self.composition_pass(scene_color, scene_depth, out, stream)

    def frame_fused(self, scene_color=None, scene_depth=None, out=None, stream=None):
        abi.check(self.lib.fiber_frame_fused(self.ctx, C.byref(scene_color) if scene_color is not None else None,
                                             C.byref(scene_depth) if scene_depth is not None else None,
                                             C.byref(out) if out is not None else None, _stream_handle(stream)),
                  "fiber_frame_fused")

    # -- readback ------------------------------------------------------------
    def stats(self, allow_overflow: bool = False) -> abi.Stats:
        s = abi.Stats()
        allow = (abi.OK, abi.EOVERFLOW) if allow_overflow else (abi.OK,)
        abi.check(self.lib.fiber_stats_get(self.ctx, C.byref(s)), "fiber_stats_get", allow)
        return s

    def telemetry(self) -> abi.Telemetry:
        """The last frame's prepass telemetry (the plugin must be created with
        telemetry=PrepassTelemetrySettings(enabled=True))."""
        t = abi.Telemetry()
        abi.check(self.lib.fiber_telemetry_get(self.ctx, C.byref(t)), "fiber_telemetry_get")
        return t

    def dump(self, what: int) -> np.ndarray:
        n = C.c_uint64()
        abi.check(self.lib.fiber_dump(self.ctx, what, None, 0, C.byref(n)), "fiber_dump(size)")
        buf = np.empty(n.value, np.uint8)
        abi.check(self.lib.fiber_dump(self.ctx, what, buf.ctypes.data_as(C.c_void_p), n.value, C.byref(n)),
                  "fiber_dump")
        return buf.view(abi.DUMP_DTYPES[what])

    def span_times(self) -> dict:
        k = self.lib.fiber_span_count()
        ms = (C.c_float * k)()
        abi.check(self.lib.fiber_span_times(self.ctx, ms, k), "fiber_span_times")
        return {self.lib.fiber_span_name(i).decode(): float(ms[i]) for i in range(k)}

    def output_image(self, what: int) -> abi.Image:
        img = abi.Image()
        abi.check(self.lib.fiber_output_image(self.ctx, what, C.byref(img)), "fiber_output_image")
        return img


def image_from_tensor(t, fmt: int) -> abi.Image:
    """fiber_image view of a contiguous CUDA tensor (H, W, C)."""
    h, w = int(t.shape[0]), int(t.shape[1])
    return abi.Image(C.c_void_p(t.data_ptr()), w, h, int(t.stride(0) * t.element_size()), fmt)
