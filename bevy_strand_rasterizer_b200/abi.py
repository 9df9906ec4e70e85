"""ctypes mirror of include/fiber.h and the loader of the in-tree libfiber.so.

The structs below are byte-for-byte the reference's `#[repr(C)]` host mirrors
(src/shader_types.rs, src/pipelines/task_contract.rs, src/components.rs,
src/plugin.rs); their numpy dtypes let tests and tools view device dumps
without copying. There is no fallback: if libfiber.so is missing or fails to
load, `load_library()` raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libfiber.so"

u32 = C.c_uint32
f32 = C.c_float


class FiberStatus(C.c_int):
    pass


OK, EINVAL, ENOMEM, EOVERFLOW, ETIMEDOUT, ECUDA, ENOTREADY = range(7)
STATUS_NAMES = {OK: "ok", EINVAL: "EINVAL", ENOMEM: "ENOMEM", EOVERFLOW: "EOVERFLOW",
                ETIMEDOUT: "ETIMEDOUT", ECUDA: "ECUDA", ENOTREADY: "ENOTREADY"}

SLAB_VERT, SLAB_INDEX, SLAB_MATERIAL, SLAB_GEO, SLAB_META = 0, 1, 5, 6, 7
FMT_RGBA16F, FMT_R32F, FMT_RGBA32F = 0, 1, 2
MAX_FRUSTA = 16  # FIBER_MAX_FRUSTA: the camera plus up to 15 lights

(DUMP_FRUSTA, DUMP_RANGES, DUMP_KEEP, DUMP_LUT, DUMP_TASKS, DUMP_PROJECTED, DUMP_PAGE_TABLE,
 DUMP_PAGE_META, DUMP_COUNTS, DUMP_OFFSETS, DUMP_REFS, DUMP_ACTIVE_TILES, DUMP_WORK, DUMP_RUNS,
 DUMP_DOM_DEPTH, DUMP_DOM_OPACITY, DUMP_SHADOW_MAP, DUMP_ATLAS, DUMP_HISTORY, DUMP_COLOR,
 DUMP_DEPTH, DUMP_FRAGMENTS, DUMP_OPAQUE_TILES) = range(23)


class DevicePtr(C.Structure):
    _fields_ = [("slab", u32), ("offset", u32), ("size", u32)]


class Aabb(C.Structure):
    _fields_ = [("min", f32 * 3), ("pad_a", f32), ("max", f32 * 3), ("pad_b", f32)]


class StrandGeo(C.Structure):
    _fields_ = [("strand_count", u32), ("max_segments_in_strand", u32), ("offset", u32), ("pad_b", u32),
                ("aabb", Aabb), ("pad_c", u32 * 4)]


class StrandMaterialC(C.Structure):
    _fields_ = [("absorption_color", f32 * 4), ("specular_color", f32 * 4), ("ambient_factor", f32),
                ("ao_factor", f32), ("eta", f32), ("beta", f32), ("alpha", f32), ("shift", f32),
                ("min_radius_pixels", f32), ("max_radius_pixels", f32)]


class StrandInstance(C.Structure):
    _fields_ = [("vertex_id", u32), ("index_id", u32), ("meta_id", u32), ("geo_id", u32),
                ("material_id", u32), ("pad0", u32), ("pad1", u32), ("pad2", u32),
                ("world_from_local", f32 * 16), ("local_from_world", f32 * 16)]


class FroxelConfigC(C.Structure):
    _fields_ = [("screen_width", u32), ("screen_height", u32), ("froxel_size_x", u32),
                ("froxel_size_y", u32), ("depth_slices", u32)]


class Camera(C.Structure):
    _fields_ = [("clip_from_world", f32 * 16), ("world_position", f32 * 3), ("pad", f32)]


class Light(C.Structure):
    _fields_ = [("clip_from_world", f32 * 16), ("direction_to_light", f32 * 3), ("pad0", f32),
                ("color", f32 * 4)]


class View(C.Structure):
    """fiber_view: one view of a multi-view frame (fiber_frame_begin_views)."""
    _fields_ = [("camera_cfg", FroxelConfigC), ("camera", Camera), ("light_cfgs", C.POINTER(FroxelConfigC)),
                ("lights", C.POINTER(Light)), ("n_lights", u32), ("instance_first", u32), ("instance_count", u32),
                ("pad", u32)]


class Settings(C.Structure):
    _fields_ = [("stochastic_cull_enabled", u32), ("target_strands_per_pixel", f32),
                ("min_keep_probability", f32), ("shadow_keep_probability", f32),
                ("telemetry_enabled", u32), ("fine_binning_backend", u32), ("dom_slices", u32),
                ("shadow_map_size", u32), ("ambient_color", f32 * 4), ("history_enabled", u32),
                ("fragment_counts_enabled", u32), ("ref_capacity_factor", u32),
                ("page_capacity_divisor", u32), ("dom_page_pool", u32)]


class Image(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("width", u32), ("height", u32), ("pitch", u32), ("format", u32)]


class Stats(C.Structure):
    _fields_ = [("frustum_count", u32), ("instance_count", u32), ("binning_tasks", u32),
                ("camera_tasks", u32), ("allocated_pages", u32), ("fine_refs", u32),
                ("active_tiles", u32), ("camera_runs", u32), ("shadow_runs", u32), ("work_items", u32),
                ("overflow_flags", u32), ("timeout_flags", u32), ("frustum_tasks", u32 * MAX_FRUSTA),
                ("frustum_pages", u32 * MAX_FRUSTA), ("frustum_refs", u32 * MAX_FRUSTA),
                ("frustum_work", u32 * MAX_FRUSTA), ("frustum_runs", u32 * MAX_FRUSTA),
                ("total_segments", C.c_uint64), ("total_points", C.c_uint64), ("total_strands", C.c_uint64),
                ("fine_refs_total", C.c_uint64), ("refs_requested", C.c_uint64)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else int(v)
        return out


# Request server (fiber_server_*).
SERVER_MAX_LIGHTS = 4
PRIORITY_ARRIVAL, PRIORITY_COST = 0, 1


class ServerConfig(C.Structure):
    _fields_ = [("slots", u32), ("max_width", u32), ("max_height", u32), ("max_lights", u32), ("max_dom", u32),
                ("priority_levels", u32), ("hbm_budget", C.c_uint64), ("priority_order", u32), ("pad", u32)]


class ServerScene(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("n_vertices", u32), ("indices", C.c_void_p), ("n_indices", u32),
                ("meta", C.c_void_p), ("n_meta", u32), ("geo", StrandGeo), ("materials", C.c_void_p),
                ("n_materials", u32), ("world_from_local", f32 * 16)]


class ServerRequest(C.Structure):
    _fields_ = [("scene", u32), ("n_lights", u32), ("camera_cfg", FroxelConfigC), ("camera", Camera),
                ("light_cfgs", FroxelConfigC * SERVER_MAX_LIGHTS), ("lights", Light * SERVER_MAX_LIGHTS),
                ("scene_rgba16f", C.c_void_p), ("out_rgba16f", C.c_void_p), ("arrival_ns", C.c_uint64)]


class ServerResult(C.Structure):
    _fields_ = [("status", C.c_int), ("slot", u32), ("arrival_ns", C.c_uint64), ("admit_ns", C.c_uint64),
                ("done_ns", C.c_uint64), ("renders", u32), ("priority", u32)]


# numpy views of the task-contract structs (src/pipelines/task_contract.rs:45-135)
BINNING_TASK = np.dtype([("id_info", "<u4"), ("chunk_id", "<u4"), ("seg_idx", "<u4"), ("packed_field", "<u4")])
PROJECTED_SEGMENT = np.dtype([("p0_xy", "<u4"), ("p1_xy", "<u4"), ("depths", "<u4")])
RASTER_WORK_ITEM = np.dtype([(n, "<u4") for n in ("seg_ref_base", "seg_ref_count", "frustum_id", "screen_tile_id",
                                                   "depth_key", "load_score", "page_idx", "cell_idx")])
RASTER_TILE_RUN = np.dtype([(n, "<u4") for n in ("work_base", "work_count", "frustum_id", "screen_tile_id",
                                                  "load_score", "flags", "reserved_a", "reserved_b")])
FINE_SEG_REF = np.dtype([("inst_id", "<u4"), ("seg_id", "<u4"), ("material_idx", "<u4")])
FINE_PAGE_META = np.dtype([(n, "<u4") for n in ("seg_ref_base", "seg_ref_count", "work_base", "work_count",
                                                 "coarse_tile_id", "coarse_z", "first_depth_key", "flags")])
LUT_ENTRY = np.dtype([(n, "<u4") for n in ("z_min_q", "z_max_q", "virtual_start_q", "virtual_count_q")])
FRUSTUM_DESC = np.dtype([(n, "<u4") for n in (
    "screen_width", "screen_height", "froxel_size_x", "froxel_size_y", "depth_slices", "bucket_base",
    "bucket_count", "kind", "coarse_depth_tile_base", "coarse_depth_tile_count", "coarse_tiles_x",
    "coarse_tiles_y", "cascade_index", "fine_depth_tile_base", "pad1", "pad2")])
STRAND_META = np.dtype([("count", "<u4"), ("offset", "<u4"), ("material_idx", "<u4"), ("pad", "<u4")])

DUMP_DTYPES = {
    DUMP_FRUSTA: FRUSTUM_DESC, DUMP_RANGES: np.dtype("<u4"), DUMP_KEEP: np.dtype("<f4"), DUMP_LUT: LUT_ENTRY,
    DUMP_TASKS: BINNING_TASK, DUMP_PROJECTED: PROJECTED_SEGMENT, DUMP_PAGE_TABLE: np.dtype("<u4"),
    DUMP_PAGE_META: FINE_PAGE_META, DUMP_COUNTS: np.dtype("<u4"), DUMP_OFFSETS: np.dtype("<u4"),
    DUMP_REFS: FINE_SEG_REF, DUMP_ACTIVE_TILES: np.dtype("<u4"), DUMP_WORK: RASTER_WORK_ITEM,
    DUMP_RUNS: RASTER_TILE_RUN, DUMP_DOM_DEPTH: np.dtype("<f4"), DUMP_DOM_OPACITY: np.dtype("<f4"),
    DUMP_SHADOW_MAP: np.dtype("<f4"), DUMP_ATLAS: np.dtype("<f2"), DUMP_HISTORY: np.dtype("<f2"),
    DUMP_COLOR: np.dtype("<f2"), DUMP_DEPTH: np.dtype("<f4"), DUMP_FRAGMENTS: np.dtype("<u4"),
    DUMP_OPAQUE_TILES: np.dtype("<u4"),
}

BATCH_ORDER_INDEX, BATCH_ORDER_LPT = 0, 1
TELEMETRY_HISTOGRAM_BINS, TELEMETRY_MAX_FRUSTA = 32, 16


class FrustumTelemetry(C.Structure):
    _fields_ = [(n, u32) for n in ("visible_instances", "visible_strands", "retained_strands", "emitted_segments",
                                   "allocated_pages", "page_candidates", "fine_refs", "raster_runs", "raster_load",
                                   "max_page_candidates", "max_raster_load")]


class Telemetry(C.Structure):
    _fields_ = [(n, u32) for n in ("allocated_pages", "binning_tasks", "page_candidates", "fine_cell_hits",
                                   "active_candidate_pages", "max_candidates_per_page", "frustum_count", "pad")] + [
        ("candidate_histogram", u32 * TELEMETRY_HISTOGRAM_BINS), ("frustum", FrustumTelemetry * TELEMETRY_MAX_FRUSTA)]


class BatchTuning(C.Structure):
    _fields_ = [("branches", u32), ("order", u32), ("ms", f32), ("pad", u32)]


# Every symbol include/fiber.h declares (checked by tests/test_abi.py).
EXPORTS = [
    "fiber_ctx_create", "fiber_ctx_destroy", "fiber_settings_default", "fiber_settings_set",
    "fiber_slab_alloc", "fiber_slab_upload", "fiber_slab_free", "fiber_instance_set", "fiber_frame_begin",
    "fiber_frame_begin_views",
    "fiber_opaque_depth", "fiber_prepass", "fiber_shadows", "fiber_shading", "fiber_raster", "fiber_composite", "fiber_frame_fused",
    "fiber_render_host", "fiber_stats_get", "fiber_telemetry_get", "fiber_dump", "fiber_output_image", "fiber_span_count", "fiber_span_name",
    "fiber_span_times", "fiber_status_string", "fiber_server_create", "fiber_server_add_scene",
    "fiber_server_start", "fiber_server_submit", "fiber_server_wait", "fiber_server_destroy", "fiber_server_now_ns",
    "fiber_batch_create", "fiber_batch_set_tuning", "fiber_batch_get_tuning", "fiber_batch_launch",
    "fiber_batch_tune", "fiber_batch_destroy", "fiber_batch_plan",
    "fiber_prefix_pages_noalloc", "fiber_debug_stall_lookback",
]

_LIB = None


class FiberError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}")
        self.status = status


def load_library(path: Path | str | None = None) -> C.CDLL:
    """Loads libfiber.so (built in-tree by bevy_strand_rasterizer_b200.build)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: run `python -m bevy_strand_rasterizer_b200.build`")
    lib = C.CDLL(str(p))
    vp, pp = C.c_void_p, C.POINTER
    sig = {
        "fiber_ctx_create": (C.c_int, [C.c_int, C.c_uint64, pp(vp)]),
        "fiber_ctx_destroy": (C.c_int, [vp]),
        "fiber_settings_default": (C.c_int, [pp(Settings)]),
        "fiber_settings_set": (C.c_int, [vp, pp(Settings)]),
        "fiber_slab_alloc": (C.c_int, [vp, u32, C.c_uint64, pp(u32), pp(DevicePtr)]),
        "fiber_slab_upload": (C.c_int, [vp, u32, u32, C.c_uint64, vp, C.c_uint64, vp]),
        "fiber_slab_free": (C.c_int, [vp, u32, u32]),
        "fiber_instance_set": (C.c_int, [vp, pp(StrandInstance), u32]),
        "fiber_frame_begin": (C.c_int, [vp, pp(FroxelConfigC), pp(Camera), pp(FroxelConfigC), pp(Light), u32, vp]),
        "fiber_frame_begin_views": (C.c_int, [vp, pp(View), u32, vp]),
        "fiber_opaque_depth": (C.c_int, [vp, pp(Image), u32, vp]),
        "fiber_prepass": (C.c_int, [vp, vp]),
        "fiber_shadows": (C.c_int, [vp, vp]),
        "fiber_shading": (C.c_int, [vp, vp]),
        "fiber_raster": (C.c_int, [vp, u32, vp]),
        "fiber_composite": (C.c_int, [vp, u32, pp(Image), pp(Image), pp(Image), vp]),
        "fiber_frame_fused": (C.c_int, [vp, pp(Image), pp(Image), pp(Image), vp]),
        "fiber_render_host": (C.c_int, [vp, vp, vp, vp, vp]),
        "fiber_stats_get": (C.c_int, [vp, pp(Stats)]),
        "fiber_debug_stall_lookback": (C.c_int, [vp, u32, u32, u32]),
        "fiber_telemetry_get": (C.c_int, [vp, pp(Telemetry)]),
        "fiber_dump": (C.c_int, [vp, u32, vp, C.c_uint64, pp(C.c_uint64)]),
        "fiber_output_image": (C.c_int, [vp, u32, pp(Image)]),
        "fiber_span_count": (u32, []),
        "fiber_span_name": (C.c_char_p, [u32]),
        "fiber_span_times": (C.c_int, [vp, pp(f32), u32]),
        "fiber_status_string": (C.c_char_p, [C.c_int]),
        "fiber_server_create": (C.c_int, [C.c_int, pp(Settings), pp(ServerConfig), pp(vp)]),
        "fiber_server_add_scene": (C.c_int, [vp, pp(ServerScene), pp(u32)]),
        "fiber_server_start": (C.c_int, [vp, pp(u32)]),
        "fiber_server_submit": (C.c_int, [vp, pp(ServerRequest), pp(C.c_uint64)]),
        "fiber_server_wait": (C.c_int, [vp, C.c_uint64, pp(ServerResult)]),
        "fiber_server_destroy": (C.c_int, [vp]),
        "fiber_server_now_ns": (C.c_uint64, []),
        "fiber_batch_create": (C.c_int, [pp(vp), u32, pp(vp)]),
        "fiber_batch_set_tuning": (C.c_int, [vp, pp(BatchTuning)]),
        "fiber_batch_get_tuning": (C.c_int, [vp, pp(BatchTuning)]),
        "fiber_batch_launch": (C.c_int, [vp, vp]),
        "fiber_batch_tune": (C.c_int, [vp, vp, pp(BatchTuning)]),
        "fiber_batch_destroy": (C.c_int, [vp]),
        "fiber_batch_plan": (C.c_int, [pp(f32), u32, u32, u32, pp(u32)]),
        "fiber_prefix_pages_noalloc": (C.c_int, [vp, u32, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def check(status: int, what: str, allow=(OK,)) -> int:
    if status not in allow:
        raise FiberError(status, what)
    return status


def default_settings() -> Settings:
    s = Settings()
    check(load_library().fiber_settings_default(C.byref(s)), "fiber_settings_default")
    return s
