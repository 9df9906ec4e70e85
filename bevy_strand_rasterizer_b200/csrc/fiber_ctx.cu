// fiber_ctx.cu — host runtime behind the C ABI (include/fiber.h).
//
// Mirrors the reference's plugin plumbing: slab allocation and the page
// tables of bevy_gpu_paging_allocator (src/plugin.rs:1395-1440, 129-160), the
// per-frame host preparation of use_prepass_buffers (src/plugin.rs:264-1209:
// frustum table, capacities, queue resets), and the render-graph node order
// (prepass -> shadows -> shading -> raster -> composite, src/plugin.rs:240-260).
// Device counts never travel back to the host inside a frame: every stage
// reads its item count from device memory, so a whole frame is one stream of
// launches that can be replayed from a CUDA graph.
#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fiber_internal.h"
#include "fiber_kernels.cuh"

using namespace fiber;

namespace {

constexpr int kSpanCount = 14;
const char* kSpanNames[kSpanCount] = {
    "strand_prepass/broad_instances",     // broad + depth-warp LUT
    "strand_prepass/fine",
    "strand_prepass/mark_count_pages",
    "strand_prepass/allocate_count_pages",
    "strand_prepass/binning",              // count
    "strand_prepass/prefix_fine_pages",
    "strand_prepass/fill_segment_refs",
    "strand_prepass/compact_active_tiles",
    "strand_prepass/emit_raster_work",     // emit + canonical cell order
    "strand_shadow_rasterizer/rasterize",  // incl. fused stampback
    "strand_shading/shade",
    "strand_rasterizer/rasterize",
    "strand_composite/composite",
    "frame/total",
};

struct Slab {
    void* ptr = nullptr;
    uint64_t bytes = 0;
    bool live = false;
};

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

int kind_slot(uint32_t kind) {
    switch (kind) {
        case FIBER_SLAB_VERT: return 0;
        case FIBER_SLAB_INDEX: return 1;
        case FIBER_SLAB_MATERIAL: return 2;
        case FIBER_SLAB_GEO: return 3;
        case FIBER_SLAB_META: return 4;
        default: return -1;
    }
}

// Checks one instance's slabs on the device: every index < vertex count, every
// strand range inside the index slab, every material index inside the material
// slab (validate_cache, src/strand_cache.rs:174-209). out: u32 errors at byte
// 0, u32 max count at byte 4, u64 segment total at byte 8 (8-byte aligned).
__global__ void k_validate(InstanceView v, uint32_t* out) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (uint32_t j = tid; j < v.n_indices; j += stride)
        if (v.indices[j] >= v.n_vertices) atomicOr(out + 0, 1u);
    unsigned long long segs = 0;
    uint32_t maxc = 0;
    for (uint32_t s = tid; s < v.n_meta; s += stride) {
        fiber_strand_meta m = v.meta[s];
        if (m.count < 2u) continue;
        if ((uint64_t)m.offset + m.count > v.n_indices) atomicOr(out + 0, 2u);
        if (m.material_idx >= v.n_materials) atomicOr(out + 0, 4u);
        segs += m.count - 1u;
        maxc = max(maxc, m.count);
    }
    atomicMax(out + 1, maxc);
    atomicAdd(reinterpret_cast<unsigned long long*>(out + 2), segs);
}

constexpr int kGraphKeyWords = 12;  // what a captured frame graph depends on (fiber_frame_fused)

}  // namespace

struct fiber_ctx {
    int device = 0;
    uint64_t budget = 0, allocated = 0;
    int sm_count = 148;
    fiber_settings settings{};
    std::vector<Slab> slabs[5];
    // registered instances
    std::vector<fiber_strand_instance> rows;
    std::vector<InstanceView> views;
    std::vector<uint64_t> inst_segments;
    uint64_t total_segments = 0, total_points = 0, total_strands = 0;
    uint32_t max_texels = 0, total_strand_count = 0, max_strand_count = 0;
    // frame description
    FrameParams P{};
    std::vector<fiber_frustum_desc> frusta;
    bool frame_ready = false;
    uint32_t epoch = 0;
    uint32_t lb_offset[kStageCount] = {0};
    // device buffers
    DevBuf d_params, d_inst, d_counters, d_lb, d_range_valid, d_ranges, d_keep, d_inst_visible, d_inst_keep;
    DevBuf d_lut_tree;  // per coarse tile: the slice lookup's search tree (kLutTreeWords)
    DevBuf d_lut, d_tasks, d_projected, d_page_table, d_page_meta, d_counts, d_offsets, d_cursors;
    DevBuf d_refs, d_ref_keys, d_active_flags, d_active_list, d_work, d_runs, d_big_cells;
    DevBuf d_visit_rec, d_visit_task, d_visit_rank, d_task_key, d_task_mat, d_cells_small, d_cells_mid, d_cells_large;
    DevBuf d_opaque;  // (covered, farthest depth q) per camera fine tile
    DevBuf d_task_proj, d_ref_task;  // k_fine's projected end points per task; each reference's task
    DevBuf d_page_nvis, d_page_vbase, d_page_bucket;  // page-CSR backend
    DevBuf d_tel, d_tel_slots;                         // prepass telemetry
    DevBuf d_dom_page_table, d_dom_pool;               // sparse DOM residency
    // fiber_render_host: the scene image's upload runs on its own stream
    // beside the frame; ev_in = uploaded, ev_out = the last download queued.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    // The prepass's cell sort runs on this stream beside the emit.
    cudaStream_t side_stream = nullptr;
    cudaStream_t side_override = nullptr;  // fiber_ctx_set_side_stream (request server priorities)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    uint32_t camera_fine_tiles = 0;
    bool opaque_frame = false;  // fiber_opaque_depth ran since fiber_frame_begin
    // A batch graph advanced this context's epoch on the device: the next
    // fiber_frame_begin clears the look-back words and restarts the epoch.
    bool epoch_dirty = false;
    // fiber_debug_stall_lookback: the next frame's look-back test hook.
    uint32_t stall_stage = 0, stall_tile = 0, stall_limit = 0;
    // Smallest reference capacity of the next frames (the request server
    // raises it after a frame whose references overflowed).
    uint64_t ref_floor = 0;
    // The frame's views (fiber_frame_begin_views) and the pixels of their
    // concatenated colour / depth / fragment images.
    uint32_t n_views = 1;
    uint64_t out_pixels = 0;
    // The last fiber_frame_begin's view, for a batch's multi-view frame.
    fiber_view last_view{};
    std::vector<fiber_froxel_config> last_light_cfgs;
    std::vector<fiber_light> last_lights;
    DevBuf d_dom_depth, d_dom_opacity, d_shadow_map, d_atlas, d_history[2];
    DevBuf d_color, d_depth, d_fragments, d_validate, d_host_scene, d_host_depth;
    int hist_cur = 0;
    // timing
    cudaEvent_t ev[kSpanCount + 1] = {};
    bool events_ok = false;
    cudaStream_t last_stream = nullptr;
    // graph replay of fiber_frame_fused
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_key[kGraphKeyWords] = {0};
    uint64_t buffer_generation = 0, graph_generation = ~0ull;
    FrameCounters h_counters{};
};

namespace {

#define FIBER_CUDA(expr)                                         \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return FIBER_ECUDA;               \
    } while (0)

fiber_status ensure(fiber_ctx* c, DevBuf& b, size_t bytes, bool zero = false) {
    if (bytes == 0) bytes = 16;
    bytes = (bytes + 255) & ~size_t(255);
    if (b.p && b.bytes >= bytes) return FIBER_OK;
    if (c->budget && c->allocated - b.bytes + bytes > c->budget) return FIBER_ENOMEM;
    if (b.p) {
        cudaFree(b.p);
        c->allocated -= b.bytes;
        b.p = nullptr;
        b.bytes = 0;
    }
    if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return FIBER_ENOMEM;
    }
    b.bytes = bytes;
    c->allocated += bytes;
    c->buffer_generation++;
    if (zero) FIBER_CUDA(cudaMemset(b.p, 0, bytes));
    return FIBER_OK;
}

void release(fiber_ctx* c, DevBuf& b) {
    if (b.p) {
        cudaFree(b.p);
        c->allocated -= b.bytes;
    }
    b.p = nullptr;
    b.bytes = 0;
}

template <typename T>
T* dp(const DevBuf& b) { return static_cast<T*>(b.p); }

void cfg_tiles(const fiber_froxel_config& cfg, uint32_t& tx, uint32_t& ty) {
    tx = (cfg.screen_width + cfg.froxel_size_x - 1u) / cfg.froxel_size_x;
    ty = (cfg.screen_height + cfg.froxel_size_y - 1u) / cfg.froxel_size_y;
}

LaunchCtx launch_ctx(fiber_ctx* c, cudaStream_t s) {
    LaunchCtx L;
    L.stream = s;
    L.P = dp<FrameParams>(c->d_params);
    L.inst = dp<InstanceView>(c->d_inst);
    L.I = c->P.I;
    L.total_coarse_tiles = c->P.total_coarse_tiles;
    L.sm_count = c->sm_count;
    L.opaque = c->opaque_frame;
    L.telemetry = c->settings.telemetry_enabled != 0u;
    return L;
}

PrepassArgs prepass_args(fiber_ctx* c) {
    PrepassArgs A{};
    A.counters = dp<FrameCounters>(c->d_counters);
    A.range_valid = dp<uint32_t>(c->d_range_valid);
    A.ranges = dp<fiber_coarse_asset_range>(c->d_ranges);
    A.keep = dp<float>(c->d_keep);
    A.inst_visible = dp<uint32_t>(c->d_inst_visible);
    A.inst_keep = dp<float>(c->d_inst_keep);
    A.lut = dp<fiber_coarse_depth_lut_entry>(c->d_lut);
    A.lut_tree = dp<uint32_t>(c->d_lut_tree);
    A.tasks = dp<fiber_binning_task>(c->d_tasks);
    A.projected = dp<fiber_projected_segment>(c->d_projected);
    A.page_table = dp<uint32_t>(c->d_page_table);
    A.page_meta = dp<fiber_fine_page_meta>(c->d_page_meta);
    A.counts = dp<uint32_t>(c->d_counts);
    A.offsets = dp<uint32_t>(c->d_offsets);
    A.cursors = dp<uint32_t>(c->d_cursors);
    A.refs = dp<fiber_fine_seg_ref>(c->d_refs);
    A.ref_keys = dp<uint32_t>(c->d_ref_keys);
    A.active_flags = dp<uint32_t>(c->d_active_flags);
    A.active_list = dp<uint32_t>(c->d_active_list);
    A.work = dp<fiber_raster_work_item>(c->d_work);
    A.runs = dp<fiber_raster_tile_run>(c->d_runs);
    A.big_cells = dp<uint2>(c->d_big_cells);
    A.visit_rec = dp<uint32_t>(c->d_visit_rec);
    A.visit_task = dp<uint32_t>(c->d_visit_task);
    A.visit_rank = dp<uint32_t>(c->d_visit_rank);
    A.task_key = dp<unsigned long long>(c->d_task_key);
    A.task_mat = dp<uint32_t>(c->d_task_mat);
    A.cells_small = dp<uint2>(c->d_cells_small);
    A.cells_mid = dp<uint2>(c->d_cells_mid);
    A.cells_large = dp<uint2>(c->d_cells_large);
    A.opaque_tiles = dp<uint2>(c->d_opaque);
    A.task_proj = dp<float4>(c->d_task_proj);
    A.ref_task = dp<uint32_t>(c->d_ref_task);
    if (c->settings.telemetry_enabled) {
        A.tel = dp<uint32_t>(c->d_tel);
        A.tel_slots = dp<uint32_t>(c->d_tel_slots);
    }
    if (c->settings.fine_binning_backend == 1u) {
        A.page_nvis = dp<uint32_t>(c->d_page_nvis);
        A.page_vbase = dp<uint32_t>(c->d_page_vbase);
        A.page_bucket = dp<uint2>(c->d_page_bucket);
    }
    return A;
}

void set_stage(fiber_ctx* c, PrepassArgs& A, uint32_t stage) {
    A.tile_counter = &dp<FrameCounters>(c->d_counters)->tile_counter[stage];
    A.lb_status = dp<unsigned long long>(c->d_lb) + c->lb_offset[stage];
}

RenderArgs render_args(fiber_ctx* c) {
    RenderArgs R{};
    R.counters = dp<FrameCounters>(c->d_counters);
    R.tasks = dp<fiber_binning_task>(c->d_tasks);
    R.refs = dp<fiber_fine_seg_ref>(c->d_refs);
    R.work = dp<fiber_raster_work_item>(c->d_work);
    R.runs = dp<fiber_raster_tile_run>(c->d_runs);
    R.ref_task = dp<uint32_t>(c->d_ref_task);
    R.task_proj = dp<float4>(c->d_task_proj);
    R.dom_depth = dp<float>(c->d_dom_depth);
    R.dom_opacity = dp<float>(c->d_dom_opacity);
    R.dom_page_table = dp<uint32_t>(c->d_dom_page_table);
    R.dom_pool = dp<float>(c->d_dom_pool);
    R.shadow_map = dp<float>(c->d_shadow_map);
    R.atlas = dp<__half>(c->d_atlas);
    R.history[0] = dp<__half>(c->d_history[0]);
    R.history[1] = dp<__half>(c->d_history[1]);
    R.color = dp<__half>(c->d_color);
    R.depth = dp<float>(c->d_depth);
    R.fragments = dp<uint32_t>(c->d_fragments);
    return R;
}

// Span events: while a stream is being captured they are recorded as external
// event nodes, so they keep timing the frame when it is replayed from the CUDA
// graph; otherwise they are plain records. A failed record only disables the
// spans; it never leaves an error behind for the node that called it.
void record(fiber_ctx* c, int span, cudaStream_t s) {
    if (!c->events_ok) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (s && cudaStreamIsCapturing(s, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cs == cudaStreamCaptureStatusActive
                        ? cudaEventRecordWithFlags(c->ev[span], s, cudaEventRecordExternal)
                        : cudaEventRecord(c->ev[span], s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->events_ok = false;
    }
}

fiber_status check_launch() {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FIBER_OK : FIBER_ECUDA;
}

// Per-frame clears of src/plugin.rs:1145-1208 that follow the frame-table
// upload: counters, page table, active flags, colour / depth / fragment
// targets and the DOM depth + stampback target.
fiber_status frame_resets(fiber_ctx* c, cudaStream_t s) {
    const FrameParams& P = c->P;
    const uint64_t table = (uint64_t)P.total_coarse_tiles * kDepthSlices;
    const uint64_t WH = c->out_pixels, L = P.L, D = P.dom_size, S = P.shadow_map_size;
    FIBER_CUDA(cudaMemsetAsync(c->d_counters.p, 0, sizeof(FrameCounters), s));
    FIBER_CUDA(cudaMemsetAsync(c->d_page_table.p, 0, table * 4, s));
    FIBER_CUDA(cudaMemsetAsync(c->d_active_flags.p, 0, table * 4, s));
    FIBER_CUDA(cudaMemsetAsync(c->d_color.p, 0, WH * 8, s));
    FIBER_CUDA(cudaMemsetAsync(c->d_depth.p, 0, WH * 4, s));
    if (P.fragment_counts) FIBER_CUDA(cudaMemsetAsync(c->d_fragments.p, 0, WH * 4, s));
    if (L) {
        if (P.dom_pool_pages) {
            const uint64_t ppx = P.dom_pages_x;
            FIBER_CUDA(cudaMemsetAsync(c->d_dom_page_table.p, 0, L * ppx * ppx * 4, s));
        } else {
            FIBER_CUDA(cudaMemsetAsync(c->d_dom_depth.p, 0, L * D * D * 4, s));
        }
        FIBER_CUDA(cudaMemsetAsync(c->d_shadow_map.p, 0, L * S * S * 4, s));
    }
    if (c->settings.telemetry_enabled) {
        FIBER_CUDA(cudaMemsetAsync(c->d_tel.p, 0, sizeof(fiber_telemetry), s));
        FIBER_CUDA(cudaMemsetAsync(c->d_tel_slots.p, 0, table * 4, s));
    }
    return FIBER_OK;
}

// The device half of fiber_frame_begin for a frame replayed from a graph: the
// next look-back epoch (on wrap-around the status words are cleared first, as
// the host does) and the shadow-history ping-pong flip. One block.
__global__ void k_frame_advance(FrameParams* P, unsigned long long* lb, uint64_t lb_words) {
    __shared__ uint32_t s_epoch;
    if (threadIdx.x == 0) s_epoch = (P->epoch + 1u) & 0x3FFFFFFFu;
    __syncthreads();
    const uint32_t e = s_epoch;
    if (e == 0u)
        for (uint64_t i = threadIdx.x; i < lb_words; i += blockDim.x) lb[i] = 0ull;
    if (threadIdx.x == 0) {
        P->epoch = e == 0u ? 1u : e;
        P->hist_in ^= 1u;
    }
}

// The camera's opaque depth for K0: R32F rows of width * samples floats.
struct OpaqueSource {
    const float* depth;
    uint32_t pitch, samples;
};

fiber_status run_prepass(fiber_ctx* c, cudaStream_t s, const OpaqueSource* opaque = nullptr) {
    LaunchCtx L = launch_ctx(c, s);
    PrepassArgs A = prepass_args(c);
    record(c, 0, s);
    if (opaque) {
        launch_opaque(L, A, opaque->depth, opaque->pitch, opaque->samples, c->camera_fine_tiles);
        L.opaque = true;
    }
    launch_broad(L, A);
    launch_lut(L, A);
    record(c, 1, s);
    set_stage(c, A, kStageFine);
    launch_fine(L, A);
    record(c, 2, s);
    launch_visit(L, A);
    record(c, 3, s);
    set_stage(c, A, kStageAlloc);
    launch_alloc(L, A);
    launch_zero_pages(L, A);
    // FineBinningBackend (src/pipelines/prepass.rs:1261-1295): segment-owned
    // count / prefix / fill, or the page CSR with page-owned cell building.
    const bool csr = c->settings.fine_binning_backend == 1u;
    record(c, 4, s);
    if (csr) launch_page_csr_count(L, A);
    else launch_count(L, A);
    record(c, 5, s);
    set_stage(c, A, kStagePrefix);
    launch_prefix(L, A, csr);
    if (csr) launch_build_pages(L, A);
    record(c, 6, s);
    if (csr) launch_fill_walk(L, A);
    else launch_fill(L, A);
    record(c, 7, s);
    // The cell sort needs only the fill; the active-tile compaction and the
    // emit need only the counts. The sort runs on the side stream beside
    // them (a branch of the frame graph when captured) and joins before the
    // rasters.
    cudaStream_t side = c->side_override ? c->side_override : c->side_stream;
    FIBER_CUDA(cudaEventRecord(c->ev_fork, s));
    FIBER_CUDA(cudaStreamWaitEvent(side, c->ev_fork, 0));
    LaunchCtx Ls = L;
    Ls.stream = side;
    launch_sort_cells(Ls, A);
    launch_sort_big(Ls, A);
    FIBER_CUDA(cudaEventRecord(c->ev_join, side));
    set_stage(c, A, kStageActive);
    launch_compact_active(L, A);
    record(c, 8, s);
    set_stage(c, A, kStageEmit);
    launch_emit(L, A);
    FIBER_CUDA(cudaStreamWaitEvent(s, c->ev_join, 0));
    if (L.telemetry) launch_telemetry(L, A);
    return check_launch();
}

fiber_status run_shadows(fiber_ctx* c, cudaStream_t s) {
    record(c, 9, s);
    if (c->P.L) {
        const LaunchCtx L = launch_ctx(c, s);
        const RenderArgs R = render_args(c);
        if (c->P.dom_pool_pages) launch_dom_paging(L, R, c->P.L * c->P.dom_pages_x * c->P.dom_pages_x);
        launch_shadow(L, R, c->P.K);
    }
    return check_launch();
}

fiber_status run_shading(fiber_ctx* c, cudaStream_t s) {
    record(c, 10, s);
    launch_shade(launch_ctx(c, s), render_args(c));
    c->hist_cur = 1 - c->hist_cur;  // shadow-history ping-pong flip (pipelines/shading.rs:564-566)
    return check_launch();
}

fiber_status run_raster(fiber_ctx* c, cudaStream_t s) {
    record(c, 11, s);
    launch_raster(launch_ctx(c, s), render_args(c));
    return check_launch();
}

uint32_t fmt_bytes(uint32_t fmt) {
    return fmt == FIBER_FMT_RGBA16F ? 8u : (fmt == FIBER_FMT_R32F ? 4u : 16u);
}

// Checks an opaque depth image against the camera (R32F, camera extent,
// `samples` floats per pixel, rows 4-byte aligned and wide enough).
fiber_status opaque_source(const fiber_ctx* c, const fiber_image* im, uint32_t samples, OpaqueSource& o) {
    if (!im || !im->ptr || im->format != FIBER_FMT_R32F || (samples != 1u && samples != 4u)) return FIBER_EINVAL;
    if (c->n_views != 1u) return FIBER_EINVAL;  // the opaque-scene cull is one camera's
    if (im->width != c->P.width || im->height != c->P.height) return FIBER_EINVAL;
    const uint64_t row = (uint64_t)im->width * samples * 4u;
    const uint64_t pitch = im->pitch ? im->pitch : row;
    if (pitch < row || pitch % 4u || pitch > 0xFFFFFFFFull || (uintptr_t)im->ptr % 4u) return FIBER_EINVAL;
    o.depth = static_cast<const float*>(im->ptr);
    o.pitch = (uint32_t)pitch;
    o.samples = samples;
    return FIBER_OK;
}

fiber_status run_composite(fiber_ctx* c, const fiber_image* scene_color, const fiber_image* scene_depth,
                           fiber_image* out, cudaStream_t s) {
    record(c, 12, s);
    if (!scene_color || !out || !scene_color->ptr || !out->ptr) return FIBER_EINVAL;
    if (c->n_views != 1u) return FIBER_EINVAL;  // a multi-view frame has no single scene image
    if (scene_color->width != c->P.width || scene_color->height != c->P.height || out->width != c->P.width ||
        out->height != c->P.height)
        return FIBER_EINVAL;
    if (scene_color->format == FIBER_FMT_R32F || out->format == FIBER_FMT_R32F) return FIBER_EINVAL;
    if (scene_depth && (scene_depth->format != FIBER_FMT_R32F || scene_depth->width != c->P.width ||
                        scene_depth->height != c->P.height))
        return FIBER_EINVAL;
    // Vector loads need 8 B (RGBA16F) / 16 B (RGBA32F) / 4 B (R32F) aligned rows.
    auto aligned = [](const fiber_image* im, uint32_t px_bytes) {
        uint32_t pitch = im->pitch ? im->pitch : im->width * px_bytes;
        return ((uintptr_t)im->ptr % px_bytes) == 0 && pitch % px_bytes == 0 && pitch >= im->width * px_bytes;
    };
    if (!aligned(scene_color, fmt_bytes(scene_color->format)) || !aligned(out, fmt_bytes(out->format)) ||
        (scene_depth && !aligned(scene_depth, 4u)))
        return FIBER_EINVAL;
    CompositeArgs C{};
    C.strand_color = dp<__half>(c->d_color);
    C.strand_depth = dp<float>(c->d_depth);
    C.scene_color = scene_color->ptr;
    C.scene_pitch = scene_color->pitch ? scene_color->pitch : scene_color->width * fmt_bytes(scene_color->format);
    C.scene_format = scene_color->format;
    C.scene_depth = scene_depth ? static_cast<const float*>(scene_depth->ptr) : nullptr;
    C.depth_pitch = scene_depth ? (scene_depth->pitch ? scene_depth->pitch : scene_depth->width * 4u) : 0u;
    C.out = out->ptr;
    C.out_pitch = out->pitch ? out->pitch : out->width * fmt_bytes(out->format);
    C.out_format = out->format;
    C.width = c->P.width;
    C.height = c->P.height;
    launch_composite(s, C);
    return check_launch();
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* fiber_status_string(fiber_status s) {
    switch (s) {
        case FIBER_OK: return "ok";
        case FIBER_EINVAL: return "invalid argument";
        case FIBER_ENOMEM: return "out of device memory or HBM budget";
        case FIBER_EOVERFLOW: return "device queue overflow";
        case FIBER_ETIMEDOUT: return "bounded device wait timed out";
        case FIBER_ECUDA: return "CUDA runtime error";
        case FIBER_ENOTREADY: return "inputs not ready";
        default: return "unknown";
    }
}

fiber_status fiber_settings_default(fiber_settings* s) {
    if (!s) return FIBER_EINVAL;
    std::memset(s, 0, sizeof(*s));
    s->stochastic_cull_enabled = 1u;          // StochasticCullSettings::default (src/resources.rs:95-104)
    s->target_strands_per_pixel = 2.0f;
    s->min_keep_probability = 0.02f;
    s->shadow_keep_probability = 1.0f;
    s->telemetry_enabled = 0u;
    s->fine_binning_backend = 0u;             // SegmentScatter
    s->dom_slices = 12u;                      // NUM_DOM_SLICES (src/pipelines/shadows.rs:38)
    s->shadow_map_size = 0u;
    s->ambient_color[0] = s->ambient_color[1] = s->ambient_color[2] = 80.0f;  // AmbientLight default x brightness
    s->ambient_color[3] = 80.0f;
    s->history_enabled = 1u;
    s->fragment_counts_enabled = 0u;
    s->ref_capacity_factor = 4u;              // fine refs = 4 x binning (src/plugin.rs:536-540)
    s->page_capacity_divisor = 1u;
    s->dom_page_pool = 0u;                    // dense deep-opacity layers
    return FIBER_OK;
}

fiber_status fiber_ctx_create(int device, uint64_t hbm_budget, fiber_ctx** out) {
    if (!out) return FIBER_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return FIBER_EINVAL;
    }
    FIBER_CUDA(cudaSetDevice(device));
    fiber_ctx* c = new fiber_ctx();
    c->device = device;
    c->budget = hbm_budget;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    fiber_settings_default(&c->settings);
    c->events_ok = true;
    for (int i = 0; i <= kSpanCount; ++i)
        if (cudaEventCreate(&c->ev[i]) != cudaSuccess) c->events_ok = false;
    fiber_status st = FIBER_OK;
    if (cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        st = FIBER_ECUDA;
    }
    if (st == FIBER_OK) st = ensure(c, c->d_counters, sizeof(FrameCounters), true);
    if (st == FIBER_OK) st = ensure(c, c->d_validate, 64, true);
    if (st != FIBER_OK) {
        fiber_ctx_destroy(c);
        return st;
    }
    *out = c;
    return FIBER_OK;
}

fiber_status fiber_ctx_destroy(fiber_ctx* c) {
    if (!c) return FIBER_EINVAL;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (auto& v : c->slabs)
        for (auto& s : v)
            if (s.live && s.ptr) cudaFree(s.ptr);
    DevBuf* bufs[] = {&c->d_params, &c->d_inst, &c->d_counters, &c->d_lb, &c->d_range_valid, &c->d_ranges,
                      &c->d_keep, &c->d_inst_visible, &c->d_inst_keep, &c->d_lut, &c->d_lut_tree, &c->d_tasks, &c->d_projected,
                      &c->d_page_table, &c->d_page_meta, &c->d_counts, &c->d_offsets, &c->d_cursors, &c->d_refs,
                      &c->d_ref_keys, &c->d_active_flags, &c->d_active_list, &c->d_work, &c->d_runs,
                      &c->d_big_cells, &c->d_dom_depth, &c->d_dom_opacity, &c->d_shadow_map, &c->d_atlas,
                      &c->d_history[0], &c->d_history[1], &c->d_color, &c->d_depth, &c->d_fragments,
                      &c->d_validate, &c->d_host_scene, &c->d_host_depth, &c->d_visit_rec,
                      &c->d_visit_task, &c->d_visit_rank, &c->d_task_key, &c->d_task_mat,
                      &c->d_cells_small, &c->d_cells_mid, &c->d_cells_large, &c->d_opaque, &c->d_page_nvis, &c->d_page_vbase,
                      &c->d_page_bucket, &c->d_tel, &c->d_tel_slots, &c->d_dom_page_table, &c->d_dom_pool,
                      &c->d_task_proj, &c->d_ref_task};
    for (DevBuf* b : bufs) release(c, *b);
    for (int i = 0; i <= kSpanCount; ++i)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->side_stream) cudaStreamDestroy(c->side_stream);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->ev_in) cudaEventDestroy(c->ev_in);
    if (c->ev_out) cudaEventDestroy(c->ev_out);
    delete c;
    return FIBER_OK;
}

fiber_status fiber_settings_set(fiber_ctx* c, const fiber_settings* s) {
    if (!c || !s) return FIBER_EINVAL;
    if (s->dom_slices == 0u || s->dom_slices > 16u) return FIBER_EINVAL;
    if (s->ref_capacity_factor == 0u || s->page_capacity_divisor == 0u) return FIBER_EINVAL;
    if (s->fine_binning_backend > 1u) return FIBER_EINVAL;  // SegmentScatter or PageCsr
    c->settings = *s;
    c->frame_ready = false;
    c->buffer_generation++;  // the captured frame graphs follow the settings' kernel sequence
    return FIBER_OK;
}

fiber_status fiber_slab_alloc(fiber_ctx* c, uint32_t kind, uint64_t bytes, uint32_t* alloc_id, fiber_devptr* out) {
    if (!c || !alloc_id || bytes == 0 || bytes > 0xFFFFFFFFull) return FIBER_EINVAL;
    int k = kind_slot(kind);
    if (k < 0) return FIBER_EINVAL;
    if (kind == FIBER_SLAB_VERT && bytes % 16u) return FIBER_EINVAL;  // float4 vertex stride
    if (c->budget && c->allocated + bytes > c->budget) return FIBER_ENOMEM;
    cudaSetDevice(c->device);
    Slab s;
    if (cudaMalloc(&s.ptr, bytes) != cudaSuccess) {
        cudaGetLastError();
        return FIBER_ENOMEM;
    }
    s.bytes = bytes;
    s.live = true;
    c->allocated += bytes;
    c->slabs[k].push_back(s);
    *alloc_id = (uint32_t)(c->slabs[k].size() - 1);
    if (out) *out = fiber_devptr{*alloc_id, 0u, (uint32_t)bytes};
    return FIBER_OK;
}

fiber_status fiber_slab_upload(fiber_ctx* c, uint32_t kind, uint32_t alloc_id, uint64_t dst_offset, const void* host,
                               uint64_t bytes, void* stream) {
    if (!c || !host) return FIBER_EINVAL;
    int k = kind_slot(kind);
    if (k < 0 || alloc_id >= c->slabs[k].size() || !c->slabs[k][alloc_id].live) return FIBER_EINVAL;
    const Slab& s = c->slabs[k][alloc_id];
    if (dst_offset + bytes > s.bytes) return FIBER_EINVAL;
    cudaSetDevice(c->device);
    FIBER_CUDA(cudaMemcpyAsync(static_cast<char*>(s.ptr) + dst_offset, host, bytes, cudaMemcpyHostToDevice,
                               (cudaStream_t)stream));
    return FIBER_OK;
}

fiber_status fiber_slab_free(fiber_ctx* c, uint32_t kind, uint32_t alloc_id) {
    if (!c) return FIBER_EINVAL;
    int k = kind_slot(kind);
    if (k < 0 || alloc_id >= c->slabs[k].size() || !c->slabs[k][alloc_id].live) return FIBER_EINVAL;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    Slab& s = c->slabs[k][alloc_id];
    cudaFree(s.ptr);
    c->allocated -= s.bytes;
    s = Slab{};
    c->frame_ready = false;
    return FIBER_OK;
}

fiber_status fiber_instance_set(fiber_ctx* c, const fiber_strand_instance* rows, uint32_t n) {
    if (!c || (n && !rows)) return FIBER_EINVAL;
    if (n >= 32768u) return FIBER_EINVAL;  // instance ids are 15 bits in the cell sort key
    cudaSetDevice(c->device);
    FIBER_CUDA(cudaDeviceSynchronize());
    std::vector<InstanceView> views(n);
    std::vector<uint64_t> segs(n, 0);
    uint64_t tot_seg = 0, tot_pts = 0, tot_str = 0;
    uint32_t max_tex = 0, strand_base = 0, max_strands = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const fiber_strand_instance& r = rows[i];
        InstanceView& v = views[i];
        std::memset(&v, 0, sizeof(v));
        auto get = [&](uint32_t kind, uint32_t id) -> const Slab* {
            int k = kind_slot(kind);
            if (id >= c->slabs[k].size() || !c->slabs[k][id].live) return nullptr;
            return &c->slabs[k][id];
        };
        const Slab *sv = get(FIBER_SLAB_VERT, r.vertex_id), *si = get(FIBER_SLAB_INDEX, r.index_id);
        const Slab *sm = get(FIBER_SLAB_META, r.meta_id), *sg = get(FIBER_SLAB_GEO, r.geo_id);
        const Slab* sa = get(FIBER_SLAB_MATERIAL, r.material_id);
        if (!sv || !si || !sm || !sg || !sa || sg->bytes < sizeof(fiber_strand_geo) ||
            sa->bytes < sizeof(fiber_strand_material))
            return FIBER_EINVAL;
        fiber_strand_geo geo;
        FIBER_CUDA(cudaMemcpy(&geo, sg->ptr, sizeof(geo), cudaMemcpyDeviceToHost));
        v.vertices = static_cast<const float4*>(sv->ptr);
        v.indices = static_cast<const uint32_t*>(si->ptr);
        v.meta = static_cast<const fiber_strand_meta*>(sm->ptr);
        v.materials = static_cast<const fiber_strand_material*>(sa->ptr);
        v.n_vertices = (uint32_t)(sv->bytes / 16u);
        v.n_indices = (uint32_t)(si->bytes / 4u);
        v.n_meta = (uint32_t)(sm->bytes / sizeof(fiber_strand_meta));
        v.n_materials = (uint32_t)(sa->bytes / sizeof(fiber_strand_material));
        v.strand_count = std::min(v.n_meta, geo.strand_count);
        v.strand_base = strand_base;
        v.valid = 1u;
        v.aabb = geo.aabb;
        std::memcpy(v.world_from_local, r.world_from_local, sizeof(v.world_from_local));
        // Device-side validation.
        FIBER_CUDA(cudaMemset(c->d_validate.p, 0, 16));
        k_validate<<<std::max(1, c->sm_count * 2), 256>>>(v, dp<uint32_t>(c->d_validate));
        uint32_t res[4];
        FIBER_CUDA(cudaMemcpy(res, c->d_validate.p, 16, cudaMemcpyDeviceToHost));
        if (res[0] != 0u) return FIBER_EINVAL;
        segs[i] = (uint64_t)res[2] | ((uint64_t)res[3] << 32);
        tot_seg += segs[i];
        tot_pts += v.n_indices;
        tot_str += v.strand_count;
        strand_base += v.strand_count;
        max_strands = std::max(max_strands, v.strand_count);
        max_tex = std::max(max_tex, v.n_indices);
    }
    if (tot_str >= 0xFFFFFFFFull || tot_seg >= 0x3FFFFFFFull) return FIBER_EINVAL;
    c->rows.assign(rows, rows + n);
    c->views = views;
    c->inst_segments = segs;
    c->total_segments = tot_seg;
    c->total_points = tot_pts;
    c->total_strands = tot_str;
    c->total_strand_count = strand_base;
    c->max_strand_count = max_strands;
    c->max_texels = max_tex;
    c->frame_ready = false;
    return FIBER_OK;
}

// The frame tables of one frame of nv views (use_prepass_buffers,
// src/plugin.rs:264-1209): frusta, clip matrices, capacities, buffers, resets.
// A frame of fiber_frame_begin is one view over every instance.
static fiber_status frame_begin_views(fiber_ctx* c, const fiber_view* views, uint32_t nv, cudaStream_t s) {
    if (!c || !views || nv == 0u || nv > kMaxViews) return FIBER_EINVAL;
    const fiber_settings& st = c->settings;
    const uint32_t I = (uint32_t)c->views.size();
    auto cfg_ok = [](const fiber_froxel_config& g) {
        return g.screen_width && g.screen_height && g.froxel_size_x && g.froxel_size_y && g.screen_width <= 16384u &&
               g.screen_height <= 16384u;
    };
    uint32_t n_frusta = 0, n_lights = 0, dmax = 0, inst_next = 0;
    for (uint32_t v = 0; v < nv; ++v) {
        const fiber_view& w = views[v];
        if (!cfg_ok(w.camera_cfg) || (w.n_lights && (!w.light_cfgs || !w.lights))) return FIBER_EINVAL;
        // The views' instances follow one another in the instance table, and
        // every view of several has strands (its frusta then have tasks' bases).
        if (w.instance_first != inst_next || w.instance_first + w.instance_count > I) return FIBER_EINVAL;
        if (nv > 1u) {
            uint32_t ns = 0;
            for (uint32_t i = w.instance_first; i < w.instance_first + w.instance_count; ++i)
                ns += c->views[i].strand_count;
            if (ns == 0u) return FIBER_EINVAL;
        }
        inst_next += w.instance_count;
        for (uint32_t l = 0; l < w.n_lights; ++l) {
            const fiber_froxel_config& g = w.light_cfgs[l];
            // Dense deep-opacity layers are square; one view's maps are one size.
            if (!cfg_ok(g) || g.screen_width != g.screen_height || g.screen_width != w.light_cfgs[0].screen_width)
                return FIBER_EINVAL;
            dmax = std::max(dmax, g.screen_width);
        }
        n_frusta += 1u + w.n_lights;
        n_lights += w.n_lights;
    }
    if (inst_next != I && nv > 1u) return FIBER_EINVAL;
    if (nv == 1u ? n_frusta > FIBER_MAX_FRUSTA : n_frusta > kMaxFrusta) return FIBER_EINVAL;
    // Several views: dense layers of the largest map, no per-frustum telemetry
    // beyond its 16 frusta, no opaque-scene cull (a single camera's).
    if (nv > 1u && (st.dom_page_pool != 0u || (st.telemetry_enabled && n_frusta > FIBER_TELEMETRY_MAX_FRUSTA)))
        return FIBER_EINVAL;
    cudaSetDevice(c->device);
    FrameParams& P = c->P;
    std::memset(&P, 0, sizeof(P));
    P.lb_spin_limit = c->stall_limit;
    P.lb_stall_stage = c->stall_stage;
    P.lb_stall_tile = c->stall_tile;
    c->stall_stage = c->stall_tile = c->stall_limit = 0;
    for (uint32_t i = 0; i < I; ++i) c->views[i].view = 0u;
    for (uint32_t v = 0; v < nv && nv > 1u; ++v)
        for (uint32_t i = views[v].instance_first; i < views[v].instance_first + views[v].instance_count; ++i)
            c->views[i].view = v;
    // Frustum table (src/plugin.rs:386-482): the cameras first (frustum v is
    // view v's camera), then each view's lights in order.
    c->frusta.clear();
    uint32_t bucket = 0, coarse = 0, fine = 0, cam_tiles = 0, light = 0;
    uint64_t out_pixels = 0;
    for (uint32_t f = 0; f < n_frusta; ++f) {
        const bool cam = f < nv;
        uint32_t v = f, l = 0;  // view, light index inside the view
        if (!cam) {
            uint32_t k = f - nv;
            for (v = 0; k >= views[v].n_lights; ++v) k -= views[v].n_lights;
            l = k;
        }
        const fiber_froxel_config& g = cam ? views[v].camera_cfg : views[v].light_cfgs[l];
        uint32_t tx, ty;
        cfg_tiles(g, tx, ty);
        uint32_t ctx_ = std::max(1u, (tx + 3u) / 4u), cty = std::max(1u, (ty + 3u) / 4u);
        fiber_frustum_desc d{};
        d.screen_width = g.screen_width;
        d.screen_height = g.screen_height;
        d.froxel_size_x = g.froxel_size_x;
        d.froxel_size_y = g.froxel_size_y;
        d.depth_slices = g.depth_slices;
        d.bucket_base = bucket;
        d.bucket_count = tx * ty * g.depth_slices;
        d.kind = cam ? 0u : 1u;
        d.coarse_depth_tile_base = coarse;
        d.coarse_depth_tile_count = ctx_ * cty;
        d.coarse_tiles_x = ctx_;
        d.coarse_tiles_y = cty;
        d.cascade_index = 0u;
        d.fine_depth_tile_base = fine;
        c->frusta.push_back(d);
        bucket += d.bucket_count;
        coarse += d.coarse_depth_tile_count;
        fine += tx * ty;
        if (f == 0) c->camera_fine_tiles = tx * ty;
        if (f + 1u == nv) cam_tiles = coarse;
        P.frusta[f] = d;
        P.fview[f] = v;
        P.flayer[f] = kInvalid;
        if (cam) {
            std::memcpy(P.clip[f], views[v].camera.clip_from_world, 64);
            P.out_base[f] = (uint32_t)out_pixels;
            out_pixels += (uint64_t)g.screen_width * g.screen_height;
        } else {
            const fiber_light& lt = views[v].lights[l];
            std::memcpy(P.clip[f], lt.clip_from_world, 64);
            std::memcpy(P.light_dir[light], lt.direction_to_light, 12);
            std::memcpy(P.light_color[light], lt.color, 16);
            P.flayer[f] = light;
            P.layer_frustum[light] = f;
            ++light;
        }
    }
    if (out_pixels >= 0xFFFFFFFFull) return FIBER_EINVAL;
    c->out_pixels = out_pixels;
    c->n_views = nv;
    for (uint32_t v = 0, l0 = 0; v < nv; ++v) {
        P.view_layer0[v] = l0;
        P.view_layers[v] = views[v].n_lights;
        l0 += views[v].n_lights;
        std::memcpy(P.view_cam_pos[v], views[v].camera.world_position, 12);
        const uint32_t i0 = nv > 1u ? views[v].instance_first : 0u;
        const uint32_t ni = nv > 1u ? views[v].instance_count : I;
        P.view_inst0[v] = i0;
        P.view_strand0[v] = ni && i0 < I ? c->views[i0].strand_base : c->total_strand_count;
        uint32_t ns = 0;
        for (uint32_t i = i0; i < i0 + ni; ++i) ns += c->views[i].strand_count;
        P.view_strands[v] = ns;
    }
    P.fine_tile_base[0] = 0u;
    for (uint32_t f = 0; f < n_frusta; ++f)
        P.fine_tile_base[f + 1] =
            P.fine_tile_base[f] + (P.view_strands[P.fview[f]] + kFineStrandsPerTile - 1u) / kFineStrandsPerTile;
    P.n_views = nv;
    std::memcpy(P.camera_pos, views[0].camera.world_position, 12);
    std::memcpy(P.ambient, st.ambient_color, 16);
    P.F = n_frusta;
    P.I = I;
    P.L = n_lights;
    P.K = st.dom_slices;
    P.total_coarse_tiles = coarse;
    P.total_strands = c->total_strand_count;
    P.max_strands = c->max_strand_count;
    P.camera_frustum_end = nv;
    P.camera_tile_end = cam_tiles;
    P.dom_size = dmax;
    P.shadow_map_size = n_lights ? (st.shadow_map_size ? st.shadow_map_size : P.dom_size) : 0u;
    P.dom_pool_pages = n_lights ? st.dom_page_pool : 0u;
    P.dom_pages_x = (P.dom_size + kDomPage - 1u) / kDomPage;
    // Shading atlas dims (create_shading_target_texture, src/pipelines/shading.rs:410-438).
    uint32_t aw = std::min(std::max(c->max_texels, 1u), 8192u);
    uint32_t ah = std::min(std::max((c->max_texels + aw - 1u) / aw, 1u), 8192u);
    P.atlas_cap = aw * ah;
    // Capacities (src/plugin.rs:483-576): prepass = next_pow2(strands) >= 2048,
    // binning = next_pow2(next_pow2(segments) >= prepass, x frusta), refs =
    // next_pow2(factor x binning). Pages and work items are sized so that only
    // the reference list can overflow. Several views: binning =
    // next_pow2(sum over views of segments x the view's frusta), as each view's
    // strands meet its own frusta only.
    auto next_pow2 = [](uint64_t x) {
        uint64_t p = 1;
        while (p < x) p <<= 1;
        return p;
    };
    const uint64_t table = (uint64_t)coarse * kDepthSlices;
    uint64_t task_cap = 0;
    if (nv == 1u) {
        const uint64_t prepass_cap = std::max<uint64_t>(next_pow2(c->total_strands), 2048);
        const uint64_t base_binning = std::max<uint64_t>(next_pow2(c->total_segments), prepass_cap);
        task_cap = std::max<uint64_t>(next_pow2(base_binning * P.F), base_binning);
    } else {
        uint64_t sum = 0;
        for (uint32_t v = 0; v < nv; ++v) {
            uint64_t segs = 0;
            for (uint32_t i = views[v].instance_first; i < views[v].instance_first + views[v].instance_count; ++i)
                segs += c->inst_segments[i];
            sum += segs * (1u + views[v].n_lights);
        }
        task_cap = std::max<uint64_t>(next_pow2(sum), 2048);
    }
    const uint64_t page_cap = std::max<uint64_t>(1, table / st.page_capacity_divisor);
    const uint64_t ref_cap = std::max<uint64_t>(
        std::max<uint64_t>(next_pow2(task_cap * st.ref_capacity_factor), std::max<uint64_t>(task_cap, 1024)),
        next_pow2(c->ref_floor));
    const uint64_t fine_tiles = table;  // coarse tiles x 16 fine tiles
    const uint64_t work_cap = std::max<uint64_t>(1, std::min<uint64_t>(ref_cap, 256ull * fine_tiles));
    if (task_cap >= 0xFFFFFFFFull || ref_cap >= 0xFFFFFFFFull || work_cap >= 0xFFFFFFFFull) return FIBER_ENOMEM;
    P.task_capacity = (uint32_t)task_cap;
    P.page_capacity = (uint32_t)page_cap;
    P.ref_capacity = (uint32_t)ref_cap;
    P.work_capacity = (uint32_t)work_cap;
    P.stochastic_cull_enabled = st.stochastic_cull_enabled;
    P.target_strands_per_pixel = st.target_strands_per_pixel;
    P.min_keep_probability = st.min_keep_probability;
    P.shadow_keep_probability = st.shadow_keep_probability;
    P.history_valid = st.history_enabled ? 1u : 0u;
    P.fragment_counts = st.fragment_counts_enabled;
    P.width = views[0].camera_cfg.screen_width;
    P.height = views[0].camera_cfg.screen_height;
    // Look-back status regions.
    uint64_t fine_tiles_lb = P.fine_tile_base[P.F];
    uint64_t lb_sizes[kStageCount] = {fine_tiles_lb + 1, table / 1024 + 2, page_cap + 1, table / 1024 + 2,
                                      fine_tiles + 1};
    uint64_t lb_total = 0;
    for (int i = 0; i < kStageCount; ++i) {
        c->lb_offset[i] = (uint32_t)lb_total;
        lb_total += lb_sizes[i];
    }
    const uint64_t L = n_lights, D = P.dom_size, S = P.shadow_map_size, K = P.K;
    const uint64_t FI = (uint64_t)I * P.F;
    fiber_status e = FIBER_OK;
#define ENSURE(buf, bytes, zero)                     \
    do {                                             \
        e = ensure(c, buf, (size_t)(bytes), zero);   \
        if (e != FIBER_OK) return e;                 \
    } while (0)
    bool lb_new = !c->d_lb.p || c->d_lb.bytes < lb_total * 8;
    ENSURE(c->d_params, sizeof(FrameParams), false);
    ENSURE(c->d_inst, std::max<uint64_t>(1, I) * sizeof(InstanceView), false);
    ENSURE(c->d_lb, lb_total * 8, true);
    if (lb_new) c->epoch = 0;
    ENSURE(c->d_range_valid, FI * 4, false);
    ENSURE(c->d_ranges, FI * sizeof(fiber_coarse_asset_range), false);
    ENSURE(c->d_keep, FI * 4, false);
    ENSURE(c->d_inst_visible, (uint64_t)I * 4, false);
    ENSURE(c->d_inst_keep, (uint64_t)I * 4, false);
    ENSURE(c->d_lut, table * sizeof(fiber_coarse_depth_lut_entry), false);
    ENSURE(c->d_lut_tree, ((uint64_t)coarse + 1u) * kLutTreeWords * 4u, false);
    ENSURE(c->d_tasks, task_cap * sizeof(fiber_binning_task), false);
    ENSURE(c->d_projected, task_cap * sizeof(fiber_projected_segment), false);
    ENSURE(c->d_page_table, table * 4, false);
    ENSURE(c->d_page_meta, page_cap * sizeof(fiber_fine_page_meta), false);
    ENSURE(c->d_counts, page_cap * kPageSize * 4, false);
    ENSURE(c->d_offsets, page_cap * kPageSize * 4, false);
    ENSURE(c->d_cursors, page_cap * kPageSize * 4, false);
    ENSURE(c->d_refs, ref_cap * sizeof(fiber_fine_seg_ref), false);
    ENSURE(c->d_ref_keys, ref_cap * 4, false);
    ENSURE(c->d_active_flags, fine_tiles * 4, false);
    ENSURE(c->d_active_list, fine_tiles * 4, false);
    ENSURE(c->d_work, work_cap * sizeof(fiber_raster_work_item), false);
    ENSURE(c->d_runs, fine_tiles * sizeof(fiber_raster_tile_run), false);
    ENSURE(c->d_big_cells, (ref_cap / 33 + 1) * sizeof(uint2), false);
    // Visit records (page-table slot << 8 | cell) hold up to ref_capacity visits;
    // slots must fit 24 bits, else count and fill walk the tasks.
    P.visit_records = table < (1ull << 24) ? 1u : 0u;
    const uint64_t visit_cap = P.visit_records ? ref_cap : 1u;
    ENSURE(c->d_visit_rec, visit_cap * 4, false);
    ENSURE(c->d_visit_task, visit_cap * 4, false);
    ENSURE(c->d_visit_rank, visit_cap * 4, false);
    ENSURE(c->d_task_key, task_cap * 8, false);
    ENSURE(c->d_task_mat, task_cap * 4, false);
    // Non-empty cells: at most one per kept reference and one per cell.
    ENSURE(c->d_cells_small, std::min<uint64_t>(ref_cap, page_cap * kPageSize) * sizeof(uint2), false);
    ENSURE(c->d_cells_mid, (ref_cap / 9 + 1) * sizeof(uint2), false);
    ENSURE(c->d_cells_large, (ref_cap / 33 + 1) * sizeof(uint2), false);
    ENSURE(c->d_opaque, (uint64_t)c->camera_fine_tiles * sizeof(uint2), false);
    ENSURE(c->d_task_proj, task_cap * 2 * sizeof(float4), false);
    ENSURE(c->d_ref_task, ref_cap * 4, false);
    if (st.telemetry_enabled) {
        ENSURE(c->d_tel, sizeof(fiber_telemetry), false);
        ENSURE(c->d_tel_slots, table * 4, false);
    }
    if (st.fine_binning_backend == 1u) {
        ENSURE(c->d_page_nvis, page_cap * 4, false);
        ENSURE(c->d_page_vbase, page_cap * 4, false);
        ENSURE(c->d_page_bucket, visit_cap * sizeof(uint2), false);
    }
    if (P.dom_pool_pages) {  // sparse residency: a page table per layer and the page pool
        const uint64_t ppx = P.dom_pages_x;
        ENSURE(c->d_dom_page_table, L * ppx * ppx * 4, false);
        ENSURE(c->d_dom_pool, (uint64_t)P.dom_pool_pages * kDomPageTexels * (K + 1) * 4, false);
    } else {
        ENSURE(c->d_dom_depth, L * D * D * 4, false);
        ENSURE(c->d_dom_opacity, L * K * D * D * 4, true);
    }
    ENSURE(c->d_shadow_map, L * S * S * 4, false);
    const uint64_t atlas_texels = (uint64_t)std::max(I, 1u) * P.atlas_cap;
    bool hist_new = !c->d_history[0].p || c->d_history[0].bytes < atlas_texels * 4;
    ENSURE(c->d_atlas, atlas_texels * 8, true);
    ENSURE(c->d_history[0], atlas_texels * 4, true);
    ENSURE(c->d_history[1], atlas_texels * 4, true);
    if (hist_new) {
        // History is cleared on reallocation (src/pipelines/shading.rs:509-525).
        cudaMemsetAsync(c->d_history[0].p, 0, c->d_history[0].bytes, s);
        cudaMemsetAsync(c->d_history[1].p, 0, c->d_history[1].bytes, s);
        c->hist_cur = 0;
    }
    ENSURE(c->d_color, out_pixels * 8, false);
    ENSURE(c->d_depth, out_pixels * 4, false);
    ENSURE(c->d_fragments, out_pixels * 4, false);
#undef ENSURE
    c->epoch = (c->epoch + 1u) & 0x3FFFFFFFu;
    if (c->epoch_dirty) c->epoch = 0u;  // a batch graph moved the device epoch on
    c->epoch_dirty = false;
    if (c->epoch == 0u) {  // epoch wrapped: old words could alias, clear them
        cudaMemsetAsync(c->d_lb.p, 0, c->d_lb.bytes, s);
        c->epoch = 1u;
    }
    P.epoch = c->epoch;
    P.hist_in = (uint32_t)c->hist_cur;
    // Per-frame uploads and resets (src/plugin.rs:1145-1208).
    FIBER_CUDA(cudaMemcpyAsync(c->d_params.p, &P, sizeof(P), cudaMemcpyHostToDevice, s));
    if (I) FIBER_CUDA(cudaMemcpyAsync(c->d_inst.p, c->views.data(), I * sizeof(InstanceView), cudaMemcpyHostToDevice, s));
    e = frame_resets(c, s);
    if (e != FIBER_OK) return e;
    c->last_stream = s;
    c->frame_ready = true;
    c->opaque_frame = false;
    return FIBER_OK;
}

fiber_status fiber_frame_begin(fiber_ctx* c, const fiber_froxel_config* cam_cfg, const fiber_camera* cam,
                               const fiber_froxel_config* light_cfgs, const fiber_light* lights, uint32_t n_lights,
                               void* stream) {
    if (!c || !cam_cfg || !cam || (n_lights && (!light_cfgs || !lights))) return FIBER_EINVAL;
    fiber_view v{};
    v.camera_cfg = *cam_cfg;
    v.camera = *cam;
    v.light_cfgs = light_cfgs;
    v.lights = lights;
    v.n_lights = n_lights;
    v.instance_first = 0u;
    v.instance_count = (uint32_t)c->views.size();
    const fiber_status st = frame_begin_views(c, &v, 1u, (cudaStream_t)stream);
    if (st == FIBER_OK) {
        // Kept for a batch that renders this context's view inside a
        // multi-view frame.
        c->last_view = v;
        c->last_light_cfgs.assign(light_cfgs, light_cfgs + n_lights);
        c->last_lights.assign(lights, lights + n_lights);
    }
    return st;
}

fiber_status fiber_frame_begin_views(fiber_ctx* c, const fiber_view* views, uint32_t n_views, void* stream) {
    return frame_begin_views(c, views, n_views, (cudaStream_t)stream);
}

fiber_status fiber_opaque_depth(fiber_ctx* c, const fiber_image* depth, uint32_t samples, void* stream) {
    if (!c) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    OpaqueSource o;
    fiber_status st = opaque_source(c, depth, samples, o);
    if (st != FIBER_OK) return st;
    cudaSetDevice(c->device);
    cudaStream_t s = (cudaStream_t)stream;
    c->last_stream = s;
    launch_opaque(launch_ctx(c, s), prepass_args(c), o.depth, o.pitch, o.samples, c->camera_fine_tiles);
    c->opaque_frame = true;
    return check_launch();
}

fiber_status fiber_prepass(fiber_ctx* c, void* stream) {
    if (!c) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    cudaSetDevice(c->device);
    c->last_stream = (cudaStream_t)stream;
    return run_prepass(c, (cudaStream_t)stream);
}

fiber_status fiber_shadows(fiber_ctx* c, void* stream) {
    if (!c) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    cudaSetDevice(c->device);
    c->last_stream = (cudaStream_t)stream;
    return run_shadows(c, (cudaStream_t)stream);
}

fiber_status fiber_shading(fiber_ctx* c, void* stream) {
    if (!c) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    cudaSetDevice(c->device);
    c->last_stream = (cudaStream_t)stream;
    return run_shading(c, (cudaStream_t)stream);
}

fiber_status fiber_raster(fiber_ctx* c, uint32_t view, void* stream) {
    if (!c || view != 0u) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    cudaSetDevice(c->device);
    c->last_stream = (cudaStream_t)stream;
    return run_raster(c, (cudaStream_t)stream);
}

fiber_status fiber_composite(fiber_ctx* c, uint32_t view, const fiber_image* scene_color,
                             const fiber_image* scene_depth, fiber_image* out, void* stream) {
    if (!c || view != 0u) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    cudaSetDevice(c->device);
    c->last_stream = (cudaStream_t)stream;
    fiber_status st = run_composite(c, scene_color, scene_depth, out, (cudaStream_t)stream);
    record(c, 13, (cudaStream_t)stream);
    return st;
}

fiber_status fiber_frame_fused(fiber_ctx* c, const fiber_image* scene_color, const fiber_image* scene_depth,
                               fiber_image* out, void* stream_) {
    if (!c) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    cudaSetDevice(c->device);
    cudaStream_t s = (cudaStream_t)stream_;
    c->last_stream = s;
    const bool composite = scene_color && out;
    OpaqueSource opaque{};
    if (scene_depth) {
        fiber_status st = opaque_source(c, scene_depth, 1u, opaque);
        if (st != FIBER_OK) return st;
    }
    const OpaqueSource* op = scene_depth ? &opaque : nullptr;
    if (!s) {  // the legacy stream cannot be captured: run the nodes directly
        fiber_status st = run_prepass(c, s, op);
        if (st == FIBER_OK) st = run_shadows(c, s);
        if (st == FIBER_OK) st = run_shading(c, s);
        if (st == FIBER_OK) st = run_raster(c, s);
        if (st == FIBER_OK && composite) st = run_composite(c, scene_color, scene_depth, out, s);
        record(c, 13, s);
        return st;
    }
    // Every kernel argument is stable across frames (per-frame values live in
    // the device FrameParams), so one captured graph serves every frame of the
    // same shape and buffers. The shape is whatever the host bakes into the
    // launches: grid sizes (instances, coarse tiles), the shadow's shared
    // memory (K) and whether it runs (lights), the composite's image
    // extents, pitches and formats, and whether the walks cull against opaque
    // tiles (their kernel variant).
    auto pitch_of = [](const fiber_image* im) -> uint64_t {
        return im ? ((uint64_t)im->pitch << 32) | (uint64_t)im->format : 0u;
    };
    uint64_t key[kGraphKeyWords] = {c->buffer_generation,
                                    (uint64_t)(composite ? 1 : 0) | (uint64_t)(op || c->opaque_frame ? 2 : 0),
                                    (uint64_t)(uintptr_t)(scene_color ? scene_color->ptr : nullptr),
                                    (uint64_t)(uintptr_t)(scene_depth ? scene_depth->ptr : nullptr),
                                    (uint64_t)(uintptr_t)(out ? out->ptr : nullptr),
                                    (uint64_t)(uintptr_t)s,
                                    composite ? pitch_of(scene_color) : 0u,
                                    composite ? pitch_of(out) : 0u,
                                    scene_depth ? pitch_of(scene_depth) : 0u,
                                    ((uint64_t)c->P.width << 32) | c->P.height ^ (c->out_pixels << 1),
                                    ((uint64_t)c->P.I << 32) | c->P.total_coarse_tiles,
                                    ((uint64_t)c->P.K << 32) | c->P.L};
    bool reuse = c->graph && std::memcmp(key, c->graph_key, sizeof(key)) == 0;
    if (!reuse) {
        if (c->graph) {
            cudaGraphExecDestroy(c->graph);
            c->graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        FIBER_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int hist_before = c->hist_cur;
        fiber_status st = run_prepass(c, s, op);
        if (st == FIBER_OK) st = run_shadows(c, s);
        if (st == FIBER_OK) st = run_shading(c, s);
        if (st == FIBER_OK) st = run_raster(c, s);
        if (st == FIBER_OK && composite) st = run_composite(c, scene_color, scene_depth, out, s);
        record(c, 13, s);
        cudaError_t ce = cudaStreamEndCapture(s, &g);
        if (st != FIBER_OK || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            c->hist_cur = hist_before;
            return st != FIBER_OK ? st : FIBER_ECUDA;
        }
        ce = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return FIBER_ECUDA;
        std::memcpy(c->graph_key, key, sizeof(key));
        c->hist_cur = hist_before;
    }
    FIBER_CUDA(cudaGraphLaunch(c->graph, s));
    c->hist_cur = 1 - c->hist_cur;
    return FIBER_OK;
}

fiber_status fiber_render_host(fiber_ctx* c, const void* scene_host, const float* depth_host, void* out_host,
                               void* stream_) {
    if (!c || !scene_host || !out_host) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    if (c->n_views != 1u) return FIBER_EINVAL;
    cudaSetDevice(c->device);
    cudaStream_t s = (cudaStream_t)stream_;
    const uint64_t W = c->P.width, H = c->P.height;
    fiber_status e = ensure(c, c->d_host_scene, W * H * 8, false);
    if (e == FIBER_OK && depth_host) e = ensure(c, c->d_host_depth, W * H * 4, false);
    if (e != FIBER_OK) return e;
    if (!c->copy_stream) {
        FIBER_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        FIBER_CUDA(cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming));
        FIBER_CUDA(cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming));
    }
    // The depth feeds the opaque-tile reduce at the start of the prepass, so
    // it is uploaded in stream order. The scene image is needed only by the
    // composite: it is uploaded on the copy stream while the frame's nodes
    // run, once the previous frame's download has left the buffer.
    if (depth_host) FIBER_CUDA(cudaMemcpyAsync(c->d_host_depth.p, depth_host, W * H * 4, cudaMemcpyHostToDevice, s));
    FIBER_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_out, 0));
    FIBER_CUDA(cudaMemcpyAsync(c->d_host_scene.p, scene_host, W * H * 8, cudaMemcpyHostToDevice, c->copy_stream));
    FIBER_CUDA(cudaEventRecord(c->ev_in, c->copy_stream));
    // The composite blends onto the loaded destination; compositing in place
    // over the scene image gives dst = scene colour (each pixel is read and
    // written by one thread).
    fiber_image scene{c->d_host_scene.p, (uint32_t)W, (uint32_t)H, (uint32_t)(W * 8), FIBER_FMT_RGBA16F};
    fiber_image depth{c->d_host_depth.p, (uint32_t)W, (uint32_t)H, (uint32_t)(W * 4), FIBER_FMT_R32F};
    fiber_status st = fiber_frame_fused(c, nullptr, depth_host ? &depth : nullptr, nullptr, stream_);
    if (st != FIBER_OK) return st;
    FIBER_CUDA(cudaStreamWaitEvent(s, c->ev_in, 0));
    st = run_composite(c, &scene, depth_host ? &depth : nullptr, &scene, s);
    if (st != FIBER_OK) return st;
    FIBER_CUDA(cudaMemcpyAsync(out_host, c->d_host_scene.p, W * H * 8, cudaMemcpyDeviceToHost, s));
    FIBER_CUDA(cudaEventRecord(c->ev_out, s));
    return FIBER_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Hooks for the request server (fiber_internal.h), C++ linkage.
// ---------------------------------------------------------------------------
struct fiber_scene_state {
    std::vector<fiber_strand_instance> rows;
    std::vector<InstanceView> views;
    std::vector<uint64_t> inst_segments;
    uint64_t total_segments = 0, total_points = 0, total_strands = 0;
    uint32_t max_texels = 0, total_strand_count = 0, max_strand_count = 0;
};

fiber_scene_state* fiber_ctx_save_scene(const fiber_ctx* c) {
    fiber_scene_state* s = new fiber_scene_state();
    s->rows = c->rows;
    s->views = c->views;
    s->inst_segments = c->inst_segments;
    s->total_segments = c->total_segments;
    s->total_points = c->total_points;
    s->total_strands = c->total_strands;
    s->max_texels = c->max_texels;
    s->total_strand_count = c->total_strand_count;
    s->max_strand_count = c->max_strand_count;
    return s;
}

fiber_status fiber_ctx_load_scene(fiber_ctx* c, const fiber_scene_state* s) {
    if (!c || !s) return FIBER_EINVAL;
    c->rows = s->rows;
    c->views = s->views;
    c->inst_segments = s->inst_segments;
    c->total_segments = s->total_segments;
    c->total_points = s->total_points;
    c->total_strands = s->total_strands;
    c->max_texels = s->max_texels;
    c->total_strand_count = s->total_strand_count;
    c->max_strand_count = s->max_strand_count;
    c->frame_ready = false;
    return FIBER_OK;
}

void fiber_scene_state_free(fiber_scene_state* s) { delete s; }

uint64_t fiber_scene_segments(const fiber_scene_state* s) { return s ? s->total_segments : 0u; }

uint64_t fiber_ctx_allocated(const fiber_ctx* c) { return c ? c->allocated : 0u; }

bool fiber_ctx_grow_refs(fiber_ctx* c, cudaStream_t s) {
    if (!c) return false;
    uint32_t overflow = 0u, refs = 0u;
    if (cudaMemcpyAsync(&overflow, reinterpret_cast<const char*>(c->d_counters.p) + offsetof(FrameCounters, overflow),
                        4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&refs, reinterpret_cast<const char*>(c->d_counters.p) + offsetof(FrameCounters, refs), 4,
                        cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (!(overflow & 4u) || refs <= c->P.ref_capacity) return false;
    c->ref_floor = std::max<uint64_t>(c->ref_floor, refs);
    return true;
}

fiber_status fiber_ctx_frame_status(fiber_ctx* c, cudaStream_t s) {
    if (!c) return FIBER_EINVAL;
    uint32_t w[2] = {0u, 0u};  // overflow, error (adjacent words of FrameCounters)
    static_assert(offsetof(FrameCounters, error) == offsetof(FrameCounters, overflow) + 4, "counter layout");
    FIBER_CUDA(cudaMemcpyAsync(w, reinterpret_cast<const char*>(c->d_counters.p) + offsetof(FrameCounters, overflow),
                               sizeof(w), cudaMemcpyDeviceToHost, s));
    FIBER_CUDA(cudaStreamSynchronize(s));
    if (w[1] != 0u) return FIBER_ETIMEDOUT;
    if (w[0] != 0u) return FIBER_EOVERFLOW;
    return FIBER_OK;
}

fiber_status fiber_ctx_enqueue_frame(fiber_ctx* c, cudaStream_t s) {
    if (!c) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    k_frame_advance<<<1, 256, 0, s>>>(dp<FrameParams>(c->d_params), dp<unsigned long long>(c->d_lb),
                                      (uint64_t)(c->d_lb.bytes / 8));
    fiber_status st = check_launch();
    if (st == FIBER_OK) st = frame_resets(c, s);
    const int hist_before = c->hist_cur;
    if (st == FIBER_OK) st = run_prepass(c, s);
    if (st == FIBER_OK) st = run_shadows(c, s);
    if (st == FIBER_OK) st = run_shading(c, s);
    if (st == FIBER_OK) st = run_raster(c, s);
    record(c, 13, s);
    c->hist_cur = hist_before;  // the device flips the history in k_frame_advance
    return st;
}

void fiber_ctx_shape_key(const fiber_ctx* c, uint64_t key[kFrameShapeWords]) {
    const FrameParams& P = c->P;
    key[0] = c->buffer_generation;
    key[1] = ((uint64_t)P.I << 32) | P.total_coarse_tiles;
    key[2] = ((uint64_t)P.K << 32) | P.L;
    key[3] = (((uint64_t)P.width << 32) | P.height) ^ (c->out_pixels << 1) ^ ((uint64_t)P.F << 56);
    key[4] = ((uint64_t)P.dom_size << 32) | P.shadow_map_size;
    key[5] = ((uint64_t)P.fragment_counts << 32) | (c->frame_ready ? 1u : 0u);
}

void fiber_ctx_mark_replayed(fiber_ctx* c, cudaStream_t s) {
    c->epoch_dirty = true;
    c->last_stream = s;  // readbacks wait for the batch launch
}

uint64_t fiber_ctx_frame_cost(const fiber_ctx* c) {
    return c->total_segments * (uint64_t)c->P.F + c->out_pixels +
           (uint64_t)c->P.L * c->P.dom_size * c->P.dom_size;
}

int fiber_ctx_device(const fiber_ctx* c) { return c->device; }

void fiber_ctx_set_side_stream(fiber_ctx* c, cudaStream_t side) {
    if (c) c->side_override = side;
}

fiber_status fiber_ctx_render_host_nodes(fiber_ctx* c, const void* scene_host, void* out_host, cudaStream_t s) {
    if (!c || !scene_host || !out_host) return FIBER_EINVAL;
    if (!c->frame_ready) return FIBER_ENOTREADY;
    if (c->n_views != 1u) return FIBER_EINVAL;
    const uint64_t W = c->P.width, H = c->P.height;
    fiber_status e = ensure(c, c->d_host_scene, W * H * 8, false);
    if (e != FIBER_OK) return e;
    c->last_stream = s;
    FIBER_CUDA(cudaMemcpyAsync(c->d_host_scene.p, scene_host, W * H * 8, cudaMemcpyHostToDevice, s));
    fiber_image scene{c->d_host_scene.p, (uint32_t)W, (uint32_t)H, (uint32_t)(W * 8), FIBER_FMT_RGBA16F};
    fiber_status st = run_prepass(c, s);
    if (st == FIBER_OK) st = run_shadows(c, s);
    if (st == FIBER_OK) st = run_shading(c, s);
    if (st == FIBER_OK) st = run_raster(c, s);
    if (st == FIBER_OK) st = run_composite(c, &scene, nullptr, &scene, s);
    record(c, 13, s);
    if (st != FIBER_OK) return st;
    FIBER_CUDA(cudaMemcpyAsync(out_host, c->d_host_scene.p, W * H * 8, cudaMemcpyDeviceToHost, s));
    return FIBER_OK;
}

extern "C" {

fiber_status fiber_debug_stall_lookback(fiber_ctx* c, uint32_t stage, uint32_t tile, uint32_t spin_limit) {
    if (!c || stage >= kStageCount) return FIBER_EINVAL;
    c->stall_stage = stage + 1u;
    c->stall_tile = tile;
    c->stall_limit = spin_limit;
    return FIBER_OK;
}

fiber_status fiber_stats_get(fiber_ctx* c, fiber_stats* out) {
    if (!c || !out) return FIBER_EINVAL;
    cudaSetDevice(c->device);
    FIBER_CUDA(cudaStreamSynchronize(c->last_stream));
    FrameCounters h{};
    FIBER_CUDA(cudaMemcpy(&h, c->d_counters.p, sizeof(h), cudaMemcpyDeviceToHost));
    c->h_counters = h;
    std::memset(out, 0, sizeof(*out));
    out->frustum_count = c->P.F;
    out->instance_count = c->P.I;
    out->binning_tasks = std::min(h.tasks, c->P.task_capacity);
    out->camera_tasks = h.frustum_task_base[c->P.camera_frustum_end];
    out->allocated_pages = h.pages;
    std::vector<fiber_fine_page_meta> pm(h.pages);
    if (h.pages) FIBER_CUDA(cudaMemcpy(pm.data(), c->d_page_meta.p, h.pages * sizeof(fiber_fine_page_meta), cudaMemcpyDeviceToHost));
    uint64_t refs = 0;
    for (const auto& m : pm) {
        refs += m.seg_ref_count;
        uint32_t f = 0;
        for (; f < c->P.F; ++f)
            if (m.coarse_tile_id >= c->P.frusta[f].coarse_depth_tile_base &&
                m.coarse_tile_id < c->P.frusta[f].coarse_depth_tile_base + c->P.frusta[f].coarse_depth_tile_count)
                break;
        if (f < FIBER_MAX_FRUSTA) {
            out->frustum_pages[f]++;
            out->frustum_refs[f] += m.seg_ref_count;
        }
    }
    out->fine_refs = (uint32_t)std::min<uint64_t>(refs, 0xFFFFFFFFull);
    out->fine_refs_total = refs;
    out->refs_requested = h.refs;
    out->active_tiles = h.active_tiles;
    out->camera_runs = h.camera_active;
    out->shadow_runs = h.active_tiles - h.camera_active;
    out->work_items = h.work_items;
    out->overflow_flags = h.overflow;
    out->timeout_flags = h.error;
    for (uint32_t f = 0; f < c->P.F && f < FIBER_MAX_FRUSTA; ++f)
        out->frustum_tasks[f] = h.frustum_task_base[f + 1] - h.frustum_task_base[f];
    std::vector<fiber_raster_tile_run> runs(h.active_tiles);
    if (h.active_tiles)
        FIBER_CUDA(cudaMemcpy(runs.data(), c->d_runs.p, h.active_tiles * sizeof(fiber_raster_tile_run), cudaMemcpyDeviceToHost));
    for (const auto& r : runs)
        if (r.frustum_id < FIBER_MAX_FRUSTA) {
            out->frustum_work[r.frustum_id] += r.work_count;
            out->frustum_runs[r.frustum_id]++;
        }
    out->total_segments = c->total_segments;
    out->total_points = c->total_points;
    out->total_strands = c->total_strands;
    if (h.error) return FIBER_ETIMEDOUT;
    if (h.overflow) return FIBER_EOVERFLOW;
    return FIBER_OK;
}

// The DOM as dense layers on the host: a copy, or the resident pages of the
// sparse pool expanded through the page tables (zeros elsewhere).
static fiber_status dom_dense(fiber_ctx* c, std::vector<float>& dep, std::vector<float>& op) {
    const FrameParams& P = c->P;
    const uint64_t L = P.L, D = P.dom_size, K = P.K;
    if (!P.dom_pool_pages) {
        FIBER_CUDA(cudaMemcpy(dep.data(), c->d_dom_depth.p, dep.size() * 4, cudaMemcpyDeviceToHost));
        FIBER_CUDA(cudaMemcpy(op.data(), c->d_dom_opacity.p, op.size() * 4, cudaMemcpyDeviceToHost));
        return FIBER_OK;
    }
    const uint64_t ppx = P.dom_pages_x, page_words = (uint64_t)kDomPageTexels * (K + 1);
    std::vector<uint32_t> table(L * ppx * ppx);
    FIBER_CUDA(cudaMemcpy(table.data(), c->d_dom_page_table.p, table.size() * 4, cudaMemcpyDeviceToHost));
    std::fill(dep.begin(), dep.end(), 0.0f);
    std::fill(op.begin(), op.end(), 0.0f);
    std::vector<float> page(page_words);
    for (uint64_t l = 0; l < L; ++l)
        for (uint64_t py = 0; py < ppx; ++py)
            for (uint64_t px = 0; px < ppx; ++px) {
                const uint32_t h = table[(l * ppx + py) * ppx + px];
                if (h == 0u || h == kMarked || h - 1u >= P.dom_pool_pages) continue;
                FIBER_CUDA(cudaMemcpy(page.data(), static_cast<const float*>(c->d_dom_pool.p) + (h - 1u) * page_words,
                                      page_words * 4, cudaMemcpyDeviceToHost));
                for (uint64_t y = 0; y < kDomPage && py * kDomPage + y < D; ++y)
                    for (uint64_t x = 0; x < kDomPage && px * kDomPage + x < D; ++x) {
                        const uint64_t t = (py * kDomPage + y) * D + px * kDomPage + x, o = y * kDomPage + x;
                        dep[l * D * D + t] = page[o];
                        for (uint64_t k = 0; k < K; ++k) op[(l * K + k) * D * D + t] = page[(1 + k) * kDomPageTexels + o];
                    }
            }
    return FIBER_OK;
}

fiber_status fiber_telemetry_get(fiber_ctx* c, fiber_telemetry* out) {
    if (!c || !out) return FIBER_EINVAL;
    if (!c->settings.telemetry_enabled || !c->d_tel.p) return FIBER_EINVAL;
    cudaSetDevice(c->device);
    FIBER_CUDA(cudaStreamSynchronize(c->last_stream));
    FIBER_CUDA(cudaMemcpy(out, c->d_tel.p, sizeof(fiber_telemetry), cudaMemcpyDeviceToHost));
    return FIBER_OK;
}

fiber_status fiber_dump(fiber_ctx* c, uint32_t what, void* host, uint64_t capacity, uint64_t* written) {
    if (!c) return FIBER_EINVAL;
    cudaSetDevice(c->device);
    FIBER_CUDA(cudaStreamSynchronize(c->last_stream));
    FrameCounters h{};
    FIBER_CUDA(cudaMemcpy(&h, c->d_counters.p, sizeof(h), cudaMemcpyDeviceToHost));
    const FrameParams& P = c->P;
    const uint64_t table = (uint64_t)P.total_coarse_tiles * kDepthSlices;
    const uint64_t L = P.L, D = P.dom_size, S = P.shadow_map_size, K = P.K;
    const void* src = nullptr;
    uint64_t bytes = 0;
    std::vector<uint32_t> tmp;
    switch (what) {
        case FIBER_DUMP_FRUSTA:
            if (written) *written = c->frusta.size() * sizeof(fiber_frustum_desc);
            if (host && capacity >= c->frusta.size() * sizeof(fiber_frustum_desc))
                std::memcpy(host, c->frusta.data(), c->frusta.size() * sizeof(fiber_frustum_desc));
            return FIBER_OK;
        case FIBER_DUMP_RANGES: {
            uint64_t n = (uint64_t)P.I * P.F;
            std::vector<uint32_t> valid(n);
            std::vector<fiber_coarse_asset_range> r(n);
            if (n) {
                FIBER_CUDA(cudaMemcpy(valid.data(), c->d_range_valid.p, n * 4, cudaMemcpyDeviceToHost));
                FIBER_CUDA(cudaMemcpy(r.data(), c->d_ranges.p, n * sizeof(fiber_coarse_asset_range), cudaMemcpyDeviceToHost));
            }
            for (uint64_t i = 0; i < n; ++i) {
                tmp.push_back(valid[i]);
                const uint32_t* w = reinterpret_cast<const uint32_t*>(&r[i]);
                if (valid[i]) tmp.insert(tmp.end(), w, w + 8);
                else tmp.insert(tmp.end(), 8, 0u);
            }
            if (written) *written = tmp.size() * 4;
            if (host && capacity >= tmp.size() * 4) std::memcpy(host, tmp.data(), tmp.size() * 4);
            return FIBER_OK;
        }
        case FIBER_DUMP_KEEP: src = c->d_keep.p; bytes = (uint64_t)P.I * P.F * 4; break;
        case FIBER_DUMP_LUT: src = c->d_lut.p; bytes = table * sizeof(fiber_coarse_depth_lut_entry); break;
        case FIBER_DUMP_TASKS: src = c->d_tasks.p; bytes = (uint64_t)std::min(h.tasks, P.task_capacity) * 16; break;
        case FIBER_DUMP_PROJECTED: src = c->d_projected.p; bytes = (uint64_t)std::min(h.tasks, P.task_capacity) * 12; break;
        case FIBER_DUMP_PAGE_TABLE: src = c->d_page_table.p; bytes = table * 4; break;
        case FIBER_DUMP_PAGE_META: src = c->d_page_meta.p; bytes = (uint64_t)h.pages * 32; break;
        case FIBER_DUMP_COUNTS: src = c->d_counts.p; bytes = (uint64_t)h.pages * kPageSize * 4; break;
        case FIBER_DUMP_OFFSETS: src = c->d_offsets.p; bytes = (uint64_t)h.pages * kPageSize * 4; break;
        case FIBER_DUMP_REFS: src = c->d_refs.p; bytes = (uint64_t)std::min(h.refs, P.ref_capacity) * 12; break;
        case FIBER_DUMP_ACTIVE_TILES: src = c->d_active_list.p; bytes = (uint64_t)h.active_tiles * 4; break;
        case FIBER_DUMP_WORK: src = c->d_work.p; bytes = (uint64_t)std::min(h.work_items, P.work_capacity) * 32; break;
        case FIBER_DUMP_RUNS: src = c->d_runs.p; bytes = (uint64_t)h.active_tiles * 32; break;
        case FIBER_DUMP_DOM_DEPTH:
        case FIBER_DUMP_DOM_OPACITY: {
            // Dense layers in canonical form: opacity of texels without a depth
            // (never written this frame) reads as 0; under sparse residency
            // the texels of pages that are not resident read as 0.
            std::vector<float> dep(L * D * D), op(L * K * D * D);
            if (!dep.empty()) {
                fiber_status e = dom_dense(c, dep, op);
                if (e != FIBER_OK) return e;
                for (uint64_t l = 0; l < L; ++l)
                    for (uint64_t k = 0; k < K; ++k)
                        for (uint64_t p = 0; p < D * D; ++p)
                            if (dep[l * D * D + p] == 0.0f) op[(l * K + k) * D * D + p] = 0.0f;
            }
            const std::vector<float>& v = what == FIBER_DUMP_DOM_DEPTH ? dep : op;
            if (written) *written = v.size() * 4;
            if (host && capacity >= v.size() * 4) std::memcpy(host, v.data(), v.size() * 4);
            return host && capacity < v.size() * 4 ? FIBER_EINVAL : FIBER_OK;
        }
        case FIBER_DUMP_SHADOW_MAP: src = c->d_shadow_map.p; bytes = L * S * S * 4; break;
        case FIBER_DUMP_ATLAS: src = c->d_atlas.p; bytes = (uint64_t)P.I * P.atlas_cap * 8; break;
        case FIBER_DUMP_HISTORY: src = c->d_history[c->hist_cur].p; bytes = (uint64_t)P.I * P.atlas_cap * 4; break;
        case FIBER_DUMP_COLOR: src = c->d_color.p; bytes = c->out_pixels * 8; break;
        case FIBER_DUMP_DEPTH: src = c->d_depth.p; bytes = c->out_pixels * 4; break;
        case FIBER_DUMP_FRAGMENTS: src = c->d_fragments.p; bytes = c->out_pixels * 4; break;
        case FIBER_DUMP_OPAQUE_TILES:
            // The reference clears the tiles when no opaque depth is bound.
            bytes = (uint64_t)c->camera_fine_tiles * sizeof(uint2);
            if (!h.opaque_bound) {
                if (written) *written = bytes;
                if (host && capacity >= bytes) std::memset(host, 0, bytes);
                return host && capacity < bytes ? FIBER_EINVAL : FIBER_OK;
            }
            src = c->d_opaque.p;
            break;
        default: return FIBER_EINVAL;
    }
    if (written) *written = bytes;
    if (host && bytes) {
        if (capacity < bytes) return FIBER_EINVAL;
        FIBER_CUDA(cudaMemcpy(host, src, bytes, cudaMemcpyDeviceToHost));
    }
    return FIBER_OK;
}

fiber_status fiber_output_image(fiber_ctx* c, uint32_t what, fiber_image* out) {
    if (!c || !out) return FIBER_EINVAL;
    const FrameParams& P = c->P;
    switch (what) {
        case FIBER_DUMP_COLOR: *out = fiber_image{c->d_color.p, P.width, P.height, P.width * 8u, FIBER_FMT_RGBA16F}; break;
        case FIBER_DUMP_DEPTH: *out = fiber_image{c->d_depth.p, P.width, P.height, P.width * 4u, FIBER_FMT_R32F}; break;
        case FIBER_DUMP_DOM_DEPTH:
            if (P.dom_pool_pages) return FIBER_EINVAL;  // sparse residency: no dense image (fiber_dump expands it)
            *out = fiber_image{c->d_dom_depth.p, P.dom_size, P.dom_size * P.L, P.dom_size * 4u, FIBER_FMT_R32F};
            break;
        case FIBER_DUMP_DOM_OPACITY:
            if (P.dom_pool_pages) return FIBER_EINVAL;
            *out = fiber_image{c->d_dom_opacity.p, P.dom_size, P.dom_size * P.L * P.K, P.dom_size * 4u, FIBER_FMT_R32F};
            break;
        case FIBER_DUMP_SHADOW_MAP:
            *out = fiber_image{c->d_shadow_map.p, P.shadow_map_size, P.shadow_map_size * P.L, P.shadow_map_size * 4u, FIBER_FMT_R32F};
            break;
        default: return FIBER_EINVAL;
    }
    return FIBER_OK;
}

uint32_t fiber_span_count(void) { return kSpanCount; }
const char* fiber_span_name(uint32_t i) { return i < (uint32_t)kSpanCount ? kSpanNames[i] : ""; }

fiber_status fiber_span_times(fiber_ctx* c, float* ms, uint32_t n) {
    if (!c || !ms) return FIBER_EINVAL;
    if (!c->events_ok) return FIBER_ENOTREADY;
    cudaSetDevice(c->device);
    FIBER_CUDA(cudaStreamSynchronize(c->last_stream));
    for (uint32_t i = 0; i < n && i < (uint32_t)kSpanCount; ++i) {
        float t = 0.0f;
        if (i + 1 < (uint32_t)kSpanCount) {
            if (cudaEventElapsedTime(&t, c->ev[i], c->ev[i + 1]) != cudaSuccess) { cudaGetLastError(); t = -1.0f; }
        } else {
            if (cudaEventElapsedTime(&t, c->ev[0], c->ev[13]) != cudaSuccess) { cudaGetLastError(); t = -1.0f; }
        }
        ms[i] = t;
    }
    return FIBER_OK;
}

}  // extern "C"
