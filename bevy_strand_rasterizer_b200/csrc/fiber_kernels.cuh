// fiber_kernels.cuh — kernel argument blocks and launch entry points.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "fiber_device.cuh"

namespace fiber {

inline unsigned ceil_div_host(uint64_t x, uint64_t y) { return (unsigned)((x + y - 1) / y); }

// Segment fetch (get_segment_vertices_from_index_unchecked,
// strand_rasterizer.wgsl:289-303): 128-bit vertex loads through the read-only
// path, world transform in the reference's evaluation order.
__device__ __forceinline__ void segment_world(const InstanceView& in, uint32_t seg, float4& w0, float4& w1) {
    uint32_t i0 = __ldg(in.indices + seg), i1 = __ldg(in.indices + seg + 1u);
    float4 a = __ldg(in.vertices + i0), b = __ldg(in.vertices + i1);
    w0 = matvec(in.world_from_local, a.x, a.y, a.z, 1.0f);
    w1 = matvec(in.world_from_local, b.x, b.y, b.z, 1.0f);
}

// fragment_position_line_relative (strand_rasterizer.wgsl:138-147)
__device__ __forceinline__ float line_t(float px, float py, float ax, float ay, float bx, float by) {
    float abx = bx - ax, aby = by - ay;
    float l2 = abx * abx + aby * aby;
    if (l2 == 0.0f) return 0.0f;
    return ((px - ax) * abx + (py - ay) * aby) / l2;
}

// blend_over_premult (strand_rasterizer.wgsl:156-162)
__device__ __forceinline__ float4 over(float4 fg, float4 bg) {
    float oma = 1.0f - fg.w;
    return make_float4(fg.x + bg.x * oma, fg.y + bg.y * oma, fg.z + bg.z * oma, fg.w + bg.w * oma);
}

__device__ __forceinline__ float4 load_half4(const __half* p) {
    uint2 v = *reinterpret_cast<const uint2*>(p);
    __half2 a = *reinterpret_cast<__half2*>(&v.x), b = *reinterpret_cast<__half2*>(&v.y);
    float2 fa = __half22float2(a), fb = __half22float2(b);
    return make_float4(fa.x, fa.y, fb.x, fb.y);
}

__device__ __forceinline__ uint2 pack_half4(float x, float y, float z, float w) {
    __half2 lo = __halves2half2(__float2half_rn(x), __float2half_rn(y));
    __half2 hi = __halves2half2(__float2half_rn(z), __float2half_rn(w));
    return make_uint2(*reinterpret_cast<uint32_t*>(&lo), *reinterpret_cast<uint32_t*>(&hi));
}

// Device buffers of the work-preparation stages.
struct PrepassArgs {
    uint32_t* tile_counter;          // virtual block ids of the current look-back stage
    unsigned long long* lb_status;   // look-back status words of the current stage
    FrameCounters* counters;
    uint32_t* range_valid;           // [I * F]
    fiber_coarse_asset_range* ranges;
    float* keep;                     // [I * F]
    uint32_t* inst_visible;          // [I]
    float* inst_keep;                // [I] max(camera, shadow) keep probability
    fiber_coarse_depth_lut_entry* lut;
    // [coarse tiles][kLutTreeWords]: the slice lookup's search tree of a LUT
    // whose 16 entries are populated, ordered and disjoint (word 0 = kInvalid
    // otherwise): the starts of entries 0, 4, 8, 12, then per quarter the
    // starts and the ends of its four entries.
    uint32_t* lut_tree;
    fiber_binning_task* tasks;
    fiber_projected_segment* projected;
    uint32_t* page_table;
    fiber_fine_page_meta* page_meta;
    uint32_t* counts;
    uint32_t* offsets;
    uint32_t* cursors;
    fiber_fine_seg_ref* refs;
    uint32_t* ref_keys;
    uint32_t* active_flags;
    uint32_t* active_list;
    fiber_raster_work_item* work;
    fiber_raster_tile_run* runs;
    uint2* big_cells;
    uint32_t* visit_rec;    // [ref_capacity] page-table slot << 8 | cell; the count pass rewrites it to the cell index
    uint32_t* visit_task;   // [ref_capacity] binning task of the visit
    uint32_t* visit_rank;   // [ref_capacity] rank of the visit inside its cell
    unsigned long long* task_key;  // [task_capacity] canonical cell-order key of the task's reference
    uint32_t* task_mat;            // [task_capacity] material index of the task's reference
    uint2* cells_small;            // (ref base, count) of cells with 1..8 references
    uint2* cells_mid;              // (ref base, count) of cells with 9..32 references
    uint2* cells_large;            // (ref base, count) of cells with more than 8
    uint2* opaque_tiles;           // [camera fine tiles] (fully covered, quantised farthest opaque depth)
    float4* task_proj;             // [task_capacity][2] both end points as world_to_screen_raw gave them
    uint32_t* ref_task;            // [ref_capacity] binning task of each reference (after the cell sort)
    // Page-CSR backend only (null otherwise).
    uint32_t* page_nvis;           // [page_capacity] visits per page
    uint32_t* page_vbase;          // [page_capacity] first bucket entry of each page
    uint2* page_bucket;            // [ref_capacity] (task, cell) of each visit, grouped by page
    // Prepass telemetry only (null otherwise): a fiber_telemetry image and the
    // candidate tasks of every page-table slot.
    uint32_t* tel;
    uint32_t* tel_slots;
};

// Word offsets inside the telemetry image (the fiber_telemetry layout).
constexpr uint32_t kTelHistogram = 8, kTelFrustum = 40, kTelFrustumStride = 11;
enum TelFrustumField : uint32_t {
    kTelVisibleInstances = 0, kTelVisibleStrands, kTelRetainedStrands, kTelEmittedSegments, kTelAllocatedPages,
    kTelPageCandidates, kTelFineRefs, kTelRasterRuns, kTelRasterLoad, kTelMaxPageCandidates, kTelMaxRasterLoad
};
__device__ __forceinline__ uint32_t* tel_frustum(uint32_t* tel, uint32_t f, uint32_t field) {
    return tel + kTelFrustum + f * kTelFrustumStride + field;
}

// Device buffers of the shadow, shading, raster and composite stages.
struct RenderArgs {
    FrameCounters* counters;
    const fiber_binning_task* tasks;
    const fiber_fine_seg_ref* refs;
    const fiber_raster_work_item* work;
    const fiber_raster_tile_run* runs;
    const uint32_t* ref_task;    // [refs] binning task of each reference
    const float4* task_proj;     // [tasks][2] the task's end points as k_fine projected them
    float* dom_depth;        // [L][D][D] (dense layers)
    float* dom_opacity;      // [L][K][D][D] (dense layers)
    uint32_t* dom_page_table;  // [L][pages_x][pages_x] pool page + 1 (sparse residency)
    float* dom_pool;           // [pool][K + 1][256][256]: depth plane, then the K opacity planes
    float* shadow_map;       // [L][S][S] stampback target
    __half* atlas;           // [I][cap][4]
    __half* history[2];      // [I][cap][2] ping-pong; FrameParams::hist_in is read
    __half* color;           // [H][W][4]
    float* depth;            // [H][W]
    uint32_t* fragments;     // [H][W]
};

// Sparse DOM pages: DOM_PAGE_XY (src/plugin.rs:68) texels a side.
constexpr uint32_t kDomPage = 256;
constexpr uint32_t kDomPageTexels = kDomPage * kDomPage;

// The deep-opacity texel (layer, x, y): its depth word and its slice-0
// opacity word, with the stride between opacity slices. Dense layers, or the
// resident pool page through the page table (false when the page is not
// resident: nothing was rasterised there this frame).
__device__ __forceinline__ bool dom_texel(const FrameParams& P, const RenderArgs& R, uint32_t layer, uint32_t x,
                                          uint32_t y, float*& depth, float*& opacity, size_t& stride) {
    const uint32_t D = P.dom_size;
    if (P.dom_pool_pages == 0u) {
        const size_t px = (size_t)y * D + x;
        depth = R.dom_depth + (size_t)layer * D * D + px;
        opacity = R.dom_opacity + (size_t)layer * P.K * D * D + px;
        stride = (size_t)D * D;
        return true;
    }
    const uint32_t px_ = P.dom_pages_x;
    const uint32_t h = R.dom_page_table[((size_t)layer * px_ + y / kDomPage) * px_ + x / kDomPage];
    if (h == 0u || h == kMarked || h - 1u >= P.dom_pool_pages) return false;
    float* page = R.dom_pool + (size_t)(h - 1u) * kDomPageTexels * (P.K + 1u);
    const uint32_t off = (y % kDomPage) * kDomPage + x % kDomPage;
    depth = page + off;
    opacity = page + kDomPageTexels + off;
    stride = kDomPageTexels;
    return true;
}

struct CompositeArgs {
    const __half* strand_color;
    const float* strand_depth;
    const void* scene_color;
    uint32_t scene_pitch, scene_format;
    const float* scene_depth;
    uint32_t depth_pitch;
    void* out;
    uint32_t out_pitch, out_format;
    uint32_t width, height;
};

struct LaunchCtx {
    cudaStream_t stream;
    const FrameParams* P;         // device copy
    const InstanceView* inst;     // device copy
    uint32_t I, total_coarse_tiles;
    int sm_count;
    bool opaque;                  // K0 wrote this frame's opaque fine tiles
    bool telemetry;               // the prepass gathers telemetry
};

void launch_opaque(const LaunchCtx& L, const PrepassArgs& A, const float* depth, uint32_t pitch, uint32_t samples,
                   uint32_t tiles);
void launch_broad(const LaunchCtx& L, const PrepassArgs& A);
void launch_lut(const LaunchCtx& L, const PrepassArgs& A);
void launch_fine(const LaunchCtx& L, const PrepassArgs& A);
void launch_visit(const LaunchCtx& L, const PrepassArgs& A);
void launch_alloc(const LaunchCtx& L, const PrepassArgs& A);
void launch_zero_pages(const LaunchCtx& L, const PrepassArgs& A);
void launch_count(const LaunchCtx& L, const PrepassArgs& A);
void launch_prefix(const LaunchCtx& L, const PrepassArgs& A, bool csr = false);
void launch_page_csr_count(const LaunchCtx& L, const PrepassArgs& A);
void launch_build_pages(const LaunchCtx& L, const PrepassArgs& A);
void launch_fill_walk(const LaunchCtx& L, const PrepassArgs& A);
void launch_fill(const LaunchCtx& L, const PrepassArgs& A);
void launch_compact_active(const LaunchCtx& L, const PrepassArgs& A);
void launch_emit(const LaunchCtx& L, const PrepassArgs& A);
void launch_sort_cells(const LaunchCtx& L, const PrepassArgs& A);
void launch_sort_big(const LaunchCtx& L, const PrepassArgs& A);
void launch_telemetry(const LaunchCtx& L, const PrepassArgs& A);

void launch_shadow(const LaunchCtx& L, const RenderArgs& R, uint32_t K);
void launch_dom_paging(const LaunchCtx& L, const RenderArgs& R, uint32_t table_entries);
void launch_shade(const LaunchCtx& L, const RenderArgs& R);
void launch_raster(const LaunchCtx& L, const RenderArgs& R);
void launch_composite(cudaStream_t s, const CompositeArgs& C);

}  // namespace fiber
