// fiber_device.cuh — device-side building blocks of the strand raster path.
//
// Arithmetic follows the WGSL semantics of the reference shaders
// (src/shaders/common.wgsl, strand_prepass.wgsl, strand_rasterizer.wgsl):
// the library is compiled with --fmad=false and IEEE div/sqrt, so every
// + - * / sqrt here is one correctly rounded binary32 operation in source
// order and matrix-vector products are c0*x + c1*y + c2*z + c3*w left to
// right. Float-to-integer conversions saturate like WGSL's.
#pragma once

#include <cuda/atomic>
#include <stdint.h>

#include "../../include/fiber.h"

namespace fiber {

constexpr uint32_t kCoarseExtent = 4;      // COARSE_FINE_TILE_EXTENT (src/plugin.rs:58)
constexpr uint32_t kDepthSlices = 16;      // COARSE_DEPTH_SLICES (src/plugin.rs:59)
constexpr uint32_t kLutTreeWords = 36;  // 4 quarter starts + 4 x (4 starts, 4 ends)
constexpr uint32_t kPageSize = 256;        // COARSE_COUNT_PAGE_SIZE (src/plugin.rs:61)
constexpr uint32_t kDepthQuantMax = 16777215u;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kMarked = 0xFFFFFFFEu;  // MARKED_COUNT_PAGE (strand_prepass.wgsl:69)
constexpr uint32_t kMaxFrusta = 128;  // frusta of a frame (a multi-view frame: every view's camera and lights)
constexpr uint32_t kMaxViews = 64;    // views of a multi-view frame
constexpr uint32_t kPixelSlots = 64;       // strand_rasterizer.wgsl:309,839
// Strands per look-back tile of the fine prepass (k_fine).
constexpr uint32_t kFineStrandsPerTile = 64;

// Error words written by device code (never trap).
constexpr uint32_t kErrTimeout = 1u;

// ---------------------------------------------------------------------------
// Per-instance view resolved on the host once per frame from the slab tables.
// ---------------------------------------------------------------------------
struct InstanceView {
    const float4* vertices;
    const uint32_t* indices;
    const fiber_strand_meta* meta;
    const fiber_strand_material* materials;
    uint32_t n_vertices, n_indices, n_meta, n_materials;
    uint32_t strand_count;       // min(meta count, geo.strand_count)
    uint32_t strand_base;        // prefix of strand_count over instances
    uint32_t valid;              // all slab pointers resolved
    uint32_t view;               // view of a multi-view frame the instance belongs to (0 otherwise)
    fiber_aabb aabb;
    float world_from_local[16];
};

// Constant frame description shared by every kernel of a frame.
struct FrameParams {
    fiber_frustum_desc frusta[kMaxFrusta];
    float clip[kMaxFrusta][16];
    float light_dir[kMaxFrusta][4];
    float light_color[kMaxFrusta][4];
    float camera_pos[4];
    float ambient[4];
    uint32_t F, I, L, K;
    uint32_t total_coarse_tiles;
    uint32_t total_strands;       // sum of instance strand counts
    uint32_t max_strands;         // max strand count of one instance
    uint32_t camera_frustum_end;  // frusta [0, end) are cameras
    uint32_t camera_tile_end;     // coarse tiles of camera frusta
    uint32_t dom_size;            // D
    uint32_t shadow_map_size;     // S
    uint32_t atlas_cap;           // texels per instance layer
    uint32_t task_capacity, page_capacity, ref_capacity, work_capacity;
    uint32_t stochastic_cull_enabled;
    float target_strands_per_pixel, min_keep_probability, shadow_keep_probability;
    uint32_t history_valid;       // previous history holds a frame
    uint32_t fragment_counts;     // count fragments per pixel
    uint32_t width, height;       // camera resolution
    uint32_t epoch;               // look-back status epoch of this frame
    uint32_t hist_in;             // shadow-history buffer read this frame (0/1)
    uint32_t visit_records;       // page-table slots fit 24 bits: count/fill stream visit records
    uint32_t dom_pool_pages;      // 0: dense DOM layers; else the sparse DOM's pool size in pages
    uint32_t dom_pages_x;         // DOM pages per side (ceil(D / 256))
    uint32_t lb_spin_limit;       // polls before a look-back wait gives up
    uint32_t lb_stall_stage;      // 1 + look-back stage with a tile that never publishes (0: none)
    uint32_t lb_stall_tile;       // that tile (fiber_debug_stall_lookback; one frame only)
    // Views (a frame of fiber_frame_begin is one view). Frusta: every view's
    // camera first (frustum v is view v's camera), then the lights view by view.
    uint32_t n_views;
    uint32_t fview[kMaxFrusta];          // view of each frustum
    uint32_t flayer[kMaxFrusta];         // DOM layer of a light frustum, kInvalid otherwise
    uint32_t layer_frustum[kMaxFrusta];  // frustum of each DOM layer
    uint32_t out_base[kMaxFrusta];       // first pixel of a camera's colour / depth / fragment image
    uint32_t fine_tile_base[kMaxFrusta + 1];  // k_fine's tiles of each frustum (prefix)
    uint32_t view_strand0[kMaxViews], view_strands[kMaxViews];  // a view's strands (global strand indices)
    uint32_t view_layer0[kMaxViews], view_layers[kMaxViews];    // a view's lights (DOM layers, light indices)
    float view_cam_pos[kMaxViews][4];    // a view's camera position
    uint32_t view_inst0[kMaxViews];      // a view's first instance (the keep hash takes view-local ids)
};

// Device counters of one frame (zeroed at frame start).
struct FrameCounters {
    uint32_t tasks;               // binning tasks written
    uint32_t frustum_task_base[kMaxFrusta + 1];
    uint32_t pages;               // allocated pages (<= capacity)
    uint32_t refs;                // seg_ref tail (may exceed capacity)
    uint32_t active_tiles;
    uint32_t camera_active;       // active tiles that belong to camera frusta
    uint32_t work_items;
    uint32_t runs;
    uint32_t overflow;            // bit0 tasks, bit1 pages, bit2 refs, bit3 work, bit4 DOM pool
    uint32_t error;               // kErrTimeout when a bounded wait gave up
    uint32_t big_cells;           // cells queued for the large-cell sort
    uint32_t tile_counter[8];     // virtual block ids of the look-back stages
    uint32_t visit_overflow;      // visit records unused this frame (did not fit, or disabled)
    unsigned long long visits;    // visit records appended by k_visit
    uint32_t small_cells;         // cells of 1..8 references listed for the cell sort
    uint32_t large_cells;         // cells of more than 32 references listed for the cell sort
    uint32_t opaque_bound;        // the opaque fine-tile depths of this frame are written
    uint32_t dom_pages;           // DOM pages requested this frame (sparse residency)
    uint32_t mid_cells;           // cells of 9..32 references listed for the cell sort
    uint32_t pad_counters;
};
static_assert(sizeof(FrameCounters) == 176 + 4 * (kMaxFrusta - 16), "FrameCounters layout");

// Look-back stages (index into FrameCounters::tile_counter and the status regions).
enum LookbackStage : uint32_t { kStageFine = 0, kStageAlloc = 1, kStagePrefix = 2, kStageActive = 3, kStageEmit = 4, kStageCount = 5 };
// Run counters of the rasters (blocks claim tile runs dynamically).
constexpr uint32_t kShadowRunCounter = 5, kCameraRunCounter = 6;

// ---------------------------------------------------------------------------
// WGSL builtin semantics
// ---------------------------------------------------------------------------
__device__ __forceinline__ float wmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float wmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float wclamp(float e, float lo, float hi) { return fminf(fmaxf(e, lo), hi); }
__device__ __forceinline__ int32_t iclamp(int32_t e, int32_t lo, int32_t hi) { return min(max(e, lo), hi); }
__device__ __forceinline__ float wmix(float a, float b, float t) { return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t)); }
__device__ __forceinline__ uint32_t f2u(float f) { return __float2uint_rz(f); }   // saturating, NaN -> 0
__device__ __forceinline__ int32_t f2i(float f) { return __float2int_rz(f); }     // saturating, NaN -> 0
__device__ __forceinline__ float u2f(uint32_t u) { return __uint2float_rn(u); }
__device__ __forceinline__ uint32_t ceil_div(uint32_t x, uint32_t y) { return (x + y - 1u) / y; }

struct F3 { float x, y, z; };
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }

// The projection helpers below spell every operation as a correctly rounded
// intrinsic, so they give the same binary32 results in a translation unit
// compiled with contraction and approximate division (the shading's).
__device__ __forceinline__ float row4(float a, float x, float b, float y, float c, float z, float d, float w) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a, x), __fmul_rn(b, y)), __fmul_rn(c, z)), __fmul_rn(d, w));
}
__device__ __forceinline__ float4 matvec(const float* m, float x, float y, float z, float w) {
    float4 r;
    r.x = row4(m[0], x, m[4], y, m[8], z, m[12], w);
    r.y = row4(m[1], x, m[5], y, m[9], z, m[13], w);
    r.z = row4(m[2], x, m[6], y, m[10], z, m[14], w);
    r.w = row4(m[3], x, m[7], y, m[11], z, m[15], w);
    return r;
}

// common.wgsl:206-212
__device__ __forceinline__ float normalize_depth01(float z) {
    if (z >= 0.0f && z <= 1.0f) return z;
    return wclamp(__fadd_rn(__fmul_rn(z, 0.5f), 0.5f), 0.0f, 1.0f);
}
// common.wgsl:93-107 -> (sx, sy, ndc z, clip w)
__device__ __forceinline__ float4 world_to_screen_raw(float4 p, const float* clip, float vw, float vh) {
    float4 c = matvec(clip, p.x, p.y, p.z, p.w);
    if (c.w <= 0.0f) return make_float4(-1.0f, -1.0f, -1.0f, -1.0f);
    float nx = __fdiv_rn(c.x, c.w), ny = __fdiv_rn(c.y, c.w), nz = __fdiv_rn(c.z, c.w);
    float sx = __fadd_rn(0.0f, __fmul_rn(__fadd_rn(__fmul_rn(nx, 0.5f), 0.5f), vw));
    float sy = __fadd_rn(0.0f, __fmul_rn(__fadd_rn(__fmul_rn(ny, -0.5f), 0.5f), vh));
    return make_float4(sx, sy, nz, c.w);
}
// common.wgsl:229-242
__device__ __forceinline__ uint32_t wang_hash(uint32_t x) {
    x = (x ^ 61u) ^ (x >> 16u);
    x = x + (x << 3u);
    x = x ^ (x >> 4u);
    x = x * 0x27d4eb2du;
    x = x ^ (x >> 15u);
    return x;
}
__device__ __forceinline__ float hash_to_unit_float(uint32_t x) { return u2f(x) / 4294967296.0f; }
// strand_prepass.wgsl:533-539 (WGSL round = half to even)
__device__ __forceinline__ uint32_t quantize_depth01(float z) {
    return f2u(rintf(wclamp(z, 0.0f, 1.0f) * (float)kDepthQuantMax));
}
__device__ __forceinline__ float dequantize_depth01(uint32_t q) { return u2f(q) / (float)kDepthQuantMax; }
// WGSL pack2x16unorm: floor(0.5 + 65535 * clamp(e, 0, 1)), x in the low half.
__device__ __forceinline__ uint32_t unorm16(float e) {
    float t = 65535.0f * fminf(1.0f, fmaxf(0.0f, e));
    return f2u(floorf(0.5f + t));
}
__device__ __forceinline__ uint32_t pack2x16unorm(float a, float b) { return unorm16(a) | (unorm16(b) << 16u); }
__device__ __forceinline__ float2 unpack2x16unorm(uint32_t p) {
    return make_float2(u2f(p & 0xFFFFu) / 65535.0f, u2f(p >> 16u) / 65535.0f);
}
__device__ __forceinline__ int32_t sgn_i32(float f) {
    if (f > 1e-6f) return 1;
    if (f < -1e-6f) return -1;
    return 0;
}

// clip_axis_to_range / clip_segment_to_box (strand_prepass.wgsl:1356-1410)
__device__ __forceinline__ bool clip_axis(float p, float d, float mn, float mx, float& tmin, float& tmax) {
    if (fabsf(d) < 1e-6f) return !(p < mn || p > mx);
    float inv_d = 1.0f / d;
    float a = (mn - p) * inv_d;
    float b = (mx - p) * inv_d;
    if (a > b) { float t = a; a = b; b = t; }
    tmin = wmax(tmin, a);
    tmax = wmin(tmax, b);
    return !(tmin > tmax);
}
__device__ __forceinline__ bool clip_segment(F3 p0, F3 p1, F3 bmin, F3 bmax, F3& o0, F3& o1) {
    F3 d = f3(p1.x - p0.x, p1.y - p0.y, p1.z - p0.z);
    float tmin = 0.0f, tmax = 1.0f;
    if (!clip_axis(p0.x, d.x, bmin.x, bmax.x, tmin, tmax)) return false;
    if (!clip_axis(p0.y, d.y, bmin.y, bmax.y, tmin, tmax)) return false;
    if (!clip_axis(p0.z, d.z, bmin.z, bmax.z, tmin, tmax)) return false;
    o0 = f3(p0.x + d.x * tmin, p0.y + d.y * tmin, p0.z + d.z * tmin);
    o1 = f3(p0.x + d.x * tmax, p0.y + d.y * tmax, p0.z + d.z * tmax);
    return true;
}

// clip_segment with the direction's reciprocals computed once: the clips of
// one segment against several boxes share p1 - p0 and so share them. Same
// operations as clip_axis, so the same results bit for bit.
struct ClipDir {
    F3 d;
    float inv[3];  // 1 / d per axis (unused where |d| < 1e-6)
};
__device__ __forceinline__ ClipDir clip_dir(F3 p0, F3 p1) {
    ClipDir c;
    c.d = f3(p1.x - p0.x, p1.y - p0.y, p1.z - p0.z);
    c.inv[0] = fabsf(c.d.x) < 1e-6f ? 0.0f : 1.0f / c.d.x;
    c.inv[1] = fabsf(c.d.y) < 1e-6f ? 0.0f : 1.0f / c.d.y;
    c.inv[2] = fabsf(c.d.z) < 1e-6f ? 0.0f : 1.0f / c.d.z;
    return c;
}
__device__ __forceinline__ bool clip_axis_pre(float p, float d, float inv_d, float mn, float mx, float& tmin,
                                              float& tmax) {
    if (fabsf(d) < 1e-6f) return !(p < mn || p > mx);
    float a = (mn - p) * inv_d;
    float b = (mx - p) * inv_d;
    if (a > b) { float t = a; a = b; b = t; }
    tmin = wmax(tmin, a);
    tmax = wmin(tmax, b);
    return !(tmin > tmax);
}
__device__ __forceinline__ bool clip_segment_pre(F3 p0, const ClipDir& c, F3 bmin, F3 bmax, F3& o0, F3& o1) {
    const F3 d = c.d;
    float tmin = 0.0f, tmax = 1.0f;
    if (!clip_axis_pre(p0.x, d.x, c.inv[0], bmin.x, bmax.x, tmin, tmax)) return false;
    if (!clip_axis_pre(p0.y, d.y, c.inv[1], bmin.y, bmax.y, tmin, tmax)) return false;
    if (!clip_axis_pre(p0.z, d.z, c.inv[2], bmin.z, bmax.z, tmin, tmax)) return false;
    o0 = f3(p0.x + d.x * tmin, p0.y + d.y * tmin, p0.z + d.z * tmin);
    o1 = f3(p0.x + d.x * tmax, p0.y + d.y * tmax, p0.z + d.z * tmax);
    return true;
}

// v / n in binary32. For a power of two n = 2^k both v / n and v * 2^-k are
// the correctly rounded value of the same real number, so the product (2^-k
// built from its exponent bits) replaces the division bit for bit.
__device__ __forceinline__ float div_by(float v, uint32_t n) {
    if ((n & (n - 1u)) == 0u && n != 0u && n < (1u << 31)) {
        const int k = __ffs((int)n) - 1;
        return v * __int_as_float((127 - k) << 23);
    }
    return v / u2f(n);
}

// Frustum of a coarse tile: frusta own consecutive, increasing tile ranges.
__device__ __forceinline__ uint32_t frustum_for_tile(const FrameParams& P, uint32_t tile) {
    if (P.F == 0u) return kInvalid;
    uint32_t lo = 0, hi = P.F;  // last frustum whose range starts at or before tile
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (P.frusta[mid].coarse_depth_tile_base <= tile) lo = mid; else hi = mid;
    }
    const fiber_frustum_desc& d = P.frusta[lo];
    return tile >= d.coarse_depth_tile_base && tile < d.coarse_depth_tile_base + d.coarse_depth_tile_count ? lo
                                                                                                          : kInvalid;
}
// DOM layer of a light frustum (the count of light frusta before it), kInvalid
// for a camera or beyond the frame's lights.
__device__ __forceinline__ uint32_t light_layer(const FrameParams& P, uint32_t f) {
    return f < P.F ? P.flayer[f] : kInvalid;
}

// ---------------------------------------------------------------------------
// Decoupled look-back (single-pass chained scan, Merrill & Garland 2016).
// status[t] = (epoch << 2 | flag) << 32 | value; flag 1 = block aggregate,
// 2 = inclusive prefix. Words stamped with another frame's epoch read as "not
// ready", so the status arrays are never cleared between frames. Every wait is
// bounded: after kSpinLimit polls the block records kErrTimeout and proceeds
// with what it has, so a broken chain cannot hang the GPU.
// ---------------------------------------------------------------------------
constexpr uint32_t kSpinLimit = 1u << 21;

__device__ __forceinline__ void lb_publish(unsigned long long* status, uint32_t tile, uint32_t epoch, uint32_t flag,
                                           uint32_t value) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> a(status[tile]);
    a.store(((unsigned long long)((epoch << 2) | flag) << 32) | value, cuda::memory_order_release);
}

// Called by one thread. Returns the exclusive prefix of `tile`.
__device__ __forceinline__ uint32_t lb_exclusive(unsigned long long* status, uint32_t tile, uint32_t epoch,
                                                 uint32_t aggregate, uint32_t* error,
                                                 uint32_t spin_limit = kSpinLimit) {
    if (tile == 0) {
        lb_publish(status, 0, epoch, 2u, aggregate);
        return 0u;
    }
    lb_publish(status, tile, epoch, 1u, aggregate);
    uint32_t excl = 0;
    int64_t pred = (int64_t)tile - 1;
    uint32_t spins = 0;
    while (pred >= 0) {
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> a(status[pred]);
        unsigned long long v = a.load(cuda::memory_order_acquire);
        uint32_t hi = (uint32_t)(v >> 32);
        uint32_t flag = (hi >> 2) == (epoch & 0x3FFFFFFFu) ? (hi & 3u) : 0u;
        if (flag == 0u) {
            // Give up after kSpinLimit polls, or at once when another block of
            // this frame already gave up, so a broken chain costs one limit.
            if (++spins > spin_limit || ((spins & 255u) == 0u && *((volatile uint32_t*)error) != 0u)) {
                atomicOr(error, kErrTimeout);
                break;
            }
            __nanosleep(32);
            continue;
        }
        excl += (uint32_t)v;
        if (flag == 2u) break;
        --pred;
    }
    lb_publish(status, tile, epoch, 2u, excl + aggregate);
    return excl;
}

// Warp form of lb_exclusive: called by all 32 lanes of one warp with the same
// tile and aggregate; returns the exclusive prefix in every lane. Each step
// reads a window of 32 predecessors at once (lane i reads tile - 1 - i) and
// adds the values up to the nearest inclusive one, so a block walks back
// through 32 published aggregates per L2 round trip. Waiting is bounded as in
// lb_exclusive, after `spin_limit` polls. A tile equal to `withheld` publishes
// nothing: the frame-level test hook that makes its successors' waits run out
// (fiber_debug_stall_lookback).
__device__ __forceinline__ uint32_t lb_exclusive_warp(unsigned long long* status, uint32_t tile, uint32_t epoch,
                                                      uint32_t aggregate, uint32_t* error,
                                                      uint32_t spin_limit = kSpinLimit,
                                                      uint32_t withheld = kInvalid) {
    const uint32_t lane = threadIdx.x & 31u;
    const bool publish = tile != withheld;
    if (tile == 0) {
        if (lane == 0 && publish) lb_publish(status, 0, epoch, 2u, aggregate);
        return 0u;
    }
    if (lane == 0 && publish) lb_publish(status, tile, epoch, 1u, aggregate);
    uint32_t excl = 0;
    int64_t end = (int64_t)tile;  // window: predecessors end - 1 - lane
    uint32_t spins = 0;
    for (;;) {
        const int64_t pred = end - 1 - (int64_t)lane;
        uint32_t flag = 2u, val = 0u;  // below tile 0: an inclusive zero
        if (pred >= 0) {
            cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> a(status[pred]);
            const unsigned long long v = a.load(cuda::memory_order_acquire);
            const uint32_t hi = (uint32_t)(v >> 32);
            flag = (hi >> 2) == (epoch & 0x3FFFFFFFu) ? (hi & 3u) : 0u;
            val = (uint32_t)v;
        }
        const unsigned incl = __ballot_sync(0xFFFFFFFFu, flag == 2u);
        const unsigned waiting = __ballot_sync(0xFFFFFFFFu, flag == 0u);
        const uint32_t first = incl ? (uint32_t)(__ffs(incl) - 1) : 32u;
        const unsigned needed = first >= 31u ? 0xFFFFFFFFu : ((2u << first) - 1u);
        if (waiting & needed) {
            bool give_up = ++spins > spin_limit;
            if ((spins & 255u) == 0u) {
                const uint32_t err = lane == 0 ? *((volatile uint32_t*)error) : 0u;
                give_up = give_up || __shfl_sync(0xFFFFFFFFu, err, 0) != 0u;
            }
            if (give_up) {
                if (lane == 0) atomicOr(error, kErrTimeout);
                break;
            }
            __nanosleep(32);
            continue;
        }
        uint32_t part = lane <= first ? val : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
        excl += part;
        if (first < 32u) break;
        end -= 32;
    }
    if (lane == 0 && publish) lb_publish(status, tile, epoch, 2u, excl + aggregate);
    return excl;
}

// The look-back wait settings of one stage of this frame.
__device__ __forceinline__ uint32_t lb_limit(const FrameParams& P) {
    return P.lb_spin_limit ? P.lb_spin_limit : kSpinLimit;
}
__device__ __forceinline__ uint32_t lb_withheld(const FrameParams& P, uint32_t stage) {
    return P.lb_stall_stage == stage + 1u ? P.lb_stall_tile : kInvalid;
}

// After a look-back wait gave up, the bases it produced are partial sums (no
// larger than the true ones, so every write stays in bounds) and the arrays
// they index may hold records of earlier frames. Every kernel that consumes
// them starts with this check and does nothing in such a frame, which then
// reports FIBER_ETIMEDOUT.
__device__ __forceinline__ bool frame_failed(const FrameCounters* c) {
    return *((const volatile uint32_t*)&c->error) != 0u;
}

// Block-wide exclusive scan of one value per thread (blockDim multiple of 32).
template <int kThreads>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem_warp, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kThreads / 32 ? smem_warp[lane] : 0u;
        uint32_t s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kThreads / 32) smem_warp[lane] = s - w;
        if (lane == kThreads / 32 - 1) smem_warp[32] = s;
    }
    __syncthreads();
    uint32_t r = smem_warp[warp] + x - v;
    total = smem_warp[32];
    __syncthreads();
    return r;
}

}  // namespace fiber
