// fiber_prepass.cu — work preparation (the reference's work_preparation_pass,
// src/nodes/prepass.rs:27-233 -> run_prepass, src/pipelines/prepass.rs:818-1397).
//
// Stage map (reference entry point -> kernel here):
//   reduce_opaque_depth (opaque_depth_reduce.wgsl:36-86)                -> k_opaque_reduce
//   broad_prepass + broad_strand_prepass (strand_prepass.wgsl:684-782) -> k_broad, folded into k_fine
//   coarse_interval_pass + build_depth_warp_lut (:835-1014)           -> k_lut
//   fine_prepass (:1016-1140)                                           -> k_fine (single-pass compaction)
//   mark_coarse_count_pages_pass (:1928-1932)                           -> k_visit (+ visit records)
//   allocate_coarse_count_pages (:1934-1969)                            -> k_alloc_pages (ordered)
//   binning_queue_pass (:1986-1990)                                     -> k_count_visits | k_traverse<kCount>
//   prefix_fine_pages (:2051-2143)                                      -> k_prefix_pages
//   fill_fine_seg_refs (:2190-2194)                                     -> k_fill_visits | k_traverse<kFill>
//   prefix_active_tile_blocks + compact_active_tiles (:2581-2676)       -> k_compact_active
//   emit_raster_work (:2678-2834)                                       -> k_emit (+ canonical cell order)
// The finalize_* indirect-argument kernels disappear: every consumer is a
// persistent or grid-stride kernel that reads its item count on the device.
// Append orders that the reference takes from atomics are replaced by
// decoupled look-back scans, so every output is deterministic.
#include "fiber_kernels.cuh"

namespace fiber {

// ===========================================================================
// K0 opaque depth reduce: per camera fine tile, whether every pixel holds
// opaque depth (reversed-Z: > 0 after the min over the pixel's samples) and
// the farthest such depth (the min), quantised. One warp per tile; lanes
// stride over the tile's pixels so a warp reads whole image rows. The result
// is a count and a min, so the lane order cannot change it.
// ===========================================================================
__global__ void __launch_bounds__(256) k_opaque_reduce(const FrameParams* __restrict__ Pp, PrepassArgs A,
                                                       const float* __restrict__ depth, uint32_t pitch,
                                                       uint32_t samples) {
    const fiber_frustum_desc& d = Pp->frusta[0];
    const uint32_t tx = (d.screen_width + d.froxel_size_x - 1u) / d.froxel_size_x;
    const uint32_t ty = (d.screen_height + d.froxel_size_y - 1u) / d.froxel_size_y;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    if (blockIdx.x == 0 && threadIdx.x == 0) A.counters->opaque_bound = 1u;
    for (uint32_t t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < tx * ty; t += warps) {
        const uint32_t x0 = (t % tx) * d.froxel_size_x, y0 = (t / tx) * d.froxel_size_y;
        const uint32_t w = min(x0 + d.froxel_size_x, d.screen_width) - x0;
        const uint32_t n = w * (min(y0 + d.froxel_size_y, d.screen_height) - y0);
        uint32_t covered = 0u;
        float farthest = 1.0f;
        for (uint32_t p = lane; p < n; p += 32u) {
            const uint32_t x = x0 + p % w, y = y0 + p / w;
            const float* px = reinterpret_cast<const float*>(reinterpret_cast<const char*>(depth) + (size_t)y * pitch) +
                              (size_t)x * samples;
            float z = __ldg(px);
            for (uint32_t q = 1u; q < samples; ++q) z = wmin(z, __ldg(px + q));
            if (z > 0.0f) {
                ++covered;
                farthest = wmin(farthest, z);
            }
        }
        covered = __reduce_add_sync(0xFFFFFFFFu, covered);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) farthest = wmin(farthest, __shfl_xor_sync(0xFFFFFFFFu, farthest, o));
        if (lane == 0u) A.opaque_tiles[t] = make_uint2(covered == n && n > 0u ? 1u : 0u, quantize_depth01(farthest));
    }
}

// ===========================================================================
// K1 broad prepass: coarse range + keep probabilities per (instance, frustum)
// ===========================================================================
struct CornerScan {
    float sminx, sminy, smaxx, smaxy, zmin, zmax;
    bool any, near_clip;
};

__device__ CornerScan scan_corners(const float4* corners, const float* clip, float vw, float vh) {
    CornerScan s{1e30f, 1e30f, -1e30f, -1e30f, 1.0f, 0.0f, false, false};
    for (int i = 0; i < 8; ++i) {
        float4 c = matvec(clip, corners[i].x, corners[i].y, corners[i].z, corners[i].w);
        if (c.w <= 1e-6f) { s.near_clip = true; continue; }
        float nx = c.x / c.w, ny = c.y / c.w, nz = c.z / c.w;
        if (nz < 0.0f) s.near_clip = true;
        float rx = 0.0f + (nx * 0.5f + 0.5f) * vw;
        float ry = 0.0f + (ny * -0.5f + 0.5f) * vh;
        s.any = true;
        s.sminx = wmin(s.sminx, rx);
        s.sminy = wmin(s.sminy, ry);
        s.smaxx = wmax(s.smaxx, rx);
        s.smaxy = wmax(s.smaxy, ry);
        float z = normalize_depth01(nz);
        s.zmin = wmin(s.zmin, z);
        s.zmax = wmax(s.zmax, z);
    }
    return s;
}

__global__ void k_broad(const FrameParams* __restrict__ Pp, const InstanceView* __restrict__ inst, PrepassArgs A) {
    const FrameParams& P = *Pp;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.I) return;
    const InstanceView& in = inst[i];
    float keep_max = 0.0f;
    bool visible = false;
    float cam_k = 0.0f, sh_k = 0.0f;
    if (in.valid) {
        const float* mn = in.aabb.min;
        const float* mx = in.aabb.max;
        const float cx[8][3] = {{mn[0], mn[1], mn[2]}, {mn[0], mn[1], mx[2]}, {mn[0], mx[1], mn[2]},
                                {mn[0], mx[1], mx[2]}, {mx[0], mn[1], mn[2]}, {mx[0], mn[1], mx[2]},
                                {mx[0], mx[1], mn[2]}, {mx[0], mx[1], mx[2]}};
        float4 corners[8];
        for (int c = 0; c < 8; ++c) corners[c] = matvec(in.world_from_local, cx[c][0], cx[c][1], cx[c][2], 1.0f);
        for (uint32_t f = 0; f < P.F; ++f) {
            const fiber_frustum_desc& d = P.frusta[f];
            float k = 0.0f;
            uint32_t slot = i * P.F + f;
            A.range_valid[slot] = 0u;
            // A frustum of another view of a multi-view frame does not see it.
            if (d.kind <= 1u && P.fview[f] == in.view) {
                // emit_coarse_asset_range_for_aabb (strand_prepass.wgsl:575-682)
                bool vis = false;
                float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
                if (d.coarse_depth_tile_count != 0u && !(d.kind == 1u && light_layer(P, f) == kInvalid)) {
                    CornerScan s = scan_corners(corners, P.clip[f], vw, vh);
                    if (s.near_clip) {
                        s.sminx = 0.0f; s.sminy = 0.0f;
                        s.smaxx = vw - 1.0f; s.smaxy = vh - 1.0f;
                        s.zmax = 1.0f;
                        if (!s.any) s.zmin = 0.0f;
                        s.any = true;
                    }
                    if (s.any && !(s.smaxx < 0.0f || s.smaxy < 0.0f || s.sminx >= vw || s.sminy >= vh) &&
                        !(s.zmax < 0.0f || s.zmin > 1.0f)) {
                        uint32_t cpx = max(1u, d.froxel_size_x * kCoarseExtent);
                        uint32_t cpy = max(1u, d.froxel_size_y * kCoarseExtent);
                        float cminx = wclamp(s.sminx, 0.0f, vw - 1.0f), cminy = wclamp(s.sminy, 0.0f, vh - 1.0f);
                        float cmaxx = wclamp(s.smaxx, 0.0f, vw - 1.0f), cmaxy = wclamp(s.smaxy, 0.0f, vh - 1.0f);
                        fiber_coarse_asset_range r;
                        r.geo_id = i;
                        r.frustum_id = f;
                        r.min_x = min(f2u(cminx) / cpx, d.coarse_tiles_x - 1u);
                        r.max_x = min(f2u(cmaxx) / cpx, d.coarse_tiles_x - 1u);
                        r.min_y = min(f2u(cminy) / cpy, d.coarse_tiles_y - 1u);
                        r.max_y = min(f2u(cmaxy) / cpy, d.coarse_tiles_y - 1u);
                        r.z_min_q = quantize_depth01(s.zmin);
                        r.z_max_q = quantize_depth01(s.zmax);
                        A.ranges[slot] = r;
                        A.range_valid[slot] = 1u;
                        vis = true;
                    }
                }
                visible = vis || visible;
                if (vis && A.tel) {  // FRUSTUM_TELEMETRY_VISIBLE_* (:735-738)
                    atomicAdd(tel_frustum(A.tel, f, kTelVisibleInstances), 1u);
                    atomicAdd(tel_frustum(A.tel, f, kTelVisibleStrands), in.strand_count);
                }
                if (vis) {
                    // aabb_projected_screen_area (:295-362)
                    CornerScan s = scan_corners(corners, P.clip[f], vw, vh);
                    float area;
                    if (s.near_clip) area = vw * vh;
                    else if (!s.any) area = -1.0f;
                    else if (s.smaxx < 0.0f || s.smaxy < 0.0f || s.sminx >= vw || s.sminy >= vh) area = -1.0f;
                    else if (s.zmax < 0.0f || s.zmin > 1.0f) area = -1.0f;
                    else {
                        float cminx = wclamp(s.sminx, 0.0f, vw - 1.0f), cminy = wclamp(s.sminy, 0.0f, vh - 1.0f);
                        float cmaxx = wclamp(s.smaxx, 0.0f, vw - 1.0f), cmaxy = wclamp(s.smaxy, 0.0f, vh - 1.0f);
                        area = wmax(cmaxx - cminx, 1.0f) * wmax(cmaxy - cminy, 1.0f);
                    }
                    // stochastic_{camera,shadow}_keep_probability (:364-392)
                    if (P.stochastic_cull_enabled == 0u) k = 1.0f;
                    else if (area < 0.0f) k = 0.0f;
                    else {
                        float density = wmax(P.target_strands_per_pixel, 1e-5f);
                        float min_keep = wclamp(P.min_keep_probability, 0.0f, 1.0f);
                        float area_keep = wclamp(area * density / wmax(u2f(in.strand_count), 1.0f), min_keep, 1.0f);
                        if (d.kind == 0u) k = area_keep;
                        else {
                            float cap = wclamp(P.shadow_keep_probability, 0.0f, 1.0f);
                            float curved = area_keep * area_keep;
                            float scale = 1.0f / exp2f(u2f(d.cascade_index));
                            k = wclamp(curved * scale * cap, min_keep, 1.0f);
                        }
                    }
                    if (d.kind == 0u) cam_k = wmax(cam_k, k);
                    else sh_k = wmax(sh_k, k);
                }
            }
            A.keep[slot] = k;
        }
        keep_max = wmax(cam_k, sh_k);
    } else {
        for (uint32_t f = 0; f < P.F; ++f) {
            A.range_valid[i * P.F + f] = 0u;
            A.keep[i * P.F + f] = 0.0f;
        }
    }
    A.inst_visible[i] = visible ? 1u : 0u;
    A.inst_keep[i] = keep_max;
}

// ===========================================================================
// K4 + K5: per coarse tile, merge the depth intervals of the ranges covering
// it (instance order) and split 16 LUT slices across them.
// ===========================================================================
__global__ void k_lut(const FrameParams* __restrict__ Pp, PrepassArgs A) {
    const FrameParams& P = *Pp;
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.total_coarse_tiles) return;
    fiber_coarse_depth_lut_entry* out = A.lut + (size_t)t * kDepthSlices;
    uint32_t f = frustum_for_tile(P, t);
    uint32_t mins[kDepthSlices], maxs[kDepthSlices];
    uint32_t count = 0;
    if (f != kInvalid) {
        const fiber_frustum_desc& d = P.frusta[f];
        uint32_t local = t - d.coarse_depth_tile_base;
        uint32_t cx = local % d.coarse_tiles_x, cy = local / d.coarse_tiles_x;
        for (uint32_t i = 0; i < P.I; ++i) {
            uint32_t slot = i * P.F + f;
            if (!A.range_valid[slot]) continue;
            fiber_coarse_asset_range r = A.ranges[slot];
            if (r.max_x < r.min_x || r.max_y < r.min_y) continue;
            if (cx < r.min_x || cx > r.max_x || cy < r.min_y || cy > r.max_y) continue;
            uint32_t zmin = min(r.z_min_q, r.z_max_q), zmax = max(r.z_min_q, r.z_max_q);
            bool merged = false;
            for (uint32_t k = 0; k < count; ++k) {
                if (zmin <= maxs[k] + 1u && zmax + 1u >= mins[k]) {
                    mins[k] = min(mins[k], zmin);
                    maxs[k] = max(maxs[k], zmax);
                    merged = true;
                }
            }
            if (merged) continue;
            if (count < kDepthSlices) {
                mins[count] = zmin;
                maxs[count] = zmax;
                ++count;
            } else {
                uint32_t best = 0, best_gap = 0xFFFFFFFFu;
                for (uint32_t k = 0; k < kDepthSlices; ++k) {
                    uint32_t g = maxs[k] < zmin ? zmin - maxs[k] : (zmax < mins[k] ? mins[k] - zmax : 0u);
                    if (g < best_gap) { best_gap = g; best = k; }
                }
                mins[best] = min(mins[best], zmin);
                maxs[best] = max(maxs[best], zmax);
            }
        }
    }
    for (uint32_t k = 1; k < count; ++k) {
        uint32_t j = k, kmin = mins[k], kmax = maxs[k];
        while (j != 0 && mins[j - 1] > kmin) {
            mins[j] = mins[j - 1];
            maxs[j] = maxs[j - 1];
            --j;
        }
        mins[j] = kmin;
        maxs[j] = kmax;
    }
    uint32_t out_slice = 0;
    // simple: all 16 entries populated, each start <= end, each end below the
    // next start (the lookup in lut_slices may then binary-search).
    bool simple = true;
    uint32_t prev_end = 0u;
    for (uint32_t k = 0; k < count; ++k) {
        uint32_t base_slices = max(1u, kDepthSlices / count);
        uint32_t rem = kDepthSlices % count;
        uint32_t slices = base_slices + (k < rem ? 1u : 0u);
        uint32_t span = max(1u, maxs[k] - mins[k] + 1u);
        for (uint32_t s = 0; s < slices && out_slice < kDepthSlices; ++s) {
            uint32_t start = mins[k] + (span * s) / slices;
            uint32_t excl_end = mins[k] + (span * (s + 1u)) / slices;
            uint32_t end = min(excl_end > start ? excl_end - 1u : start, maxs[k]);
            simple = simple && start <= end && (out_slice == 0u || prev_end < start);
            prev_end = end;
            out[out_slice++] = fiber_coarse_depth_lut_entry{start, end, start, max(1u, end - start + 1u)};
        }
    }
    for (uint32_t k = out_slice; k < kDepthSlices; ++k) out[k] = fiber_coarse_depth_lut_entry{0u, 0u, 0u, 0u};
    // The search tree of a simple LUT (read back from this thread's own
    // entries); word 0 = kInvalid marks a LUT that takes the linear lookup.
    uint4* tree = reinterpret_cast<uint4*>(A.lut_tree + (size_t)t * kLutTreeWords);
    if (simple && out_slice == kDepthSlices) {
        tree[0] = make_uint4(out[0].z_min_q, out[4].z_min_q, out[8].z_min_q, out[12].z_min_q);
        for (uint32_t g = 0; g < 4u; ++g) {
            const fiber_coarse_depth_lut_entry* e = out + 4u * g;
            tree[1u + 2u * g] = make_uint4(e[0].z_min_q, e[1].z_min_q, e[2].z_min_q, e[3].z_min_q);
            tree[2u + 2u * g] = make_uint4(e[0].z_max_q, e[1].z_max_q, e[2].z_max_q, e[3].z_max_q);
        }
    } else {
        tree[0] = make_uint4(kInvalid, kInvalid, kInvalid, kInvalid);
    }
}

// ===========================================================================
// K2 + K6 fine prepass: a warp per strand (a lane per segment), each warp
// taking kFineStrandsPerWarp consecutive strands, one block per (frustum,
// kFineStrandsPerTile-strand chunk) in frustum-major order. Pass A counts
// every strand's clipped segments; the block takes its output offset from a
// decoupled look-back; pass B projects again and writes BinningTask +
// ProjectedSegment in (frustum, inst, strand, seg) order — the binning
// queue's canonical order, produced without a sort. A tile of 64 strands
// spends one look-back (and two block barriers) on 64 strands' work.
// ===========================================================================
constexpr int kFineThreads = 256;
constexpr int kFineWarps = kFineThreads / 32;
constexpr uint32_t kFineStrandsPerWarp = kFineStrandsPerTile / kFineWarps;
static_assert(kFineStrandsPerWarp * kFineWarps == kFineStrandsPerTile, "fine tile shape");

struct SegOut {
    uint32_t seg;
    uint32_t p0, p1, dz;
    float4 r0, r1;  // world_to_screen_raw of both end points, kept for the rasters
};

// world_to_screen_raw (common.wgsl:93-107) of the strand point at index
// position `pos` after the instance transform.
__device__ __forceinline__ float4 fine_vertex(const FrameParams& P, const InstanceView& in, uint32_t f, uint32_t pos) {
    const fiber_frustum_desc& d = P.frusta[f];
    const float4 a = __ldg(in.vertices + __ldg(in.indices + pos));
    const float4 w = matvec(in.world_from_local, a.x, a.y, a.z, 1.0f);
    return world_to_screen_raw(w, P.clip[f], u2f(d.screen_width), u2f(d.screen_height));
}

// A segment from its two projected end points: normalised depth, clip to the
// screen box, quantise (fine_prepass, strand_prepass.wgsl:1016-1140).
__device__ __forceinline__ bool fine_segment(const FrameParams& P, uint32_t f, uint32_t seg, float4 r0, float4 r1,
                                             SegOut& o) {
    const fiber_frustum_desc& d = P.frusta[f];
    const float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
    F3 p0 = f3(r0.x, r0.y, normalize_depth01(r0.z)), p1 = f3(r1.x, r1.y, normalize_depth01(r1.z));
    F3 c0, c1;
    if (!clip_segment(p0, p1, f3(0.0f, 0.0f, 0.0f), f3(wmax(0.0f, vw - 1e-3f), wmax(0.0f, vh - 1e-3f), 1.0f), c0, c1))
        return false;
    float ssx = wmax(1.0f, vw), ssy = wmax(1.0f, vh);
    o.seg = seg;
    o.r0 = r0;
    o.r1 = r1;
    o.p0 = pack2x16unorm(wclamp(c0.x / ssx, 0.0f, 1.0f), wclamp(c0.y / ssy, 0.0f, 1.0f));
    o.p1 = pack2x16unorm(wclamp(c1.x / ssx, 0.0f, 1.0f), wclamp(c1.y / ssy, 0.0f, 1.0f));
    o.dz = pack2x16unorm(wclamp(c0.z, 0.0f, 1.0f), wclamp(c1.z, 0.0f, 1.0f));
    return true;
}

// Segments c .. c + 30 of a strand, one per lane 0..30: lane l projects point
// c + l once and takes its segment's far end point from lane l + 1 (a point
// shared by two segments is projected once, by the same operations).
constexpr uint32_t kFineChunk = 31;
__device__ __forceinline__ bool fine_chunk(const FrameParams& P, const InstanceView& in, uint32_t f,
                                           uint32_t first, uint32_t nseg, uint32_t c, uint32_t lane, SegOut& o) {
    const uint32_t pos = first + c + lane;
    const bool has_point = c + lane <= nseg && pos < in.n_indices;
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (has_point) r = fine_vertex(P, in, f, pos);
    float4 r1;
    r1.x = __shfl_down_sync(0xFFFFFFFFu, r.x, 1);
    r1.y = __shfl_down_sync(0xFFFFFFFFu, r.y, 1);
    r1.z = __shfl_down_sync(0xFFFFFFFFu, r.z, 1);
    r1.w = __shfl_down_sync(0xFFFFFFFFu, r.w, 1);
    const bool seg_ok = lane < kFineChunk && c + lane < nseg && pos + 1u < in.n_indices;
    return seg_ok && fine_segment(P, f, pos, r, r1, o);
}

// The strand g of frustum f: instance, local strand, segment count, first
// index and the task's packed field; nseg = 0 when the keep tests drop it.
struct FineStrand {
    uint32_t i, s, nseg, meta_offset, packed;
};

__device__ __forceinline__ FineStrand fine_strand(const FrameParams& P, const InstanceView* __restrict__ inst,
                                                  const PrepassArgs& A, uint32_t f, uint32_t g, uint32_t g_end) {
    FineStrand r{0u, 0u, 0u, 0u, 0u};
    if (g >= g_end) return r;
    uint32_t lo = 0, hi = P.I;  // last instance with strand_base <= g
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (inst[mid].strand_base <= g) lo = mid; else hi = mid;
    }
    r.i = lo;
    r.s = g - inst[lo].strand_base;
    const InstanceView& in = inst[lo];
    const fiber_frustum_desc& d = P.frusta[f];
    // The keep hash takes the instance's id inside its view, so a view keeps
    // the same strands in a multi-view frame as alone (one view: the id).
    const uint32_t local_i = lo - P.view_inst0[P.fview[f]];
    const float h = hash_to_unit_float(wang_hash((local_i * 16777619u) ^ r.s));
    bool ok = in.valid && in.view == P.fview[f] && A.inst_visible[lo] != 0u && r.s < in.strand_count &&
              !(h > A.inst_keep[lo]);
    ok = ok && d.kind <= 1u && r.s < in.n_meta;
    if (ok) {
        const fiber_strand_meta m = in.meta[r.s];
        ok = m.count >= 2u && !(h > A.keep[lo * P.F + f]) && !(d.kind == 1u && light_layer(P, f) == kInvalid);
        if (ok) {
            r.nseg = m.count - 1u;
            r.meta_offset = m.offset;
            r.packed = ((d.kind == 1u ? 1u : 0u) << 2u) | (f << 3u);
        }
    }
    return r;
}

__global__ void __launch_bounds__(kFineThreads, 4) k_fine(const FrameParams* __restrict__ Pp,
                                                       const InstanceView* __restrict__ inst, PrepassArgs A) {
    const FrameParams& P = *Pp;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_count[kFineWarps];
    __shared__ uint32_t s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Each frustum's tiles cover its view's strands (every strand of a
    // single-view frame): fine_tile_base is their prefix over frusta.
    const uint32_t n_tiles = P.fine_tile_base[P.F];
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(A.tile_counter, 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= n_tiles) break;
        uint32_t f = 0, fhi = P.F;  // last frustum whose tiles start at or before tile
        while (fhi - f > 1u) {
            const uint32_t mid = (f + fhi) >> 1;
            if (P.fine_tile_base[mid] <= tile) f = mid; else fhi = mid;
        }
        const uint32_t lt = tile - P.fine_tile_base[f];
        const uint32_t v = P.fview[f];
        const uint32_t g_end = P.view_strand0[v] + P.view_strands[v];
        const uint32_t g0 = P.view_strand0[v] + lt * kFineStrandsPerTile + (uint32_t)warp * kFineStrandsPerWarp;
        // Pass A: count the clipped segments of the warp's strands.
        uint32_t count = 0;
        for (uint32_t k = 0; k < kFineStrandsPerWarp; ++k) {
            const FineStrand fs = fine_strand(P, inst, A, f, g0 + k, g_end);
            // FRUSTUM_TELEMETRY_RETAINED_STRANDS (:1085): every strand the
            // keep tests pass.
            if (A.tel && lane == 0 && fs.nseg > 0u) atomicAdd(tel_frustum(A.tel, f, kTelRetainedStrands), 1u);
            for (uint32_t c = 0; c < fs.nseg; c += kFineChunk) {
                SegOut o;
                const bool ok = fine_chunk(P, inst[fs.i], f, fs.meta_offset, fs.nseg, c, lane, o);
                count += __popc(__ballot_sync(0xFFFFFFFFu, ok));
            }
        }
        if (lane == 0) s_warp_count[warp] = count;
        __syncthreads();
        if (threadIdx.x < 32u) {
            uint32_t agg = 0;
            for (int w = 0; w < kFineWarps; ++w) agg += s_warp_count[w];
            uint32_t base = lb_exclusive_warp(A.lb_status, tile, P.epoch, agg, &A.counters->error, lb_limit(P),
                                              lb_withheld(P, kStageFine));
            if (threadIdx.x == 0) {
                s_base = base;
                if (lt == 0u) A.counters->frustum_task_base[f] = base;
                if (tile == n_tiles - 1u) {
                    A.counters->tasks = base + agg;
                    A.counters->frustum_task_base[P.F] = base + agg;
                }
            }
        }
        __syncthreads();
        uint32_t out = s_base;
        for (int w = 0; w < warp; ++w) out += s_warp_count[w];
        // Pass B: project again and write in segment order.
        for (uint32_t k = 0; k < kFineStrandsPerWarp; ++k) {
            const FineStrand fs = fine_strand(P, inst, A, f, g0 + k, g_end);
            for (uint32_t c = 0; c < fs.nseg; c += kFineChunk) {
                SegOut o;
                const bool ok = fine_chunk(P, inst[fs.i], f, fs.meta_offset, fs.nseg, c, lane, o);
                const uint32_t mask = __ballot_sync(0xFFFFFFFFu, ok);
                if (ok) {
                    const uint32_t dst = out + __popc(mask & ((1u << lane) - 1u));
                    if (dst < P.task_capacity) {
                        reinterpret_cast<uint4*>(A.tasks)[dst] = make_uint4(fs.i, fs.s, o.seg, fs.packed);
                        fiber_projected_segment ps{o.p0, o.p1, o.dz};
                        A.projected[dst] = ps;
                        A.task_proj[2u * (size_t)dst] = o.r0;
                        A.task_proj[2u * (size_t)dst + 1u] = o.r1;
                    } else {
                        atomicOr(&A.counters->overflow, 1u);
                    }
                }
                out += __popc(mask);
            }
        }
        __syncthreads();
    }
}

// ===========================================================================
// K7 / K9 / K11 traversal: coarse-tile 2-D DDA, LUT slices, then the fine
// 3-D DDA inside each page (strand_prepass.wgsl:1251-1696,1894-1926).
//
// The walk is written once; what a pass does at a page-table slot that
// survives the depth clip, and at each fine cell the 3-D DDA visits, is a sink:
//   VisitSink  k_visit: marks the slot (mark_coarse_count_pages_pass) and
//              records the visit (slot << 8 | cell) in a per-thread buffer
//   SpillSink  k_visit: re-walks a task with more visits than the buffer and
//              writes the visits past it
//   CountSink, FillSink  the walking form of binning_queue_pass and
//              fill_fine_seg_refs, used only when the visit records did not fit
// With the records, the count and fill passes stream over visits instead of
// walking every task again (k_count_visits, k_fill_visits).
// ===========================================================================
enum : int { kCount = 1, kFill = 2 };
constexpr uint32_t kVisitThreads = 256;
constexpr uint32_t kVisitSlots = 32;  // buffered visits per task; p99 is about 17 on the camera
// Cell sort sizes: a thread sorts a cell of up to 8 references, a warp one of
// up to 256 (32 lanes x 8 registers), a block anything longer.
constexpr uint32_t kThreadSortMax = 8;
constexpr uint32_t kGroupSortMax = 32;  // 8 lanes x 4 registers: four cells per warp
constexpr uint32_t kWarpSortMax = 256;

// lut_slices for one end point of a LUT whose 16 entries are all populated,
// each start <= end and each end below the next start: at most one entry
// holds the quantised depth q, and the nearest entry otherwise is a neighbour
// of the gap q falls in, so the last entry whose start is <= q (the starts
// increase strictly) answers what the linear scan answers (first holding
// entry, else first nearest). The search reads the LUT's tree: the quarter
// starts (piv, shared by both end points), then the quarter's starts and ends.
__device__ __forceinline__ uint32_t lut_slice_tree(const uint4* tree, const uint4& piv, float z) {
    const uint32_t q = quantize_depth01(z);
    if (piv.x > q) return 0u;  // no entry starts at or below q: the first is nearest
    const uint32_t g = (piv.y <= q ? 1u : 0u) + (piv.z <= q ? 1u : 0u) + (piv.w <= q ? 1u : 0u);
    const uint4 st = __ldg(tree + 1u + 2u * g), en = __ldg(tree + 2u + 2u * g);
    const uint32_t r = (st.y <= q ? 1u : 0u) + (st.z <= q ? 1u : 0u) + (st.w <= q ? 1u : 0u);
    const uint32_t lo = 4u * g + r;
    const uint32_t end = r == 0u ? en.x : (r == 1u ? en.y : (r == 2u ? en.z : en.w));
    if (q <= end || lo == kDepthSlices - 1u) return lo;
    const uint32_t next_piv = g == 0u ? piv.y : (g == 1u ? piv.z : piv.w);
    const uint32_t next_start = r == 0u ? st.y : (r == 1u ? st.z : (r == 2u ? st.w : next_piv));
    return (q - end <= next_start - q) ? lo : lo + 1u;
}

// lut_slice for both clipped end points at once: per end point, the first
// populated slice whose [z_min_q, z_max_q] holds its quantised depth, else the
// first populated slice nearest to it, else kInvalid. One unrolled pass over
// the 16 entries without an early exit, so their loads issue together.
__device__ __forceinline__ void lut_slices(const fiber_coarse_depth_lut_entry* e, float za, float zb, uint32_t& sa,
                                           uint32_t& sb) {
    const uint32_t qa = quantize_depth01(za), qb = quantize_depth01(zb);
    uint32_t fa = kInvalid, fb = kInvalid, ba = kInvalid, bb = kInvalid, da = 0xFFFFFFFFu, db = 0xFFFFFFFFu;
#pragma unroll
    for (uint32_t i = 0; i < kDepthSlices; ++i) {
        const uint4 x = __ldg(reinterpret_cast<const uint4*>(e) + i);  // z_min_q, z_max_q, -, virtual_count_q
        if (x.w == 0u) continue;
        if (qa >= x.x && qa <= x.y && fa == kInvalid) fa = i;
        if (qb >= x.x && qb <= x.y && fb == kInvalid) fb = i;
        const uint32_t ea = qa > x.y ? qa - x.y : x.x - qa;  // meaningful only while nothing holds qa
        const uint32_t eb = qb > x.y ? qb - x.y : x.x - qb;
        if (ea < da) { da = ea; ba = i; }
        if (eb < db) { db = eb; bb = i; }
    }
    sa = fa != kInvalid ? fa : ba;
    sb = fb != kInvalid ? fb : bb;
}

// Sinks. page_slot(pti) returns whether to walk the slot's fine cells.
// kTel: count the task as a candidate of the slot (telemetry); a task visits
// each slot once.
template <bool kTel>
struct VisitSink {
    uint32_t* page_table;
    uint32_t* buf;  // this thread's column of the block buffer (stride kVisitThreads)
    uint32_t cur, n;
    bool records;
    uint32_t* tel_slots;
    __device__ __forceinline__ bool page_slot(uint32_t pti) {
        page_table[pti] = kMarked;
        if (kTel) atomicAdd(tel_slots + pti, 1u);
        cur = pti << 8;
        return records;
    }
    __device__ __forceinline__ void cell(uint32_t c) {
        if (n < kVisitSlots) buf[n * kVisitThreads] = cur | c;
        ++n;
    }
};

struct SpillSink {
    uint32_t* rec;
    uint32_t* task;
    uint32_t at, k, lim, cur, n;  // lim: visits the first walk counted (the room reserved)
    __device__ __forceinline__ bool page_slot(uint32_t pti) {
        cur = pti << 8;
        return true;
    }
    __device__ __forceinline__ void cell(uint32_t c) {
        if (n >= kVisitSlots && n < lim) {
            rec[at + n] = cur | c;
            task[at + n] = k;
        }
        ++n;
    }
};

struct CountSink {
    const uint32_t* page_table;
    uint32_t* counts;
    uint32_t page;
    __device__ __forceinline__ bool page_slot(uint32_t pti) {
        uint32_t h = page_table[pti];
        if (h == 0u || h == kMarked) return false;
        page = h - 1u;
        return true;
    }
    __device__ __forceinline__ void cell(uint32_t c) { atomicAdd(counts + (size_t)page * kPageSize + c, 1u); }
};

struct FillSink {
    const PrepassArgs* A;
    uint32_t page, base, count, task;
    __device__ __forceinline__ bool page_slot(uint32_t pti) {
        uint32_t h = A->page_table[pti];
        if (h == 0u || h == kMarked) return false;
        page = h - 1u;
        const fiber_fine_page_meta pm = A->page_meta[page];
        base = pm.seg_ref_base;
        count = pm.seg_ref_count;
        return count != 0u;
    }
    __device__ __forceinline__ void cell(uint32_t c) {
        const size_t g = (size_t)page * kPageSize + c;
        const uint32_t lw = atomicAdd(A->cursors + g, 1u);
        const uint64_t dst = (uint64_t)base + A->offsets[g] + lw;
        if (dst >= (uint64_t)base + count) return;
        A->ref_keys[dst] = task;  // k_sort_cells turns it into the reference
    }
};

// opq: the opaque fine tiles of the camera (null when none are bound); pd:
// the segment's clip direction (p1 - p0 and its reciprocals); (ccx, ccy): the
// coarse tile's column and row in the frustum.
template <class Sink>
__device__ __forceinline__ void walk_page(const PrepassArgs& A, F3 p0, const ClipDir& pd, const fiber_frustum_desc& d,
                                          uint32_t tile, uint32_t ccx, uint32_t ccy, const uint2* opq, Sink& sink) {
    // fine_tile_occluded_by_opaque (:551-573) applies to the camera only. The
    // opaque tiles hold the camera's fine tiles alone, so the camera's
    // fine_depth_tile_base (0) is not added.
    if (d.kind != 0u) opq = nullptr;
    uint32_t ftx = 0u, fty = 0u;
    if (opq) {
        ftx = (d.screen_width + d.froxel_size_x - 1u) / d.froxel_size_x;
        fty = (d.screen_height + d.froxel_size_y - 1u) / d.froxel_size_y;
    }
    uint32_t cpx = max(1u, d.froxel_size_x * kCoarseExtent);
    uint32_t cpy = max(1u, d.froxel_size_y * kCoarseExtent);
    float ox = u2f(ccx * cpx), oy = u2f(ccy * cpy);
    float tmx = wmin(ox + u2f(cpx), u2f(d.screen_width)) - 1e-3f;
    float tmy = wmin(oy + u2f(cpy), u2f(d.screen_height)) - 1e-3f;
    F3 bmax = f3(wmax(ox, tmx), wmax(oy, tmy), 1.0f);
    F3 c0, c1;
    if (!clip_segment_pre(p0, pd, f3(ox, oy, 0.0f), bmax, c0, c1)) return;
    const ClipDir cd = clip_dir(c0, c1);  // shared by the slice clips below
    const fiber_coarse_depth_lut_entry* lut = A.lut + (size_t)tile * kDepthSlices;
    const uint4* tree = reinterpret_cast<const uint4*>(A.lut_tree + (size_t)tile * kLutTreeWords);
    const uint4 piv = __ldg(tree);
    uint32_t z0s, z1s;
    if (piv.x != kInvalid) {
        z0s = lut_slice_tree(tree, piv, c0.z);
        z1s = lut_slice_tree(tree, piv, c1.z);
    } else {
        lut_slices(lut, c0.z, c1.z, z0s, z1s);
    }
    if (z0s == kInvalid || z1s == kInvalid) return;
    for (uint32_t cz = min(z0s, z1s); cz <= max(z0s, z1s); ++cz) {
        fiber_coarse_depth_lut_entry e = lut[cz];
        if (e.virtual_count_q == 0u) continue;
        float zmin = dequantize_depth01(e.z_min_q), zmax = dequantize_depth01(e.z_max_q);
        F3 d0, d1;
        if (!clip_segment_pre(c0, cd, f3(ox, oy, zmin), f3(bmax.x, bmax.y, zmax), d0, d1)) continue;
        if (!sink.page_slot(tile * kDepthSlices + cz)) continue;
        float zspan = wmax(zmax - zmin, 1.0f / (float)kDepthQuantMax);
        const uint32_t fsx = d.froxel_size_x, fsy = d.froxel_size_y;
        float l0[3] = {div_by(d0.x - ox, fsx), div_by(d0.y - oy, fsy),
                       wclamp((d0.z - zmin) / zspan, 0.0f, 0.999999f) * 16.0f};
        float l1[3] = {div_by(d1.x - ox, fsx), div_by(d1.y - oy, fsy),
                       wclamp((d1.z - zmin) / zspan, 0.0f, 0.999999f) * 16.0f};
        int32_t f1[3], fc[3], step[3];
        float tm[3], dd[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int32_t hi = a == 2 ? 15 : 3;
            fc[a] = iclamp(f2i(floorf(l0[a])), 0, hi);
            f1[a] = iclamp(f2i(floorf(l1[a])), 0, hi);
            float dir = l1[a] - l0[a];
            step[a] = sgn_i32(dir);
            float sd = fabsf(dir) < 1e-6f ? 1e-6f : dir;
            dd[a] = fabsf(1.0f / sd);
            float fl = floorf(l0[a]);
            tm[a] = step[a] > 0 ? ((fl + 1.0f) - l0[a]) / sd : (fl - l0[a]) / sd;
            if (fabsf(dir) < 1e-6f) tm[a] = 1e38f;
        }
        uint32_t safety = 0;
        for (;;) {
            if (safety > kCoarseExtent + kCoarseExtent + kDepthSlices + 3u) break;
            // A covered fine tile whose farthest opaque depth is in front of
            // this slice's nearest depth (reversed-Z: z_max) hides the cell.
            bool occluded = false;
            if (opq) {
                const uint32_t fx = ccx * kCoarseExtent + (uint32_t)fc[0], fy = ccy * kCoarseExtent + (uint32_t)fc[1];
                if (fx < ftx && fy < fty) {
                    const uint2 o = __ldg(opq + (size_t)fy * ftx + fx);
                    occluded = o.x != 0u && zmax <= dequantize_depth01(o.y) - 1e-4f;
                }
            }
            if (!occluded) sink.cell((uint32_t)((fc[2] * 4 + fc[1]) * 4 + fc[0]));
            if (fc[0] == f1[0] && fc[1] == f1[1] && fc[2] == f1[2]) break;
            float m = wmin(wmin(tm[0], tm[1]), tm[2]);  // canonical_min_mask
            int a = tm[0] == m ? 0 : (tm[1] == m ? 1 : 2);
            if (a == 0) { fc[0] += step[0]; tm[0] += dd[0]; }
            else if (a == 1) { fc[1] += step[1]; tm[1] += dd[1]; }
            else { fc[2] += step[2]; tm[2] += dd[2]; }
            if (fc[0] < 0 || fc[1] < 0 || fc[2] < 0 || fc[0] >= 4 || fc[1] >= 4 || fc[2] >= 16) break;
            ++safety;
        }
    }
}

// One binning task's walk inputs (binning_queue_pass preamble, :1894-1926).
struct TaskWalk {
    F3 p0, p1;        // projected endpoints in pixels / depth01
    uint32_t f;       // frustum
    uint32_t i, strand, seg;
    uint32_t depths;  // packed projected depths (the sort key source)
    uint32_t min_cx, max_cx, min_cy, max_cy;
};

__device__ __forceinline__ bool task_walk(const FrameParams& P, const PrepassArgs& A, uint32_t k, TaskWalk& w) {
    const uint4 t = reinterpret_cast<const uint4*>(A.tasks)[k];
    const uint32_t f = t.w >> 3u;
    if (f >= P.F) return false;
    const uint32_t i = t.x;
    if (i >= P.I) return false;
    const fiber_frustum_desc& d = P.frusta[f];
    const fiber_projected_segment pr = A.projected[k];
    const float sw = u2f(d.screen_width), sh = u2f(d.screen_height);
    const float2 a = unpack2x16unorm(pr.p0_xy), b = unpack2x16unorm(pr.p1_xy), z = unpack2x16unorm(pr.depths);
    const F3 p0 = f3(a.x * sw, a.y * sh, z.x), p1 = f3(b.x * sw, b.y * sh, z.y);
    const uint32_t slot = i * P.F + f;
    if (!A.range_valid[slot]) return false;
    const fiber_coarse_asset_range r = A.ranges[slot];
    const uint32_t cpx = max(1u, d.froxel_size_x * kCoarseExtent);
    const uint32_t cpy = max(1u, d.froxel_size_y * kCoarseExtent);
    w.min_cx = max(r.min_x, min(f2u(wmax(wmin(p0.x, p1.x), 0.0f)) / cpx, d.coarse_tiles_x - 1u));
    w.max_cx = min(r.max_x, min(f2u(wmax(wmax(p0.x, p1.x), 0.0f)) / cpx, d.coarse_tiles_x - 1u));
    w.min_cy = max(r.min_y, min(f2u(wmax(wmin(p0.y, p1.y), 0.0f)) / cpy, d.coarse_tiles_y - 1u));
    w.max_cy = min(r.max_y, min(f2u(wmax(wmax(p0.y, p1.y), 0.0f)) / cpy, d.coarse_tiles_y - 1u));
    if (w.max_cx < w.min_cx || w.max_cy < w.min_cy) return false;
    w.p0 = p0;
    w.p1 = p1;
    w.f = f;
    w.i = i;
    w.strand = t.y;
    w.seg = t.z;
    w.depths = pr.depths;
    return true;
}

// Coarse-tile 2-D DDA over the task's clipped range; each coarse tile is
// walked by walk_page.
template <class Sink>
__device__ __forceinline__ void walk_task(const FrameParams& P, const PrepassArgs& A, const TaskWalk& w,
                                          const uint2* opq, Sink& sink) {
    const fiber_frustum_desc& d = P.frusta[w.f];
    const float sw = u2f(d.screen_width), sh = u2f(d.screen_height);
    const uint32_t cpx = max(1u, d.froxel_size_x * kCoarseExtent);
    const uint32_t cpy = max(1u, d.froxel_size_y * kCoarseExtent);
    const uint32_t min_cx = w.min_cx, max_cx = w.max_cx, min_cy = w.min_cy, max_cy = w.max_cy;
    F3 bmin = f3(u2f(min_cx * cpx), u2f(min_cy * cpy), 0.0f);
    F3 bmax = f3(wmin(u2f((max_cx + 1u) * cpx), sw) - 1e-3f, wmin(u2f((max_cy + 1u) * cpy), sh) - 1e-3f, 1.0f);
    F3 c0, c1;
    const ClipDir pd = clip_dir(w.p0, w.p1);  // shared by every coarse tile's clip
    if (!clip_segment_pre(w.p0, pd, bmin, bmax, c0, c1)) return;
    float x0 = div_by(c0.x, cpx), y0 = div_by(c0.y, cpy), x1 = div_by(c1.x, cpx), y1 = div_by(c1.y, cpy);
    int32_t fx = iclamp(f2i(floorf(x0)), (int32_t)min_cx, (int32_t)max_cx);
    int32_t fy = iclamp(f2i(floorf(y0)), (int32_t)min_cy, (int32_t)max_cy);
    int32_t ex = iclamp(f2i(floorf(x1)), (int32_t)min_cx, (int32_t)max_cx);
    int32_t ey = iclamp(f2i(floorf(y1)), (int32_t)min_cy, (int32_t)max_cy);
    float dx = x1 - x0, dy = y1 - y0;
    int32_t sx = sgn_i32(dx), sy = sgn_i32(dy);
    float sdx = fabsf(dx) < 1e-6f ? 1e-6f : dx, sdy = fabsf(dy) < 1e-6f ? 1e-6f : dy;
    float ddx = fabsf(1.0f / sdx), ddy = fabsf(1.0f / sdy);
    float flx = floorf(x0), fly = floorf(y0);
    float tx = sx > 0 ? ((flx + 1.0f) - x0) / sdx : (flx - x0) / sdx;
    float ty = sy > 0 ? ((fly + 1.0f) - y0) / sdy : (fly - y0) / sdy;
    if (fabsf(dx) < 1e-6f) tx = 1e38f;
    if (fabsf(dy) < 1e-6f) ty = 1e38f;
    uint32_t safety = 0, max_steps = (max_cx - min_cx + 1u) + (max_cy - min_cy + 1u) + 2u;
    for (;;) {
        if (safety > max_steps) break;
        if (fx < (int32_t)min_cx || fx > (int32_t)max_cx || fy < (int32_t)min_cy || fy > (int32_t)max_cy) break;
        uint32_t local = (uint32_t)fy * d.coarse_tiles_x + (uint32_t)fx;
        if (local < d.coarse_depth_tile_count)
            walk_page(A, w.p0, pd, d, d.coarse_depth_tile_base + local, (uint32_t)fx, (uint32_t)fy, opq, sink);
        if (fx == ex && fy == ey) break;
        if (tx <= ty) { fx += sx; tx += ddx; } else { fy += sy; ty += ddy; }
        ++safety;
    }
}

// Canonical order of the references in a cell as one 64-bit key: projected
// depth key (z0_16 + z1_16, 17 bits) descending, then instance, then segment.
__device__ __forceinline__ unsigned long long ref_sort_key(uint32_t key17, uint32_t inst, uint32_t seg) {
    return ((unsigned long long)(0x1FFFFu - (key17 & 0x1FFFFu)) << 47) |
           ((unsigned long long)(inst & 0x7FFFu) << 32) | (unsigned long long)seg;
}

__device__ __forceinline__ bool visits_unused(const PrepassArgs& A) {
    return *((volatile uint32_t*)&A.counters->visit_overflow) != 0u;
}

// K7: page marks + visit records. Warps walk 32 tasks at a time; each task's
// first kVisitSlots visits go to shared memory, the warp reserves room for all
// its visits with one atomic, and a task with more visits walks again to write
// the rest. When the records do not fit (or slots exceed 24 bits) the pass
// still marks every page and raises visit_overflow, which hands count and fill
// to the walking kernels.
// kOpaque: the frame has opaque fine tiles (K0 ran); the variant without them
// carries no cull code. kTel: count page candidates for the telemetry.
template <bool kOpaque, bool kTel>
__global__ void __launch_bounds__(kVisitThreads, 4) k_visit(const FrameParams* __restrict__ Pp,
                                                            const InstanceView* __restrict__ inst, PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    const FrameParams& P = *Pp;
    __shared__ uint32_t s_buf[kVisitSlots * kVisitThreads];
    const uint32_t n = *((volatile uint32_t*)&A.counters->tasks);
    const uint32_t n_cap = min(n, P.task_capacity);
    const bool records = P.visit_records != 0u;
    const uint2* opq = kOpaque ? A.opaque_tiles : nullptr;
    if (!records && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&A.counters->visit_overflow, 1u);
    // Warps take 32 tasks at a time and reserve their records on their own,
    // so a warp never waits for the slowest walk of its block.
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp_id = (blockIdx.x * kVisitThreads + threadIdx.x) >> 5;
    const uint32_t warps = gridDim.x * (kVisitThreads / 32u);
    for (uint32_t k0 = warp_id * 32u; k0 < n_cap; k0 += warps * 32u) {
        const uint32_t k = k0 + lane;
        TaskWalk w;
        const bool ok = k < n_cap && task_walk(P, A, k, w);
        VisitSink<kTel> vs{A.page_table, s_buf + threadIdx.x, 0u, 0u, records, A.tel_slots};
        if (ok) {
            // The task's reference (make_fine_seg_ref, :1313-1327) as its sort
            // key and material, gathered later by k_sort_cells from these
            // compact arrays instead of from the task records.
            const InstanceView& in = inst[w.i];
            A.task_key[k] = ref_sort_key((w.depths & 0xFFFFu) + (w.depths >> 16u), w.i, w.seg);
            A.task_mat[k] = w.strand < in.n_meta ? in.meta[w.strand].material_idx : 0u;
            walk_task(P, A, w, opq, vs);
        }
        if (!records) continue;
        uint32_t incl = vs.n;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        uint32_t base = kInvalid;
        if (lane == 31u && total > 0u && !visits_unused(A)) {
            const unsigned long long b = atomicAdd(&A.counters->visits, (unsigned long long)total);
            if (b + total <= (unsigned long long)P.ref_capacity) base = (uint32_t)b;
            else atomicOr(&A.counters->visit_overflow, 1u);
        }
        base = __shfl_sync(0xFFFFFFFFu, base, 31);
        if (base != kInvalid && vs.n > 0u) {
            // Visit records are placed in reservation order; the count and fill
            // passes and the cell sort make the references independent of it.
            const uint32_t at = base + incl - vs.n;
            const uint32_t nb = min(vs.n, kVisitSlots);
            // Streaming stores: the records are read once, by the count pass.
            for (uint32_t j = 0; j < nb; ++j) {
                __stcs(A.visit_rec + at + j, s_buf[j * kVisitThreads + threadIdx.x]);
                __stcs(A.visit_task + at + j, k);
            }
            if (vs.n > kVisitSlots) {
                SpillSink sp{A.visit_rec, A.visit_task, at, k, vs.n, 0u, 0u};
                walk_task(P, A, w, opq, sp);
            }
        }
    }
}

// K9 over visit records: cell counts by atomics; each visit keeps its rank.
__global__ void __launch_bounds__(256) k_count_visits(PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    if (visits_unused(A)) return;
    const uint32_t n = (uint32_t)*((volatile unsigned long long*)&A.counters->visits);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t rec = A.visit_rec[r];
        const uint32_t h = A.page_table[rec >> 8];
        uint32_t g = kInvalid, rank = 0u;
        if (h != 0u && h != kMarked) {
            g = (h - 1u) * kPageSize + (rec & 0xFFu);
            rank = atomicAdd(A.counts + g, 1u);
        }
        A.visit_rec[r] = g;
        A.visit_rank[r] = rank;
    }
}

// K11 over visit records: the visit's slot is page base + cell offset + rank.
// The fill scatters only the binning task index (4 B, into ref_keys, which a
// frame's L2 holds); k_sort_cells gathers each cell's tasks, builds the
// references (make_fine_seg_ref, :1313-1327) and writes them in canonical
// order, contiguously.
__global__ void __launch_bounds__(256) k_fill_visits(PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    if (visits_unused(A)) return;
    const uint32_t n = (uint32_t)*((volatile unsigned long long*)&A.counters->visits);
    // The visit records stream through once (evict-first loads), so L2 keeps
    // the scattered task-index lines until their sectors are complete.
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t g = __ldcs(A.visit_rec + r);
        if (g == kInvalid) continue;
        const fiber_fine_page_meta pm = A.page_meta[g / kPageSize];
        if (pm.seg_ref_count == 0u) continue;
        const uint64_t dst = (uint64_t)pm.seg_ref_base + A.offsets[g] + __ldcs(A.visit_rank + r);
        if (dst >= (uint64_t)pm.seg_ref_base + pm.seg_ref_count) continue;
        A.ref_keys[dst] = __ldcs(A.visit_task + r);
    }
}

// K9 / K11 walking form, for frames whose visit records did not fit.
template <int PASS, bool kOpaque>
__global__ void __launch_bounds__(256) k_traverse(const FrameParams* __restrict__ Pp,
                                                  const InstanceView* __restrict__ inst, PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    if (!visits_unused(A)) return;
    const FrameParams& P = *Pp;
    const uint32_t n = *((volatile uint32_t*)&A.counters->tasks);
    const uint32_t n_cap = min(n, P.task_capacity);
    const uint2* opq = kOpaque ? A.opaque_tiles : nullptr;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_cap; k += gridDim.x * blockDim.x) {
        TaskWalk w;
        if (!task_walk(P, A, k, w)) continue;
        if (PASS == kCount) {
            CountSink cs{A.page_table, A.counts, 0u};
            walk_task(P, A, w, opq, cs);
        } else {
            FillSink fs{&A, 0u, 0u, 0u, k};
            walk_task(P, A, w, opq, fs);
        }
    }
}

// ===========================================================================
// K8: allocate marked pages in page-table order.
// ===========================================================================
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;

__global__ void __launch_bounds__(kScanThreads) k_alloc_pages(const FrameParams* __restrict__ Pp, PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    const FrameParams& P = *Pp;
    __shared__ uint32_t s_tile, s_base;
    __shared__ uint32_t s_warp[33];
    const uint32_t n = P.total_coarse_tiles * kDepthSlices;
    const uint32_t per_tile = kScanThreads * kScanItems;
    const uint32_t n_tiles = ceil_div(n, per_tile);
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(A.tile_counter, 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= n_tiles) break;
        const uint32_t e0 = tile * per_tile + threadIdx.x * kScanItems;
        uint32_t flags[kScanItems], cnt = 0;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            flags[j] = (e0 + j < n && A.page_table[e0 + j] == kMarked) ? 1u : 0u;
            cnt += flags[j];
        }
        uint32_t total;
        uint32_t excl = block_exclusive_scan<kScanThreads>(cnt, s_warp, total);
        if (threadIdx.x < 32u) {
            uint32_t base = lb_exclusive_warp(A.lb_status, tile, P.epoch, total, &A.counters->error, lb_limit(P),
                                              lb_withheld(P, kStageAlloc));
            if (threadIdx.x == 0) {
                s_base = base;
                if (tile == n_tiles - 1u) A.counters->pages = min(base + total, P.page_capacity);
            }
        }
        __syncthreads();
        uint32_t idx = s_base + excl;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            if (!flags[j]) continue;
            uint32_t pti = e0 + j;
            if (idx >= P.page_capacity) {
                A.page_table[pti] = 0u;
                atomicOr(&A.counters->overflow, 2u);
            } else {
                A.page_meta[idx] = fiber_fine_page_meta{0u, 0u, 0u, 0u, pti / kDepthSlices, pti % kDepthSlices, 0u, 0u};
                A.page_table[pti] = idx + 1u;
            }
            ++idx;
        }
        __syncthreads();
    }
}

__global__ void k_zero_pages(PrepassArgs A) {
    const uint32_t pages = *((volatile uint32_t*)&A.counters->pages);
    const uint32_t n = pages * (kPageSize / 4u);
    uint4* c = reinterpret_cast<uint4*>(A.counts);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        c[k] = make_uint4(0u, 0u, 0u, 0u);
    if (A.page_nvis)
        for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < pages; k += gridDim.x * blockDim.x)
            A.page_nvis[k] = 0u;
}

// ===========================================================================
// K10: per page exclusive scan of the 256 cell counts; page ref bases from a
// look-back over pages (page order); active fine-tile flags.
// ===========================================================================

// The page's cell offsets (this thread's cell count c in, its exclusive offset
// out), the page's reference base from a look-back over pages in page order,
// its metadata and overflow flag (s_flags) and base (s_pbase). Ends with a
// block barrier.
__device__ __forceinline__ uint32_t page_prefix(const FrameParams& P, const PrepassArgs& A, uint32_t page,
                                                uint32_t pages, uint32_t c, uint32_t* s_warp, uint32_t& s_flags,
                                                uint32_t& s_pbase) {
    const size_t g = (size_t)page * kPageSize + threadIdx.x;
    uint32_t total;
    const uint32_t excl = block_exclusive_scan<256>(c, s_warp, total);
    A.offsets[g] = excl;
    A.cursors[g] = 0u;
    uint32_t base = 0u;
    if (threadIdx.x < 32u) base = lb_exclusive_warp(A.lb_status, page, P.epoch, total, &A.counters->error, lb_limit(P),
                                              lb_withheld(P, kStagePrefix));
    if (threadIdx.x == 0) {
        fiber_fine_page_meta pm = A.page_meta[page];
        uint32_t flags = 0u;
        if (total > 0u && (uint64_t)base + total > (uint64_t)P.ref_capacity) {
            flags = 1u;
            atomicOr(&A.counters->overflow, 4u);
        }
        pm.seg_ref_base = total > 0u ? base : 0u;
        pm.seg_ref_count = flags ? 0u : total;
        pm.flags = flags;
        A.page_meta[page] = pm;
        s_flags = flags;
        s_pbase = base;
        if (page == pages - 1u) A.counters->refs = base + total;
    }
    __syncthreads();
    return excl;
}

// append_active_fine_tile (:2207-2238) for a page: each of its 16 fine tiles
// with a non-empty cell that lies on screen.
__device__ __forceinline__ void page_active_tiles(const FrameParams& P, const PrepassArgs& A, uint32_t page,
                                                  const uint32_t* s_counts) {
    if (threadIdx.x >= 16u) return;
    const uint32_t lt = threadIdx.x;
    bool has = false;
    for (uint32_t z = 0; z < kDepthSlices; ++z) has = has || s_counts[z * 16u + lt] > 0u;
    if (!has) return;
    fiber_fine_page_meta pm = A.page_meta[page];
    uint32_t f = frustum_for_tile(P, pm.coarse_tile_id);
    if (f == kInvalid) return;
    const fiber_frustum_desc& d = P.frusta[f];
    uint32_t lc = pm.coarse_tile_id - d.coarse_depth_tile_base;
    uint32_t fx = (lc % d.coarse_tiles_x) * kCoarseExtent + lt % kCoarseExtent;
    uint32_t fy = (lc / d.coarse_tiles_x) * kCoarseExtent + lt / kCoarseExtent;
    if (fx < ceil_div(d.screen_width, d.froxel_size_x) && fy < ceil_div(d.screen_height, d.froxel_size_y))
        A.active_flags[(size_t)pm.coarse_tile_id * 16u + lt] = 1u;
}

// csr: a page-CSR frame, where k_build_pages does this work unless the visit
// records went unused. One warp per page, claimed in page order: lane l holds
// cells 8 l .. 8 l + 7 (one fine depth slice, fine tiles 8 (l & 1) .. + 7), so
// a warp scan gives the cell offsets and the look-back the page base, with no
// block barrier.
__global__ void __launch_bounds__(256) k_prefix_pages(const FrameParams* __restrict__ Pp, PrepassArgs A, bool csr) {
    if (frame_failed(A.counters)) return;
    if (csr && !visits_unused(A)) return;
    const FrameParams& P = *Pp;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t pages = *((volatile uint32_t*)&A.counters->pages);
    for (;;) {
        uint32_t page = 0u;
        if (lane == 0u) page = atomicAdd(A.tile_counter, 1u);
        page = __shfl_sync(0xFFFFFFFFu, page, 0);
        if (page >= pages) break;
        const size_t g0 = (size_t)page * kPageSize + lane * 8u;
        const uint4 ca = *reinterpret_cast<const uint4*>(A.counts + g0);
        const uint4 cb = *reinterpret_cast<const uint4*>(A.counts + g0 + 4u);
        const uint32_t c[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
        uint32_t e[8], sum = 0u, nsmall = 0u, nmid = 0u, nlarge = 0u, nz = 0u;
#pragma unroll
        for (uint32_t k = 0; k < 8u; ++k) {
            e[k] = sum;
            sum += c[k];
            nsmall += (c[k] >= 1u && c[k] <= kThreadSortMax) ? 1u : 0u;
            nmid += (c[k] > kThreadSortMax && c[k] <= kGroupSortMax) ? 1u : 0u;
            nlarge += c[k] > kGroupSortMax ? 1u : 0u;
            nz |= (c[k] > 0u ? 1u : 0u) << k;
        }
        // One scan carries the reference count (exclusive per cell) and, packed
        // 10 bits each, the small / mid / large cell counts for the lists.
        const uint32_t mine = nsmall | (nmid << 10) | (nlarge << 20);
        uint32_t x = sum, y = mine;
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t xa = __shfl_up_sync(0xFFFFFFFFu, x, o), ya = __shfl_up_sync(0xFFFFFFFFu, y, o);
            if (lane >= o) { x += xa; y += ya; }
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, x, 31), both = __shfl_sync(0xFFFFFFFFu, y, 31);
        const uint32_t lane_base = x - sum, list_base = y - mine;
#pragma unroll
        for (uint32_t k = 0; k < 8u; ++k) e[k] += lane_base;
        *reinterpret_cast<uint4*>(A.offsets + g0) = make_uint4(e[0], e[1], e[2], e[3]);
        *reinterpret_cast<uint4*>(A.offsets + g0 + 4u) = make_uint4(e[4], e[5], e[6], e[7]);
        *reinterpret_cast<uint4*>(A.cursors + g0) = make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(A.cursors + g0 + 4u) = make_uint4(0u, 0u, 0u, 0u);
        const uint32_t base = lb_exclusive_warp(A.lb_status, page, P.epoch, total, &A.counters->error, lb_limit(P),
                                              lb_withheld(P, kStagePrefix));
        uint32_t flags = 0u, tile = 0u;
        if (lane == 0u) {
            fiber_fine_page_meta pm = A.page_meta[page];
            if (total > 0u && (uint64_t)base + total > (uint64_t)P.ref_capacity) {
                flags = 1u;
                atomicOr(&A.counters->overflow, 4u);
            }
            pm.seg_ref_base = total > 0u ? base : 0u;
            pm.seg_ref_count = flags ? 0u : total;
            pm.flags = flags;
            A.page_meta[page] = pm;
            tile = pm.coarse_tile_id;
            if (page == pages - 1u) A.counters->refs = base + total;
        }
        flags = __shfl_sync(0xFFFFFFFFu, flags, 0);
        // A page that lost its references lists no cells and no active tiles.
        if (flags != 0u) continue;
        // The page's non-empty cells for k_sort_cells: up to 8 references in the
        // small list, more in the large one, in cell order.
        uint32_t s_small = 0u, s_mid = 0u, s_large = 0u;
        if (lane == 0u) {
            const uint32_t ns = both & 0x3FFu, nm = (both >> 10) & 0x3FFu, nl = both >> 20;
            s_small = ns ? atomicAdd(&A.counters->small_cells, ns) : 0u;
            s_mid = nm ? atomicAdd(&A.counters->mid_cells, nm) : 0u;
            s_large = nl ? atomicAdd(&A.counters->large_cells, nl) : 0u;
        }
        uint32_t ks = __shfl_sync(0xFFFFFFFFu, s_small, 0) + (list_base & 0x3FFu);
        uint32_t km = __shfl_sync(0xFFFFFFFFu, s_mid, 0) + ((list_base >> 10) & 0x3FFu);
        uint32_t kl = __shfl_sync(0xFFFFFFFFu, s_large, 0) + (list_base >> 20);
#pragma unroll
        for (uint32_t k = 0; k < 8u; ++k) {
            if (c[k] >= 1u && c[k] <= kThreadSortMax) A.cells_small[ks++] = make_uint2(base + e[k], c[k]);
            else if (c[k] > kThreadSortMax && c[k] <= kGroupSortMax) A.cells_mid[km++] = make_uint2(base + e[k], c[k]);
            else if (c[k] > kGroupSortMax) A.cells_large[kl++] = make_uint2(base + e[k], c[k]);
        }
        // append_active_fine_tile (:2207-2238): each of the page's 16 fine tiles
        // with a non-empty cell that lies on screen. Lanes of one parity hold
        // the same 8 fine tiles at the 16 depth slices.
        uint32_t m = nz;
#pragma unroll
        for (uint32_t o = 2; o < 32u; o <<= 1) m |= __shfl_xor_sync(0xFFFFFFFFu, m, o);
        tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
        const uint32_t lt = lane;
        const uint32_t has = __shfl_sync(0xFFFFFFFFu, m, (int)(lane >> 3) & 1);
        if (lt < 16u && ((has >> (lt & 7u)) & 1u)) {
            const uint32_t f = frustum_for_tile(P, tile);
            if (f != kInvalid) {
                const fiber_frustum_desc& d = P.frusta[f];
                const uint32_t lc = tile - d.coarse_depth_tile_base;
                const uint32_t fx = (lc % d.coarse_tiles_x) * kCoarseExtent + lt % kCoarseExtent;
                const uint32_t fy = (lc / d.coarse_tiles_x) * kCoarseExtent + lt / kCoarseExtent;
                if (fx < ceil_div(d.screen_width, d.froxel_size_x) && fy < ceil_div(d.screen_height, d.froxel_size_y))
                    A.active_flags[(size_t)tile * 16u + lt] = 1u;
            }
        }
    }
}

// ===========================================================================
// K13: ordered compaction of the active fine-tile flags.
// ===========================================================================
__global__ void __launch_bounds__(kScanThreads) k_compact_active(const FrameParams* __restrict__ Pp, PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    const FrameParams& P = *Pp;
    __shared__ uint32_t s_tile, s_base;
    __shared__ uint32_t s_warp[33];
    const uint32_t n = P.total_coarse_tiles * 16u;
    const uint32_t cam_end = P.camera_tile_end * 16u;
    const uint32_t per_tile = kScanThreads * kScanItems;
    const uint32_t n_tiles = ceil_div(n, per_tile);
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(A.tile_counter, 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= n_tiles) break;
        const uint32_t e0 = tile * per_tile + threadIdx.x * kScanItems;
        uint32_t flags[kScanItems], cnt = 0, cam = 0;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            flags[j] = (e0 + j < n && A.active_flags[e0 + j] != 0u) ? 1u : 0u;
            cnt += flags[j];
            cam += (flags[j] && e0 + j < cam_end) ? 1u : 0u;
        }
        uint32_t total;
        uint32_t excl = block_exclusive_scan<kScanThreads>(cnt, s_warp, total);
        for (int o = 16; o > 0; o >>= 1) cam += __shfl_xor_sync(0xFFFFFFFFu, cam, o);
        if ((threadIdx.x & 31) == 0 && cam) atomicAdd(&A.counters->camera_active, cam);
        if (threadIdx.x < 32u) {
            uint32_t base = lb_exclusive_warp(A.lb_status, tile, P.epoch, total, &A.counters->error, lb_limit(P),
                                              lb_withheld(P, kStageActive));
            if (threadIdx.x == 0) {
                s_base = base;
                if (tile == n_tiles - 1u) A.counters->active_tiles = base + total;
            }
        }
        __syncthreads();
        uint32_t idx = s_base + excl;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j)
            if (flags[j]) A.active_list[idx++] = e0 + j;
        __syncthreads();
    }
}

// ===========================================================================
// K14: emit raster work per active fine tile (256 lanes = 16 coarse z x 16
// fine z, near to far); work bases from a look-back over active tiles. The
// canonical order inside each cell (projected depth key descending, then
// instance, then segment) is made by k_sort_cells after the fill.
// ===========================================================================

// One warp sorts a cell of up to 32 * R references in registers: element
// e = lane * R + r, bitonic network over 32 R keys (padding sorts last).
// Strides below R compare registers of one lane; larger strides exchange the
// same register with lane ^ (stride / R).
// The reference of binning task k (make_fine_seg_ref, :1313-1327) as a sort
// key (depth key, instance, segment) and its material, as k_visit stored them
// (12 B per task, which a frame's L2 mostly holds).
// A cell entry: the task's canonical-order key and the task index; the sort
// moves the pair, and the store writes the reference (with the task's
// material), its depth key and its task.
__device__ __forceinline__ void task_entry(const PrepassArgs& A, const InstanceView* __restrict__ /*inst*/,
                                           uint32_t k, unsigned long long& key, uint32_t& task) {
    key = A.task_key[k];
    task = k;
}

__device__ __forceinline__ void store_entry(const PrepassArgs& A, uint32_t dst, unsigned long long key, uint32_t task) {
    A.refs[dst] = fiber_fine_seg_ref{(uint32_t)(key >> 32) & 0x7FFFu, (uint32_t)key, A.task_mat[task]};
    A.ref_keys[dst] = 0x1FFFFu - (uint32_t)(key >> 47);
    A.ref_task[dst] = task;
}

template <int R>
__device__ __forceinline__ void warp_sort_cell(const PrepassArgs& A, const InstanceView* __restrict__ inst,
                                               uint32_t base, uint32_t n, int lane) {
    unsigned long long k[R];
    uint32_t task[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t e = (uint32_t)lane * R + r;
        k[r] = ~0ull;
        task[r] = 0u;
        if (e < n) task_entry(A, inst, A.ref_keys[base + e], k[r], task[r]);
    }
#pragma unroll
    for (int size = 2; size <= 32 * R; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= R) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int e = lane * R + r;
                    unsigned long long ok = __shfl_xor_sync(0xFFFFFFFFu, k[r], stride / R);
                    uint32_t om = __shfl_xor_sync(0xFFFFFFFFu, task[r], stride / R);
                    const bool up = (e & size) == 0;
                    const bool lower = (e & stride) == 0;
                    const bool take_other = lower == up ? (ok < k[r]) : (ok > k[r]);
                    if (take_other) { k[r] = ok; task[r] = om; }
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int r2 = r ^ stride;
                    if (r2 > r) {
                        const int e = lane * R + r;
                        const bool up = (e & size) == 0;
                        if (up ? (k[r] > k[r2]) : (k[r] < k[r2])) {
                            unsigned long long tk = k[r]; k[r] = k[r2]; k[r2] = tk;
                            uint32_t tt = task[r]; task[r] = task[r2]; task[r2] = tt;
                        }
                    }
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t e = (uint32_t)lane * R + r;
        if (e < n) store_entry(A, base + e, k[r], task[r]);
    }
}


// A group of G lanes (G-aligned inside the warp) sorts one cell of up to
// G x R references: the bitonic network of warp_sort_cell over element
// e = (lane % G) R + r, shuffles exchanging only inside the group. Groups
// without a cell (n = 0) take part with padding. Every lane of the warp calls
// it.
template <int G, int R>
__device__ __forceinline__ void group_sort_cell(const PrepassArgs& A, const InstanceView* __restrict__ inst,
                                                uint32_t base, uint32_t n, int lane) {
    const int gl = lane & (G - 1);
    unsigned long long k[R];
    uint32_t task[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t e = (uint32_t)gl * R + r;
        k[r] = ~0ull;
        task[r] = 0u;
        if (e < n) task_entry(A, inst, A.ref_keys[base + e], k[r], task[r]);
    }
#pragma unroll
    for (int size = 2; size <= G * R; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= R) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int e = gl * R + r;
                    unsigned long long ok = __shfl_xor_sync(0xFFFFFFFFu, k[r], stride / R);
                    uint32_t om = __shfl_xor_sync(0xFFFFFFFFu, task[r], stride / R);
                    const bool up = (e & size) == 0;
                    const bool lower = (e & stride) == 0;
                    const bool take_other = lower == up ? (ok < k[r]) : (ok > k[r]);
                    if (take_other) { k[r] = ok; task[r] = om; }
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int r2 = r ^ stride;
                    if (r2 > r) {
                        const int e = gl * R + r;
                        const bool up = (e & size) == 0;
                        if (up ? (k[r] > k[r2]) : (k[r] < k[r2])) {
                            unsigned long long tk = k[r]; k[r] = k[r2]; k[r2] = tk;
                            uint32_t tt = task[r]; task[r] = task[r2]; task[r2] = tt;
                        }
                    }
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t e = (uint32_t)gl * R + r;
        if (e < n) store_entry(A, base + e, k[r], task[r]);
    }
}

__device__ __forceinline__ void warp_sort_any(const PrepassArgs& A, const InstanceView* __restrict__ inst,
                                              uint32_t base, uint32_t n, int lane) {
    if (n <= 32u) warp_sort_cell<1>(A, inst, base, n, lane);
    else if (n <= 64u) warp_sort_cell<2>(A, inst, base, n, lane);
    else if (n <= 128u) warp_sort_cell<4>(A, inst, base, n, lane);
    else warp_sort_cell<8>(A, inst, base, n, lane);
}

// Batcher's odd-even merge network for 8 (key, task) pairs in registers.
__device__ __forceinline__ void sort8(unsigned long long* k, uint32_t* task) {
    auto cas = [&](int a, int b) {
        if (k[a] > k[b]) {
            const unsigned long long tk = k[a]; k[a] = k[b]; k[b] = tk;
            const uint32_t tt = task[a]; task[a] = task[b]; task[b] = tt;
        }
    };
    cas(0, 1); cas(2, 3); cas(4, 5); cas(6, 7);
    cas(0, 2); cas(1, 3); cas(4, 6); cas(5, 7);
    cas(1, 2); cas(5, 6);
    cas(0, 4); cas(1, 5); cas(2, 6); cas(3, 7);
    cas(2, 4); cas(3, 5);
    cas(1, 2); cas(3, 4); cas(5, 6);
}

// One thread sorts a cell of at most 8 references in registers: Batcher's
// odd-even merge network for 8 inputs (19 comparators); padding sorts last.
__device__ __forceinline__ void thread_sort_cell(const PrepassArgs& A, const InstanceView* __restrict__ inst,
                                                 uint32_t base, uint32_t n) {
    unsigned long long k[8];
    uint32_t task[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        k[e] = ~0ull;
        task[e] = 0u;
        if ((uint32_t)e < n) task_entry(A, inst, A.ref_keys[base + e], k[e], task[e]);
    }
    sort8(k, task);
#pragma unroll
    for (int e = 0; e < 8; ++e)
        if ((uint32_t)e < n) store_entry(A, base + e, k[e], task[e]);
}

// One warp per active tile: the tile's 256 depth slots (16 coarse z x 16 fine
// z, near to far) are slots t = 8 lane .. 8 lane + 7, so each lane's slots
// share one coarse z (one page) and the warp scan keeps the slot order. Warps
// claim tiles and look back on their own; no block barrier is involved.
__global__ void __launch_bounds__(256) k_emit(const FrameParams* __restrict__ Pp, PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    const FrameParams& P = *Pp;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n_active = *((volatile uint32_t*)&A.counters->active_tiles);
    for (;;) {
        uint32_t a = 0u;
        if (lane == 0) a = atomicAdd(A.tile_counter, 1u);
        a = __shfl_sync(0xFFFFFFFFu, a, 0);
        if (a >= n_active) break;
        const uint32_t packed = A.active_list[a];
        const uint32_t lt = packed % 16u, tile = packed / 16u;
        const uint32_t f = frustum_for_tile(P, tile);
        const fiber_frustum_desc& d = P.frusta[f < P.F ? f : 0];
        const uint32_t lc = tile - d.coarse_depth_tile_base;
        const uint32_t lx = lt % kCoarseExtent, ly = lt / kCoarseExtent;
        const uint32_t fx = (lc % d.coarse_tiles_x) * kCoarseExtent + lx;
        const uint32_t fy = (lc / d.coarse_tiles_x) * kCoarseExtent + ly;
        const uint32_t screen_tile = fy * ceil_div(d.screen_width, d.froxel_size_x) + fx;
        const uint32_t dl0 = kPageSize - 1u - lane * 8u;  // depth slot of j = 0; slot j is dl0 - j
        const uint32_t cz = dl0 / kDepthSlices;
        const uint32_t pti = tile * kDepthSlices + cz;
        uint32_t page = kInvalid, pbase = 0u;
        bool ok = false;
        if (f != kInvalid) {
            const uint32_t handle = A.page_table[pti];
            if (handle != 0u && handle != kMarked) {
                page = handle - 1u;
                const fiber_fine_page_meta pm = A.page_meta[page];
                ok = pm.seg_ref_count > 0u && pm.flags == 0u;
                pbase = pm.seg_ref_base;
            }
        }
        uint32_t cnt[8];
        uint32_t nh = 0u, load = 0u;
#pragma unroll
        for (uint32_t j = 0; j < 8u; ++j) {
            const uint32_t fz = (dl0 - j) % kDepthSlices;
            const uint32_t cell = (fz * kCoarseExtent + ly) * kCoarseExtent + lx;
            cnt[j] = ok ? A.counts[(size_t)page * kPageSize + cell] : 0u;
            nh += cnt[j] > 0u ? 1u : 0u;
            load += cnt[j];
        }
        uint32_t x = nh;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        const uint32_t excl = x - nh;
        const uint32_t n_work = __shfl_sync(0xFFFFFFFFu, x, 31);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) load += __shfl_xor_sync(0xFFFFFFFFu, load, o);
        const uint32_t wb = lb_exclusive_warp(A.lb_status, a, P.epoch, n_work, &A.counters->error, lb_limit(P),
                                              lb_withheld(P, kStageEmit));
        if (lane == 0) {
            A.runs[a] = fiber_raster_tile_run{wb, n_work, f, screen_tile, load, 0u, 0u, 0u};
            if (a == n_active - 1u) A.counters->work_items = wb + n_work;
        }
        if (nh) {
            const fiber_coarse_depth_lut_entry lut = A.lut[pti];
            uint32_t dst = wb + excl;
#pragma unroll
            for (uint32_t j = 0; j < 8u; ++j) {
                if (cnt[j] == 0u) continue;
                const uint32_t fz = (dl0 - j) % kDepthSlices;
                const uint32_t cell = (fz * kCoarseExtent + ly) * kCoarseExtent + lx;
                const uint32_t dkey =
                    lut.virtual_count_q == 0u ? fz : lut.virtual_start_q + (lut.virtual_count_q * fz) / kDepthSlices;
                const uint32_t base = pbase + A.offsets[(size_t)page * kPageSize + cell];
                if (dst < P.work_capacity)
                    A.work[dst] = fiber_raster_work_item{base, cnt[j], f, screen_tile, dkey, cnt[j], page, cell};
                else
                    atomicOr(&A.counters->overflow, 8u);
                ++dst;
            }
        }
    }
}

// A cell longer than a warp sort: its warp writes the references in final
// form (unsorted) and queues the cell for k_sort_big_cells.
__device__ __forceinline__ void convert_big_cell(const PrepassArgs& A, const InstanceView* __restrict__ inst,
                                                 uint32_t b, uint32_t n, uint32_t lane) {
    for (uint32_t j = lane; j < n; j += 32u) {
        unsigned long long key;
        uint32_t task;
        task_entry(A, inst, A.ref_keys[b + j], key, task);
        store_entry(A, b + j, key, task);
    }
    if (lane == 0u) {
        const uint32_t slot = atomicAdd(&A.counters->big_cells, 1u);
        A.big_cells[slot] = make_uint2(b, n);
    }
}

// 32 consecutive small cells at once. k_prefix_pages lists a page's small
// cells together, in cell order, so their references usually form one span
// [lo, hi) of the reference array (holes: the page's larger cells). When the
// span fits kSortSpan, each lane loads the task index of every 32nd entry of
// the span (8 independent loads), gathers those tasks' keys and materials (16
// independent loads), and parks them in shared memory; each lane then sorts
// its own cell there with the network of thread_sort_cell and the warp writes
// the span's own entries back coalesced. Otherwise each lane sorts its cell
// alone.
constexpr uint32_t kSortSpan = 256;
constexpr uint32_t kSortPerLane = kSortSpan / 32u;
struct SortSpanSmem {
    unsigned long long key[kSortSpan];
    uint32_t task[kSortSpan];
    uint32_t mat[kSortSpan];
    uint8_t own[kSortSpan];
};

__device__ __forceinline__ void warp_sort_small_cells(const PrepassArgs& A, const InstanceView* __restrict__ inst,
                                                      uint32_t i0, uint32_t n_small, uint32_t lane,
                                                      SortSpanSmem& sm) {
    const uint32_t i = i0 + lane;
    const bool has = i < n_small;
    const uint2 e = has ? A.cells_small[i] : make_uint2(0u, 0u);
    uint32_t lo = has ? e.x : 0xFFFFFFFFu, hi = has ? e.x + e.y : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
    }
    if (hi <= lo || hi - lo > kSortSpan) {
        if (has) thread_sort_cell(A, inst, e.x, e.y);
        return;
    }
    const uint32_t span = hi - lo;
#pragma unroll
    for (uint32_t m = 0; m < kSortPerLane; ++m) sm.own[lane + 32u * m] = 0u;
    __syncwarp();
    if (has)
        for (uint32_t r = 0; r < e.y; ++r) sm.own[e.x - lo + r] = 1u;
    __syncwarp();
    uint32_t tk[kSortPerLane];
#pragma unroll
    for (uint32_t m = 0; m < kSortPerLane; ++m) {
        const uint32_t j = lane + 32u * m;
        tk[m] = (j < span && sm.own[j]) ? A.ref_keys[lo + j] : kInvalid;
    }
    unsigned long long kk[kSortPerLane];
    uint32_t mt[kSortPerLane];
#pragma unroll
    for (uint32_t m = 0; m < kSortPerLane; ++m) {
        kk[m] = tk[m] != kInvalid ? A.task_key[tk[m]] : ~0ull;
        mt[m] = tk[m] != kInvalid ? A.task_mat[tk[m]] : 0u;
    }
#pragma unroll
    for (uint32_t m = 0; m < kSortPerLane; ++m) {
        const uint32_t j = lane + 32u * m;
        sm.key[j] = kk[m];
        sm.task[j] = tk[m];
        sm.mat[j] = mt[m];
    }
    __syncwarp();
    if (has) {
        // Sort (key, position); the task and material follow their position.
        unsigned long long k[8];
        uint32_t pos[8];
        const uint32_t b = e.x - lo;
#pragma unroll
        for (uint32_t r = 0; r < 8u; ++r) {
            k[r] = r < e.y ? sm.key[b + r] : ~0ull;
            pos[r] = b + min(r, e.y - 1u);
        }
        sort8(k, pos);
        uint32_t t[8], mm[8];
#pragma unroll
        for (uint32_t r = 0; r < 8u; ++r) {
            t[r] = sm.task[pos[r]];
            mm[r] = sm.mat[pos[r]];
        }
#pragma unroll
        for (uint32_t r = 0; r < 8u; ++r)
            if (r < e.y) {
                sm.key[b + r] = k[r];
                sm.task[b + r] = t[r];
                sm.mat[b + r] = mm[r];
            }
    }
    __syncwarp();
#pragma unroll
    for (uint32_t m = 0; m < kSortPerLane; ++m) {
        const uint32_t j = lane + 32u * m;
        if (j < span && sm.own[j]) {
            const unsigned long long key = sm.key[j];
            A.refs[lo + j] = fiber_fine_seg_ref{(uint32_t)(key >> 32) & 0x7FFFu, (uint32_t)key, sm.mat[j]};
            A.ref_keys[lo + j] = 0x1FFFFu - (uint32_t)(key >> 47);
            A.ref_task[lo + j] = sm.task[j];
        }
    }
    __syncwarp();
}

// Canonical order inside every cell (projected depth key descending, then
// instance, then segment), after the fill, over the cell lists k_prefix_pages
// made: a warp per 32 cells of up to 8 references (a lane per cell), four
// cells of 9..32 references per warp (eight lanes each), then a warp per
// larger cell. A cell longer than a warp sort is converted in place by its
// warp and queued for k_sort_big_cells.
__global__ void __launch_bounds__(256, 5) k_sort_cells(const InstanceView* __restrict__ inst, PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    __shared__ SortSpanSmem s_span[8];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n_small = *((volatile uint32_t*)&A.counters->small_cells);
    const uint32_t n_large = *((volatile uint32_t*)&A.counters->large_cells);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; i0 < n_small; i0 += stride)
        warp_sort_small_cells(A, inst, i0, n_small, lane, s_span[threadIdx.x >> 5]);
    const uint32_t warps = stride >> 5;
    // Cells of 9..32 references: four per warp, eight lanes each.
    const uint32_t n_mid = *((volatile uint32_t*)&A.counters->mid_cells);
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 4u < n_mid; w += warps) {
        const uint32_t ci = w * 4u + (lane >> 3);
        const uint2 e = ci < n_mid ? A.cells_mid[ci] : make_uint2(0u, 0u);
        group_sort_cell<8, 4>(A, inst, e.x, e.y, (int)lane);
    }
    // Cells of more than 32: a warp per cell.
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n_large; w += warps) {
        const uint2 e = A.cells_large[w];
        const uint32_t b = e.x, n = e.y;
        if (n <= kWarpSortMax) {
            warp_sort_any(A, inst, b, n, (int)lane);
        } else {
            convert_big_cell(A, inst, b, n, lane);
        }
    }
}

// ===========================================================================
// Page-CSR backend (FineBinningBackend::PageCsr: prefix_page_candidates,
// scatter_page_candidates and build_fine_pages_csr, strand_prepass.wgsl:
// 1992-2049, 2387-2507). The reference lists each page's candidate tasks and
// traces every task again inside the page's workgroup; here the visit
// records of k_visit already hold every (page, cell, task) visit, so they are
// grouped by page (count, scan, scatter) and one block per page counts its
// cells in shared memory, takes the page's reference base in page order (as
// k_prefix_pages), fills the page's slots and sorts its cells while they are
// in L2. The results are the canonical ones of the default backend.
// ===========================================================================

// Visits per page; each visit keeps its rank inside its page. Lanes of a warp
// that hit the same page share one atomic.
__global__ void __launch_bounds__(256) k_page_count(PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    if (visits_unused(A)) return;
    const uint32_t n = (uint32_t)*((volatile unsigned long long*)&A.counters->visits);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t r0 = blockIdx.x * blockDim.x; r0 < n; r0 += gridDim.x * blockDim.x) {
        const uint32_t r = r0 + threadIdx.x;
        uint32_t page = kInvalid, cell = 0u;
        if (r < n) {
            const uint32_t rec = A.visit_rec[r];
            const uint32_t h = A.page_table[rec >> 8];
            if (h != 0u && h != kMarked) {
                page = h - 1u;
                cell = rec & 0xFFu;
            }
        }
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, page);
        const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
        uint32_t base = 0u;
        if (page != kInvalid && lane == leader) base = atomicAdd(A.page_nvis + page, (uint32_t)__popc(peers));
        base = __shfl_sync(0xFFFFFFFFu, base, (int)leader);
        if (r < n) {
            A.visit_rec[r] = page == kInvalid ? kInvalid : (page << 8) | cell;
            A.visit_rank[r] = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
        }
    }
}

// Exclusive scan of the per-page visit counts (one block).
__global__ void __launch_bounds__(1024) k_page_scan(PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    if (visits_unused(A)) return;
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_carry;
    const uint32_t pages = *((volatile uint32_t*)&A.counters->pages);
    if (threadIdx.x == 0) s_carry = 0u;
    __syncthreads();
    for (uint32_t b = 0; b < pages; b += 1024u) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < pages ? A.page_nvis[i] : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan<1024>(v, s_warp, total);
        if (i < pages) A.page_vbase[i] = s_carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) s_carry += total;
        __syncthreads();
    }
}

// Visits into their page's bucket: (task, cell) at page base + rank.
__global__ void __launch_bounds__(256) k_page_scatter(PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    if (visits_unused(A)) return;
    const uint32_t n = (uint32_t)*((volatile unsigned long long*)&A.counters->visits);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t rec = A.visit_rec[r];
        if (rec == kInvalid) continue;
        A.page_bucket[A.page_vbase[rec >> 8] + A.visit_rank[r]] = make_uint2(A.visit_task[r], rec & 0xFFu);
    }
}

// One block per page, in page order (the look-back of the page bases).
__global__ void __launch_bounds__(256) k_build_pages(const FrameParams* __restrict__ Pp,
                                                     const InstanceView* __restrict__ inst, PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    if (visits_unused(A)) return;
    const FrameParams& P = *Pp;
    __shared__ uint32_t s_tile, s_flags, s_pbase, s_nlarge;
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_counts[kPageSize], s_off[kPageSize], s_cur[kPageSize];
    __shared__ uint16_t s_large[kPageSize];
    const uint32_t pages = *((volatile uint32_t*)&A.counters->pages);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) {
            s_tile = atomicAdd(A.tile_counter, 1u);
            s_nlarge = 0u;
        }
        s_counts[threadIdx.x] = 0u;
        s_cur[threadIdx.x] = 0u;
        __syncthreads();
        const uint32_t page = s_tile;
        if (page >= pages) break;
        const uint32_t n = A.page_nvis[page], vb = A.page_vbase[page];
        for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) atomicAdd(&s_counts[A.page_bucket[vb + e].y], 1u);
        __syncthreads();
        const uint32_t c = s_counts[threadIdx.x];
        A.counts[(size_t)page * kPageSize + threadIdx.x] = c;
        const uint32_t excl = page_prefix(P, A, page, pages, c, s_warp, s_flags, s_pbase);
        s_off[threadIdx.x] = excl;
        if (s_flags == 0u) {
            __syncthreads();
            const uint32_t pbase = s_pbase;
            // Fill: the task index of every visit into its slot (the slots of
            // one page are a few KB, so these writes and the sort's reads stay
            // in L2); the order inside a cell is fixed by the sort below.
            for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) {
                const uint2 v = A.page_bucket[vb + e];
                A.ref_keys[pbase + s_off[v.y] + atomicAdd(&s_cur[v.y], 1u)] = v.x;
            }
            __syncthreads();
            if (c >= 1u && c <= kThreadSortMax) thread_sort_cell(A, inst, pbase + excl, c);
            else if (c > kThreadSortMax) s_large[atomicAdd(&s_nlarge, 1u)] = (uint16_t)threadIdx.x;
            __syncthreads();
            const uint32_t nl = s_nlarge;
            for (uint32_t i = warp; i < nl; i += blockDim.x >> 5) {
                const uint32_t cell = s_large[i], cb = pbase + s_off[cell], cn = s_counts[cell];
                if (cn <= kWarpSortMax) warp_sort_any(A, inst, cb, cn, (int)lane);
                else convert_big_cell(A, inst, cb, cn, lane);
            }
            page_active_tiles(P, A, page, s_counts);
        }
        __syncthreads();
    }
}

// Large cells: one block per cell. Bitonic sort in the ascending-only form
// (each stage starts with a "flip" compare i <-> i ^ (size - 1)), which never
// moves the virtual +inf padding below n, so the padding needs no storage.
// Up to kBigSmem entries sort in shared memory; longer cells sort in place in
// global memory with the same network.
constexpr uint32_t kBigSmem = 8192;
constexpr size_t kBigSmemBytes = kBigSmem * (sizeof(unsigned long long) + sizeof(uint32_t));

__device__ __forceinline__ void big_load(const PrepassArgs& A, uint32_t base, uint32_t n, uint32_t i,
                                         unsigned long long& k, uint32_t& m) {
    if (i < n) {
        fiber_fine_seg_ref r = A.refs[base + i];
        k = ref_sort_key(A.ref_keys[base + i], r.inst_id, r.seg_id);
        m = A.ref_task[base + i];
    } else {
        k = ~0ull;
        m = 0u;
    }
}
__device__ __forceinline__ void big_store(const PrepassArgs& A, uint32_t base, uint32_t i, unsigned long long k,
                                          uint32_t m) {
    A.refs[base + i] = fiber_fine_seg_ref{(uint32_t)(k >> 32) & 0x7FFFu, (uint32_t)k, A.task_mat[m]};
    A.ref_keys[base + i] = 0x1FFFFu - (uint32_t)(k >> 47);
    A.ref_task[base + i] = m;
}
// Pair t of a stage: (i, j) with i < j.
__device__ __forceinline__ void bitonic_pair(uint32_t t, uint32_t size, uint32_t stride, bool flip, uint32_t& i,
                                             uint32_t& j) {
    if (flip) {
        uint32_t half = size >> 1, blk = t / half, off = t % half;
        i = blk * size + off;
        j = blk * size + size - 1u - off;
    } else {
        i = (t / stride) * 2u * stride + (t % stride);
        j = i + stride;
    }
}

__global__ void __launch_bounds__(256) k_sort_big_cells(PrepassArgs A) {
    if (frame_failed(A.counters)) return;
    extern __shared__ unsigned char s_raw[];
    unsigned long long* s_k = reinterpret_cast<unsigned long long*>(s_raw);
    uint32_t* s_m = reinterpret_cast<uint32_t*>(s_raw + kBigSmem * sizeof(unsigned long long));
    const uint32_t n_cells = *((volatile uint32_t*)&A.counters->big_cells);
    for (uint32_t c = blockIdx.x; c < n_cells; c += gridDim.x) {
        const uint2 bc = A.big_cells[c];
        const uint32_t base = bc.x, n = bc.y;
        uint32_t np = 1;
        while (np < n) np <<= 1;
        const bool in_smem = np <= kBigSmem;
        if (in_smem) {
            for (uint32_t i = threadIdx.x; i < np; i += blockDim.x) big_load(A, base, n, i, s_k[i], s_m[i]);
            __syncthreads();
        }
        for (uint32_t size = 2; size <= np; size <<= 1) {
            for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
                const bool flip = stride == (size >> 1);
                for (uint32_t t = threadIdx.x; t < np / 2u; t += blockDim.x) {
                    uint32_t i, j;
                    bitonic_pair(t, size, stride, flip, i, j);
                    if (in_smem) {
                        unsigned long long ki = s_k[i], kj = s_k[j];
                        if (ki > kj) {
                            s_k[i] = kj; s_k[j] = ki;
                            uint32_t tm = s_m[i]; s_m[i] = s_m[j]; s_m[j] = tm;
                        }
                    } else if (j < n) {
                        unsigned long long ki, kj;
                        uint32_t mi, mj;
                        big_load(A, base, n, i, ki, mi);
                        big_load(A, base, n, j, kj, mj);
                        if (ki > kj) {
                            big_store(A, base, i, kj, mj);
                            big_store(A, base, j, ki, mi);
                        }
                    }
                }
                __syncthreads();
            }
        }
        if (in_smem) {
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) big_store(A, base, i, s_k[i], s_m[i]);
            __syncthreads();
        }
    }
}

// finalize_telemetry (:2145-2188): totals, per-page candidate statistics and
// the per-frustum page, reference and raster-run sums, after the emit. The
// candidate count of a page is the number of tasks that marked its slot.
__global__ void __launch_bounds__(256) k_telemetry(const FrameParams* __restrict__ Pp, PrepassArgs A) {
    const FrameParams& P = *Pp;
    uint32_t* tel = A.tel;
    const uint32_t pages = min(*((volatile uint32_t*)&A.counters->pages), P.page_capacity);
    const uint32_t runs = *((volatile uint32_t*)&A.counters->active_tiles);
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (t0 == 0) {
        tel[0] = pages;
        tel[1] = *((volatile uint32_t*)&A.counters->tasks);
        tel[3] = *((volatile uint32_t*)&A.counters->refs);
        tel[6] = P.F;
        for (uint32_t f = 0; f < P.F && f < FIBER_TELEMETRY_MAX_FRUSTA; ++f) {
            const uint32_t a = A.counters->frustum_task_base[f], b = A.counters->frustum_task_base[f + 1];
            *tel_frustum(tel, f, kTelEmittedSegments) = b - a;
        }
    }
    for (uint32_t p = t0; p < pages; p += stride) {
        const fiber_fine_page_meta pm = A.page_meta[p];
        const uint32_t f = frustum_for_tile(P, pm.coarse_tile_id);
        if (f != kInvalid) atomicAdd(tel_frustum(tel, f, kTelAllocatedPages), 1u);
        const uint32_t cand = A.tel_slots[pm.coarse_tile_id * kDepthSlices + pm.coarse_z];
        if (cand == 0u) continue;
        atomicAdd(tel + 2, cand);
        atomicAdd(tel + 4, 1u);
        atomicMax(tel + 5, cand);
        atomicAdd(tel + kTelHistogram + min(31u - (uint32_t)__clz(cand), 31u), 1u);
        if (f != kInvalid) {
            atomicAdd(tel_frustum(tel, f, kTelPageCandidates), cand);
            atomicAdd(tel_frustum(tel, f, kTelFineRefs), pm.seg_ref_count);
            atomicMax(tel_frustum(tel, f, kTelMaxPageCandidates), cand);
        }
    }
    // FRUSTUM_TELEMETRY_RASTER_* (:2830-2832): every tile run with work.
    for (uint32_t r = t0; r < runs; r += stride) {
        const fiber_raster_tile_run run = A.runs[r];
        if (run.work_count == 0u || run.frustum_id >= P.F) continue;
        atomicAdd(tel_frustum(tel, run.frustum_id, kTelRasterRuns), 1u);
        atomicAdd(tel_frustum(tel, run.frustum_id, kTelRasterLoad), run.load_score);
        atomicMax(tel_frustum(tel, run.frustum_id, kTelMaxRasterLoad), run.load_score);
    }
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
void launch_opaque(const LaunchCtx& L, const PrepassArgs& A, const float* depth, uint32_t pitch, uint32_t samples,
                   uint32_t tiles) {
    unsigned blocks = ceil_div_host(tiles, 8);
    if (blocks > (unsigned)L.sm_count * 16u) blocks = (unsigned)L.sm_count * 16u;
    if (blocks == 0u) blocks = 1u;
    k_opaque_reduce<<<blocks, 256, 0, L.stream>>>(L.P, A, depth, pitch, samples);
}
void launch_broad(const LaunchCtx& L, const PrepassArgs& A) {
    k_broad<<<ceil_div_host(L.I, 64), 64, 0, L.stream>>>(L.P, L.inst, A);
}
void launch_lut(const LaunchCtx& L, const PrepassArgs& A) {
    if (L.total_coarse_tiles) k_lut<<<ceil_div_host(L.total_coarse_tiles, 128), 128, 0, L.stream>>>(L.P, A);
}
void launch_fine(const LaunchCtx& L, const PrepassArgs& A) {
    k_fine<<<L.sm_count * 6, kFineThreads, 0, L.stream>>>(L.P, L.inst, A);
}
void launch_visit(const LaunchCtx& L, const PrepassArgs& A) {
    const unsigned grid = L.sm_count * 4;  // the resident blocks (4 per SM), each looping over warps of tasks
    if (L.telemetry) {
        if (L.opaque) k_visit<true, true><<<grid, kVisitThreads, 0, L.stream>>>(L.P, L.inst, A);
        else k_visit<false, true><<<grid, kVisitThreads, 0, L.stream>>>(L.P, L.inst, A);
    } else {
        if (L.opaque) k_visit<true, false><<<grid, kVisitThreads, 0, L.stream>>>(L.P, L.inst, A);
        else k_visit<false, false><<<grid, kVisitThreads, 0, L.stream>>>(L.P, L.inst, A);
    }
}
void launch_alloc(const LaunchCtx& L, const PrepassArgs& A) {
    k_alloc_pages<<<L.sm_count * 4, kScanThreads, 0, L.stream>>>(L.P, A);
}
void launch_zero_pages(const LaunchCtx& L, const PrepassArgs& A) {
    k_zero_pages<<<L.sm_count * 4, 256, 0, L.stream>>>(A);
}
void launch_count(const LaunchCtx& L, const PrepassArgs& A) {
    k_count_visits<<<L.sm_count * 8, 256, 0, L.stream>>>(A);
    if (L.opaque) k_traverse<kCount, true><<<L.sm_count * 8, 256, 0, L.stream>>>(L.P, L.inst, A);
    else k_traverse<kCount, false><<<L.sm_count * 8, 256, 0, L.stream>>>(L.P, L.inst, A);
}
void launch_prefix(const LaunchCtx& L, const PrepassArgs& A, bool csr) {
    k_prefix_pages<<<L.sm_count * 6, 256, 0, L.stream>>>(L.P, A, csr);
}
void launch_page_csr_count(const LaunchCtx& L, const PrepassArgs& A) {
    k_page_count<<<L.sm_count * 8, 256, 0, L.stream>>>(A);
    if (L.opaque) k_traverse<kCount, true><<<L.sm_count * 8, 256, 0, L.stream>>>(L.P, L.inst, A);
    else k_traverse<kCount, false><<<L.sm_count * 8, 256, 0, L.stream>>>(L.P, L.inst, A);
    k_page_scan<<<1, 1024, 0, L.stream>>>(A);
    k_page_scatter<<<L.sm_count * 8, 256, 0, L.stream>>>(A);
}
void launch_build_pages(const LaunchCtx& L, const PrepassArgs& A) {
    k_build_pages<<<L.sm_count * 6, 256, 0, L.stream>>>(L.P, L.inst, A);
}
void launch_fill_walk(const LaunchCtx& L, const PrepassArgs& A) {
    if (L.opaque) k_traverse<kFill, true><<<L.sm_count * 8, 256, 0, L.stream>>>(L.P, L.inst, A);
    else k_traverse<kFill, false><<<L.sm_count * 8, 256, 0, L.stream>>>(L.P, L.inst, A);
}
void launch_fill(const LaunchCtx& L, const PrepassArgs& A) {
    k_fill_visits<<<L.sm_count * 8, 256, 0, L.stream>>>(A);
    if (L.opaque) k_traverse<kFill, true><<<L.sm_count * 8, 256, 0, L.stream>>>(L.P, L.inst, A);
    else k_traverse<kFill, false><<<L.sm_count * 8, 256, 0, L.stream>>>(L.P, L.inst, A);
}
void launch_compact_active(const LaunchCtx& L, const PrepassArgs& A) {
    k_compact_active<<<L.sm_count * 4, kScanThreads, 0, L.stream>>>(L.P, A);
}
void launch_emit(const LaunchCtx& L, const PrepassArgs& A) {
    k_emit<<<L.sm_count * 6, 256, 0, L.stream>>>(L.P, A);
}
void launch_sort_cells(const LaunchCtx& L, const PrepassArgs& A) {
    k_sort_cells<<<L.sm_count * 5, 256, 0, L.stream>>>(L.inst, A);  // the resident blocks (5 per SM)
}
void launch_telemetry(const LaunchCtx& L, const PrepassArgs& A) {
    k_telemetry<<<L.sm_count * 2, 256, 0, L.stream>>>(L.P, A);
}
void launch_sort_big(const LaunchCtx& L, const PrepassArgs& A) {
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !configured[dev]) {
        cudaFuncSetAttribute(k_sort_big_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBigSmemBytes);
        if (dev >= 0 && dev < 64) configured[dev] = true;
    }
    k_sort_big_cells<<<L.sm_count * 2, 256, kBigSmemBytes, L.stream>>>(A);
}

}  // namespace fiber
