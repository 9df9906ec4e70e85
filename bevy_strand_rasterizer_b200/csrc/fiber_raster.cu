// fiber_raster.cu — the deep-opacity shadow raster (with the shadow-map
// stampback fused into its epilogue) and the camera colour raster:
// strand_rasterizer.wgsl:391-711 (SHADOWS) and :855-1044 (LINEAR),
// shadow_dom_stampback.wgsl:74-123.
//
// One 64-thread block per tile run, one thread per pixel slot (the reference's
// 64 slots; its 4 depth workers per pixel become the order in which one
// thread applies the same operations). Blocks claim runs from a counter. The
// run's references are staged into shared memory a round at a time
// (per-reference projection, radii, shading texels, by asynchronous copies);
// a round holds whole work items, or one CAP-sized chunk of an item longer
// than CAP (CAP is a multiple of 16, so the reference's groups of 4 never
// straddle a round). Each round also builds per-pixel coverage-candidate bits
// from a conservative band test, and each pixel walks only its candidates,
// two at a time. Block barriers happen only between rounds. The blend order is the reference's: work items near to far,
// references in groups of 4 from each item's start, (w0 over w1) over (w2 over
// w3), early out after each item once alpha > 0.98.
#include "fiber_kernels.cuh"

namespace fiber {

constexpr uint32_t kMaxRunItems = 256;  // 16 coarse z x 16 fine z cells per fine tile

struct RoundPlan {
    uint32_t lo, hi;     // work items [lo, hi) of the run in this round
    uint32_t off;        // first reference of item lo covered by the round
    uint32_t n;          // staged references
    uint32_t completes;  // the round ends item hi - 1
};

// Thread 0: plans the next round from (cur_item, cur_off); writes the staged
// prefix of each item of the round into s_prefix.
__device__ __forceinline__ RoundPlan plan_round(const uint32_t* s_wcount, uint32_t n_items, uint32_t cap,
                                                uint32_t& cur_item, uint32_t& cur_off, uint32_t* s_prefix) {
    RoundPlan rp;
    rp.lo = cur_item;
    rp.off = cur_off;
    const uint32_t c = s_wcount[cur_item];
    if (cur_off > 0u || c > cap) {
        const uint32_t n = min(cap, c - cur_off);
        s_prefix[0] = 0u;
        s_prefix[1] = n;
        rp.hi = cur_item + 1u;
        rp.n = n;
        cur_off += n;
        rp.completes = cur_off == c ? 1u : 0u;
        if (cur_off == c) { ++cur_item; cur_off = 0u; }
    } else {
        uint32_t total = 0u, k = 0u;
        while (cur_item < n_items && total + s_wcount[cur_item] <= cap) {
            s_prefix[k++] = total;
            total += s_wcount[cur_item];
            ++cur_item;
        }
        s_prefix[k] = total;
        rp.hi = cur_item;
        rp.n = total;
        rp.completes = 1u;
    }
    return rp;
}

// Staged slot s -> (item, reference offset inside the item).
__device__ __forceinline__ void slot_source(const uint32_t* s_prefix, const RoundPlan& rp, uint32_t s, uint32_t& item,
                                            uint32_t& j) {
    uint32_t lo = 0u, hi = rp.hi - rp.lo;  // last k with s_prefix[k] <= s
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (s_prefix[mid] <= s) lo = mid; else hi = mid;
    }
    item = rp.lo + lo;
    j = (lo == 0u ? rp.off : 0u) + (s - s_prefix[lo]);
}

// ===========================================================================
// K16 deep-opacity shadow raster + K17 stampback.
//
// One 64-thread block per shadow tile run, one thread per pixel. The pixel's
// thread walks its coverage candidates in entry order: pass 1 finds the
// nearest covered depth, pass 2 accumulates the opacity of every covered
// entry into the partial of the reference's depth worker that owns the entry
// (worker w takes entries w, w+4, ... from each item's start), so each
// worker's partial sees its entries in the reference's order; the four
// partials combine in worker order as the reference does.
// ===========================================================================
constexpr uint32_t kShadowThreads = 64;  // = kPixelSlots
constexpr uint32_t kShadowCap = 128;
constexpr uint32_t kShadowWords = kShadowCap / 32;
constexpr int kMaxDomSlices = 16;

size_t shadow_smem_bytes(uint32_t K) {
    return (size_t)kShadowCap * (2 * sizeof(float4) + 3 * sizeof(float)) + (size_t)kShadowThreads * 4u * K * sizeof(float);
}

// Asynchronous global -> shared copies (cp.async): a thread's copies land
// without holding registers; cp_async_wait_all waits for the thread's own.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Coverage candidates. The exact test below covers pixel p (cov > 0) only if
// p lies within the radius bound rb = rmin + (rmax - rmin) clamp(max z) of the
// segment's line and between the normals through its end points (t in [0, 1]).
// The band is widened by 1e-4 rb + 1e-6 rmax + 0.01 px + 1e-5 of the largest
// coordinate magnitude, hundreds of float ulps beyond the rounding of the
// exact test and of this one, so every pixel the band rejects is one the exact
// test leaves uncovered. Comparisons are written so that NaN never rejects;
// a segment shorter than 1e-6 px is a candidate of every pixel (the exact
// test decides), which keeps the per-pixel test free of branches.
struct Band {
    float nx, ny, c;    // d = n . p - c
    float ux, uy, cu;   // s = u . p - cu
    float thr, slo, shi;
};

__device__ __forceinline__ Band make_band(float ax, float ay, float bx, float by, float z0, float z1, float rmin,
                                          float rmax, float tile_max) {
    Band B;
    const float X = fmaxf(fmaxf(fmaxf(fabsf(ax), fabsf(ay)), fmaxf(fabsf(bx), fabsf(by))), tile_max);
    const float rb = rmin + (rmax - rmin) * wclamp(fmaxf(z0, z1), 0.0f, 1.0f);
    const float slack = 0.01f + 1e-5f * X;
    B.thr = rb * 1.0001f + 1e-6f * rmax + slack;
    const float abx = bx - ax, aby = by - ay;
    const float l2 = abx * abx + aby * aby;
    const float len = sqrtf(l2);
    B.ux = abx / len;
    B.uy = aby / len;
    B.nx = -B.uy;
    B.ny = B.ux;
    B.c = __fmaf_rn(B.nx, ax, B.ny * ay);
    B.cu = __fmaf_rn(B.ux, ax, B.uy * ay);
    B.slo = -slack;
    B.shi = len + slack;
    if (!(l2 > 1e-12f)) {  // degenerate (or NaN): d = s = 0 within unbounded limits
        const float inf = __int_as_float(0x7f800000);
        B.nx = B.ny = B.c = B.ux = B.uy = B.cu = 0.0f;
        B.thr = inf;
        B.slo = -inf;
        B.shi = inf;
    }
    return B;
}

// 32 x 32 bit transpose across the warp: lane i holds row i on entry, lane p
// holds column p on return (bit i = bit p of lane i's row). Each stage swaps
// one bit of the lane index with the same bit of the bit position.
template <uint32_t J, uint32_t M>
__device__ __forceinline__ uint32_t transpose_stage(uint32_t x, uint32_t lane) {
    const uint32_t y = __shfl_xor_sync(0xFFFFFFFFu, x, J);
    return (lane & J) ? ((x & ~M) | ((y >> J) & M)) : ((x & M) | ((y & M) << J));
}
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, uint32_t lane) {
    x = transpose_stage<16u, 0x0000FFFFu>(x, lane);
    x = transpose_stage<8u, 0x00FF00FFu>(x, lane);
    x = transpose_stage<4u, 0x0F0F0F0Fu>(x, lane);
    x = transpose_stage<2u, 0x33333333u>(x, lane);
    return transpose_stage<1u, 0x55555555u>(x, lane);
}

// The columns of the tile where a linear function f = f00 + g i + h j (i the
// column, j the row) lies in [lo, hi] are, on row j, the interval
// [L + G j, H + G j] with G = -h / g. `line_columns` sets L, H, G once per
// entry; `row_columns` evaluates one row. A slope |g| <= 1e-20 makes the test
// the same for the whole row (flat): the row is in or out as a whole. The
// interval ends are widened by 1e-3 column; their rounding (a few ulps of
// (|f00| + |lo| + |hi| + 8 |h|) / |g|) stays far inside the band's own slack
// (0.01 px + 1e-5 of the largest coordinate, divided by |g| in columns), so
// the set stays a superset of the pixels the exact tests can cover.
struct RowLine {
    float L, H, G;
    bool flat;
};

__device__ __forceinline__ RowLine line_columns(float f00, float g, float h, float lo, float hi) {
    RowLine r;
    r.flat = !(fabsf(g) > 1e-20f);
    if (!r.flat) {
        const float inv = 1.0f / g;
        const float e0 = (lo - f00) * inv, e1 = (hi - f00) * inv;
        r.L = fminf(e0, e1) - 1e-3f;
        r.H = fmaxf(e0, e1) + 1e-3f;
        r.G = -h * inv;
    } else {
        r.L = r.H = r.G = 0.0f;
    }
    return r;
}

__device__ __forceinline__ void row_columns(const RowLine& r, float f00, float h, float lo, float hi, float jf,
                                            float& ilo, float& ihi) {
    if (!r.flat) {
        ilo = __fmaf_rn(r.G, jf, r.L);
        ihi = __fmaf_rn(r.G, jf, r.H);
    } else {
        const float f = __fmaf_rn(h, jf, f00);
        const bool in = !(f < lo) && !(f > hi);
        ilo = in ? -1.0f : 1.0f;
        ihi = in ? 1e30f : -1.0f;
    }
}

// Candidate bits of one 32-entry word: lane = entry (valid if v), against the
// tile's pixel slots p = j fsx + i (p < 64), pixel centres (x0 + i, y0 + j).
// Per pixel row the band is an interval of columns: |d| <= thr gives one
// through the normal distance d, and slo <= s <= shi another through the
// distance s along u; their intersection sets the row's bits. The 64-bit
// per-entry masks are then transposed to per-pixel words, written to out[p].
// An entry with a non-finite band parameter (degenerate or NaN segments) is a
// candidate of every pixel; a NaN interval end drops that bound (fmaxf and
// fminf ignore NaN), which only widens the set.
__device__ __forceinline__ void candidate_word(const Band& B, bool v, float x0, float y0, uint32_t fsx, uint32_t fsy,
                                               uint32_t lane, uint32_t* out) {
    unsigned long long bits = 0ull;
    if (v) {
        const bool finite = isfinite(B.nx) && isfinite(B.ny) && isfinite(B.c) && isfinite(B.ux) && isfinite(B.uy) &&
                            isfinite(B.cu) && isfinite(B.thr) && isfinite(B.slo) && isfinite(B.shi);
        if (!finite) {
            bits = ~0ull;
        } else {
            const uint32_t cols = min(fsx, 64u);
            const uint32_t rows = min(fsy, (64u + fsx - 1u) / fsx);
            const float cmax = u2f(cols - 1u);
            const float d00 = __fmaf_rn(B.nx, x0, __fmaf_rn(B.ny, y0, -B.c));
            const float s00 = __fmaf_rn(B.ux, x0, __fmaf_rn(B.uy, y0, -B.cu));
            const RowLine rd = line_columns(d00, B.nx, B.ny, -B.thr, B.thr);
            const RowLine rs = line_columns(s00, B.ux, B.uy, B.slo, B.shi);
            for (uint32_t j = 0; j < rows; ++j) {
                const float jf = u2f(j);
                float dlo, dhi, slo, shi;
                row_columns(rd, d00, B.ny, -B.thr, B.thr, jf, dlo, dhi);
                row_columns(rs, s00, B.uy, B.slo, B.shi, jf, slo, shi);
                const float lo = fmaxf(ceilf(fmaxf(dlo, slo)), 0.0f);
                const float hi = fminf(floorf(fminf(dhi, shi)), cmax);
                if (lo <= hi) {
                    const uint32_t il = f2u(lo), ih = f2u(hi);
                    bits |= (((2ull << ih) - 1ull) & ~((1ull << il) - 1ull)) << (j * fsx);
                }
            }
        }
    }
    out[lane] = warp_transpose32((uint32_t)bits, lane);
    out[32u + lane] = warp_transpose32((uint32_t)(bits >> 32), lane);
}

__global__ void __launch_bounds__(kShadowThreads, 14) k_shadow(const FrameParams* __restrict__ Pp,
                                                           const InstanceView* __restrict__ inst, RenderArgs R) {
    if (frame_failed(R.counters)) return;
    const FrameParams& P = *Pp;
    extern __shared__ float4 s_dyn4[];
    // Per staged entry: the projected end points (x, y, normalised depth, w),
    // radii and opacity. The radius and opacity words first receive the
    // entry's task, instance and material index (the first copy level).
    float4* sa = s_dyn4;
    float4* sb = sa + kShadowCap;
    float* srmin = reinterpret_cast<float*>(sb + kShadowCap);
    float* srmax = srmin + kShadowCap;
    float* sabs = srmax + kShadowCap;
    uint32_t* s_task = reinterpret_cast<uint32_t*>(srmin);
    uint32_t* s_inst = reinterpret_cast<uint32_t*>(srmax);
    uint32_t* s_midx = reinterpret_cast<uint32_t*>(sabs);
    // [worker][K][pixel]: a warp's 32 pixels hit 32 banks whatever the slice.
    float* s_partial = sabs + kShadowCap;
    __shared__ uint32_t s_wbase[kMaxRunItems], s_wcount[kMaxRunItems], s_prefix[kMaxRunItems + 1];
    __shared__ uint32_t s_pmask[kShadowWords * kPixelSlots];  // [word][pixel] candidate bits
    __shared__ uint16_t s_item[kShadowCap];                   // run item << 2 | worker of each staged entry
    __shared__ RoundPlan s_plan;
    __shared__ uint32_t s_more, s_run;

    const uint32_t first = *((volatile uint32_t*)&R.counters->camera_active);
    const uint32_t last = *((volatile uint32_t*)&R.counters->active_tiles);
    const uint32_t K = P.K, D = P.dom_size, S = P.shadow_map_size;
    const uint32_t slot = threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    float* partial = s_partial + slot;  // partial[(w K + i) kShadowThreads]

    // Blocks claim runs from a counter, so long runs do not pile up on one block.
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_run = first + atomicAdd(&R.counters->tile_counter[kShadowRunCounter], 1u);
        __syncthreads();
        const uint32_t r = s_run;
        if (r >= last) break;
        const fiber_raster_tile_run run = R.runs[r];
        const uint32_t f = run.frustum_id;
        const uint32_t layer = light_layer(P, f);
        if (run.work_count == 0u || layer == kInvalid) continue;
        const uint32_t n_items = min(run.work_count, kMaxRunItems);
        const fiber_frustum_desc& d = P.frusta[f];
        const uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x);
        const uint32_t tx = run.screen_tile_id % ftx, ty = run.screen_tile_id / ftx;
        const uint32_t px = tx * d.froxel_size_x + slot % d.froxel_size_x;
        const uint32_t py = ty * d.froxel_size_y + slot / d.froxel_size_x;
        const bool active = slot < d.froxel_size_x * d.froxel_size_y && px < d.screen_width && py < d.screen_height;
        const float pfx = u2f(px) + 0.5f, pfy = u2f(py) + 0.5f;
        const float tile_max = fmaxf(u2f((tx + 1u) * d.froxel_size_x), u2f((ty + 1u) * d.froxel_size_y)) + 1.0f;
        for (uint32_t i = threadIdx.x; i < n_items; i += blockDim.x) {
            const fiber_raster_work_item wi = R.work[run.work_base + i];
            const bool valid_item = wi.frustum_id == f && wi.screen_tile_id == run.screen_tile_id;
            s_wbase[i] = wi.seg_ref_base;
            s_wcount[i] = valid_item ? wi.seg_ref_count : 0u;
        }
        const float x0 = u2f(tx * d.froxel_size_x) + 0.5f, y0 = u2f(ty * d.froxel_size_y) + 0.5f;
        __syncthreads();

        // Stage a round (projection, radii, run item and worker of each entry),
        // then build the candidate bits: warp per 32-entry word. The entries'
        // data arrive by asynchronous copies in two levels: the reference's
        // task, instance and material index, then the task's projected end
        // points (as k_fine projected them for this frustum:
        // world_to_screen_raw of the segment's vertices), so a round waits
        // for each level's latency once, whatever its entries.
        auto stage = [&](const RoundPlan& rp) {
            for (uint32_t s = threadIdx.x; s < rp.n; s += blockDim.x) {
                uint32_t item, j;
                slot_source(s_prefix, rp, s, item, j);
                const uint32_t g = s_wbase[item] + j;
                cp_async4(s_task + s, R.ref_task + g);
                cp_async4(s_inst + s, &R.refs[g].inst_id);
                cp_async4(s_midx + s, &R.refs[g].material_idx);
                s_item[s] = (uint16_t)((item << 2) | (j & 3u));
            }
            cp_async_wait_all();
            for (uint32_t s = threadIdx.x; s < rp.n; s += blockDim.x) {
                const size_t t = s_task[s];
                cp_async16(sa + s, R.task_proj + 2u * t);
                cp_async16(sb + s, R.task_proj + 2u * t + 1u);
                const fiber_strand_material& m = inst[s_inst[s]].materials[s_midx[s]];
                const float rmin = wmax(m.min_radius_pixels, 1e-4f);
                srmin[s] = rmin;
                srmax[s] = wmax(m.max_radius_pixels, rmin);
                sabs[s] = m.absorption_color[3];
            }
            cp_async_wait_all();
            for (uint32_t s = threadIdx.x; s < rp.n; s += blockDim.x) {
                sa[s].z = normalize_depth01(sa[s].z);
                sb[s].z = normalize_depth01(sb[s].z);
            }
            __syncthreads();
            const uint32_t nq = (rp.n + 31u) >> 5;
            for (uint32_t q = warp; q < nq; q += blockDim.x >> 5) {
                const uint32_t s = q * 32u + lane;
                const bool v = s < rp.n;
                const uint32_t e = v ? s : 0u;
                const float4 ea = sa[e], eb = sb[e];
                const Band B = make_band(ea.x, ea.y, eb.x, eb.y, ea.z, eb.z, srmin[e], srmax[e], tile_max);
                candidate_word(B, v, x0, y0, d.froxel_size_x, d.froxel_size_y, lane, s_pmask + q * kPixelSlots);
            }
        };

        // This pixel's candidates in entry order.
        auto next_candidate = [&](uint32_t nq, uint32_t& q, uint32_t& m) -> uint32_t {
            while (m == 0u && q < nq) {
                m = s_pmask[q * kPixelSlots + slot];
                ++q;
            }
            if (m == 0u) return kInvalid;
            const uint32_t bit = (uint32_t)(__ffs(m) - 1);
            m &= m - 1u;
            return (q - 1u) * 32u + bit;
        };

        // Exact coverage of staged entry bi at this pixel (0 when the pixel's
        // projection falls outside the segment) and the depth there.
        auto coverage = [&](uint32_t bi, float& qz) -> float {
            const float4 ea = sa[bi], eb = sb[bi];
            const float t = line_t(pfx, pfy, ea.x, ea.y, eb.x, eb.y);
            const float qx = wmix(ea.x, eb.x, t), qy = wmix(ea.y, eb.y, t);
            qz = wmix(ea.z, eb.z, t);
            const float rr = wmix(srmin[bi], srmax[bi], wclamp(qz, 0.0f, 1.0f));
            const float dx = pfx - qx, dy = pfy - qy;
            const float cov = wclamp(1.0f - sqrtf(dx * dx + dy * dy) / rr, 0.0f, 1.0f);
            return (t < 0.0f || t > 1.0f) ? 0.0f : cov;
        };

        // ---- Pass 1: nearest covered depth = max depth of the covered entries
        // of the first run item holding one; the walk stops once the next
        // candidate lies past that item. Candidates are taken two at a time:
        // both coverages are computed side by side, then applied in entry
        // order.
        uint32_t best = kInvalid;  // first item with a covered entry
        float z0 = -1.0f;          // its max covered depth
        bool complete = !active;   // the best item is fully processed
        uint32_t cur_item = 0u, cur_off = 0u;
        uint32_t rounds1 = 0u, item0 = 0u, off0 = 0u;  // pass 1's staged rounds; thread 0: the state after round 0
        bool single_round = false, staged_all = false;
        for (bool first_round = true;; first_round = false) {
            if (threadIdx.x == 0) {
                s_more = cur_item < n_items ? 1u : 0u;
                if (s_more) s_plan = plan_round(s_wcount, n_items, kShadowCap, cur_item, cur_off, s_prefix);
                if (first_round) {
                    s_more |= (cur_item >= n_items ? 2u : 0u);
                    item0 = cur_item;
                    off0 = cur_off;
                }
            }
            __syncthreads();
            const uint32_t more = s_more;
            if (!(more & 1u)) break;
            if (first_round) single_round = (more & 2u) != 0u;
            const RoundPlan rp = s_plan;
            stage(rp);
            __syncthreads();
            ++rounds1;
            staged_all = single_round;
            if (!complete) {
                const uint32_t nq = (rp.n + 31u) >> 5;
                uint32_t q = 0u, m = 0u;
                for (;;) {
                    const uint32_t b0 = next_candidate(nq, q, m);
                    if (b0 == kInvalid) break;
                    const uint32_t b1 = next_candidate(nq, q, m);
                    const bool two = b1 != kInvalid;
                    const uint32_t c1 = two ? b1 : b0;
                    const uint32_t item0 = (uint32_t)(s_item[b0] >> 2), item1 = (uint32_t)(s_item[c1] >> 2);
                    float qz0, qz1;
                    const float cov0 = coverage(b0, qz0);
                    const float cov1 = coverage(c1, qz1);
                    if (best != kInvalid && item0 > best) break;
                    if (cov0 > 0.0f) {
                        if (best == kInvalid) { best = item0; z0 = wmax(-1.0f, qz0); }
                        else z0 = wmax(z0, qz0);
                    }
                    if (!two || (best != kInvalid && item1 > best)) break;
                    if (cov1 > 0.0f) {
                        if (best == kInvalid) { best = item1; z0 = wmax(-1.0f, qz1); }
                        else z0 = wmax(z0, qz1);
                    }
                }
                complete = best != kInvalid && (best + 1u < rp.hi || rp.completes);
            }
            if (__syncthreads_and(complete)) break;
        }
        const bool found = active && best != kInvalid;

        // ---- Pass 2: opacity partials, each covered entry into its worker's.
        for (uint32_t i = 0; i < 4u * K; ++i) partial[i * kShadowThreads] = 0.0f;
        const float alpha_z0 = found ? z0 : 1.0f;
        const float inv_span = 1.0f / wmax(1e-6f, alpha_z0);
        if (__syncthreads_or(found)) {
            cur_item = 0u;
            cur_off = 0u;
            // Pass 1 that stopped after the first round leaves that round
            // staged: pass 2 starts on it and plans from the state after it.
            bool reuse = !staged_all && rounds1 == 1u;
            if (reuse) {
                cur_item = item0;
                cur_off = off0;
            }
            for (;;) {
                if (!staged_all && !reuse) {
                    if (threadIdx.x == 0) {
                        s_more = cur_item < n_items ? 1u : 0u;
                        if (s_more) s_plan = plan_round(s_wcount, n_items, kShadowCap, cur_item, cur_off, s_prefix);
                    }
                    __syncthreads();
                    if (!s_more) break;
                    stage(s_plan);
                    __syncthreads();
                }
                reuse = false;
                const RoundPlan rp = s_plan;
                if (found) {
                    const uint32_t nq = (rp.n + 31u) >> 5;
                    uint32_t q = 0u, m = 0u;
                    // Slice, weight and opacity of one covered entry; the
                    // deposits into the worker's partials keep entry order.
                    auto split = [&](uint32_t bi, float cov, float qz, float*& pw, float& wf, float& al, bool& next) {
                        const float dzp = wmax(0.0f, alpha_z0 - qz) * inv_span;
                        const float u = wclamp(dzp, 0.0f, 1.0f);  // pow(u, DOM_GAMMA = 1)
                        const float tl = u * u2f(K);
                        const uint32_t si = min(f2u(floorf(tl)), K - 1u);
                        wf = tl - floorf(tl);
                        al = cov * sabs[bi] * 0.5f;
                        pw = partial + ((uint32_t)(s_item[bi] & 3u) * K + si) * kShadowThreads;
                        next = si + 1u < K;
                    };
                    auto deposit = [&](float* pw, float wf, float al, bool next) {
                        const float a0 = pw[0];
                        pw[0] = wclamp(a0 + (1.0f - a0) * (1.0f - wf) * al, 0.0f, 1.0f);
                        if (next) {
                            const float a1 = pw[kShadowThreads];
                            pw[kShadowThreads] = wclamp(a1 + (1.0f - a1) * wf * al, 0.0f, 1.0f);
                        }
                    };
                    for (;;) {
                        const uint32_t b0 = next_candidate(nq, q, m);
                        if (b0 == kInvalid) break;
                        const uint32_t b1 = next_candidate(nq, q, m);
                        const bool two = b1 != kInvalid;
                        const uint32_t c1 = two ? b1 : b0;
                        float qz0, qz1;
                        const float cov0 = coverage(b0, qz0);
                        const float cov1 = coverage(c1, qz1);
                        float *pw0, *pw1, wf0, wf1, al0, al1;
                        bool n0, n1;
                        split(b0, cov0, qz0, pw0, wf0, al0, n0);
                        split(c1, cov1, qz1, pw1, wf1, al1, n1);
                        if (cov0 > 0.0f) deposit(pw0, wf0, al0, n0);
                        if (!two) break;
                        if (cov1 > 0.0f) deposit(pw1, wf1, al1, n1);
                    }
                }
                if (staged_all) break;
                __syncthreads();
            }
        }
        // ---- Combine the 4 workers per slice, write the DOM, stamp the shadow map.
        if (active) {
            // A texel of a page the sparse pool could not hold is not stored
            // (counted as a DOM pool overflow); the stampback still runs.
            // Dense layers index the texel directly; the sparse pool goes
            // through the page table (dom_texel).
            const bool dense = P.dom_pool_pages == 0u;
            float* dz = nullptr;
            float* dop = nullptr;
            size_t ds = 0;
            const size_t dom_px = (size_t)py * D + px;
            const bool stored = dense || dom_texel(P, R, layer, px, py, dz, dop, ds);
            if (!found) {
                if (dense) {
                    R.dom_depth[(size_t)layer * D * D + dom_px] = 0.0f;
                    for (uint32_t i = 0; i < K; ++i) R.dom_opacity[((size_t)layer * K + i) * D * D + dom_px] = 0.0f;
                } else if (stored) {
                    *dz = 0.0f;
                    for (uint32_t i = 0; i < K; ++i) dop[i * ds] = 0.0f;
                }
            } else {
                if (dense) R.dom_depth[(size_t)layer * D * D + dom_px] = z0;
                else if (stored) *dz = z0;
                float acc = 0.0f;
                for (uint32_t i = 0; i < K; ++i) {
                    float a = 0.0f;
                    for (uint32_t wk = 0; wk < 4u; ++wk) a = a + (1.0f - a) * partial[(wk * K + i) * kShadowThreads];
                    acc = acc + (1.0f - acc) * a;  // opaque_terminal_slice = K without an opaque depth
                    if (dense) R.dom_opacity[((size_t)layer * K + i) * D * D + dom_px] = acc;
                    else if (stored) dop[i * ds] = acc;
                }
                // Fused stampback: every target texel whose DOM footprint holds
                // this texel takes the max depth (the target starts cleared).
                if (z0 > 0.0f) {
                    uint32_t x_lo = (uint32_t)(((uint64_t)px * S) / D), y_lo = (uint32_t)(((uint64_t)py * S) / D);
                    x_lo = x_lo > 0u ? x_lo - 1u : 0u;
                    y_lo = y_lo > 0u ? y_lo - 1u : 0u;
                    for (uint32_t ty2 = y_lo; ty2 < S && ty2 <= y_lo + 2u + S / D; ++ty2) {
                        uint32_t mny = min((ty2 * D) / S, D - 1u), mxy = min(((ty2 + 1u) * D + S - 1u) / S, D);
                        if (py < mny || py >= mxy) continue;
                        for (uint32_t tx2 = x_lo; tx2 < S && tx2 <= x_lo + 2u + S / D; ++tx2) {
                            uint32_t mnx = min((tx2 * D) / S, D - 1u), mxx = min(((tx2 + 1u) * D + S - 1u) / S, D);
                            if (px < mnx || px >= mxx) continue;
                            atomicMax(reinterpret_cast<int*>(R.shadow_map + (size_t)layer * S * S + (size_t)ty2 * S + tx2),
                                      __float_as_int(z0));
                        }
                    }
                }
            }
        }
    }
}

// ===========================================================================
// Sparse DOM residency (the reference's bevy_vsms demand paging, replaced by
// a per-frame page pool). Every shadow tile run with work requests the DOM
// pages under its tile and their neighbours (request_shadow_dom_pages,
// strand_prepass.wgsl:2540-2579, DOM_PREFETCH_PAGE_BORDER = 1); requested
// pages take pool pages in page-table order (layer, row, column), as many as
// the pool holds; their depth planes are cleared (a texel without depth is
// empty whatever its opacity words hold).
// ===========================================================================
constexpr uint32_t kDomBorder = 1;

__global__ void __launch_bounds__(256) k_dom_request(const FrameParams* __restrict__ Pp, RenderArgs R) {
    if (frame_failed(R.counters)) return;
    const FrameParams& P = *Pp;
    const uint32_t first = *((volatile uint32_t*)&R.counters->camera_active);
    const uint32_t last = *((volatile uint32_t*)&R.counters->active_tiles);
    const uint32_t ppx = P.dom_pages_x;
    for (uint32_t r = first + blockIdx.x * blockDim.x + threadIdx.x; r < last; r += gridDim.x * blockDim.x) {
        const fiber_raster_tile_run run = R.runs[r];
        const uint32_t layer = light_layer(P, run.frustum_id);
        if (run.work_count == 0u || layer == kInvalid) continue;
        const fiber_frustum_desc& d = P.frusta[run.frustum_id];
        const uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x);
        const uint32_t x0 = (run.screen_tile_id % ftx) * d.froxel_size_x, y0 = (run.screen_tile_id / ftx) * d.froxel_size_y;
        const uint32_t x1 = min(x0 + d.froxel_size_x - 1u, d.screen_width - 1u);
        const uint32_t y1 = min(y0 + d.froxel_size_y - 1u, d.screen_height - 1u);
        const uint32_t pmx0 = x0 / kDomPage, pmy0 = y0 / kDomPage;
        const uint32_t px0 = pmx0 - min(pmx0, kDomBorder), py0 = pmy0 - min(pmy0, kDomBorder);
        const uint32_t px1 = min(x1 / kDomPage + kDomBorder, ppx - 1u), py1 = min(y1 / kDomPage + kDomBorder, ppx - 1u);
        for (uint32_t py = py0; py <= py1; ++py)
            for (uint32_t px = px0; px <= px1; ++px) R.dom_page_table[((size_t)layer * ppx + py) * ppx + px] = kMarked;
    }
}

// One block: requested entries, in table order, get pool page index + 1.
__global__ void __launch_bounds__(1024) k_dom_alloc(const FrameParams* __restrict__ Pp, RenderArgs R, uint32_t entries) {
    if (frame_failed(R.counters)) return;
    const FrameParams& P = *Pp;
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_carry;
    if (threadIdx.x == 0) s_carry = 0u;
    __syncthreads();
    for (uint32_t b = 0; b < entries; b += 1024u) {
        const uint32_t i = b + threadIdx.x;
        const bool req = i < entries && R.dom_page_table[i] == kMarked;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan<1024>(req ? 1u : 0u, s_warp, total);
        if (req) {
            const uint32_t idx = s_carry + ex;
            R.dom_page_table[i] = idx < P.dom_pool_pages ? idx + 1u : 0u;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        R.counters->dom_pages = s_carry;
        if (s_carry > P.dom_pool_pages) atomicOr(&R.counters->overflow, 16u);
    }
}

__global__ void __launch_bounds__(256) k_dom_clear(const FrameParams* __restrict__ Pp, RenderArgs R) {
    const FrameParams& P = *Pp;
    const uint32_t pages = min(*((volatile uint32_t*)&R.counters->dom_pages), P.dom_pool_pages);
    const size_t per_page = kDomPageTexels / 4u, n = (size_t)pages * per_page;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        float* page = R.dom_pool + (k / per_page) * kDomPageTexels * (P.K + 1u);
        reinterpret_cast<float4*>(page)[k % per_page] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

void launch_dom_paging(const LaunchCtx& L, const RenderArgs& R, uint32_t table_entries) {
    k_dom_request<<<L.sm_count * 2, 256, 0, L.stream>>>(L.P, R);
    k_dom_alloc<<<1, 1024, 0, L.stream>>>(L.P, R, table_entries);
    k_dom_clear<<<L.sm_count * 4, 256, 0, L.stream>>>(L.P, R);
}

// ===========================================================================
// K19 camera colour raster.
//
// One 64-thread block per camera tile run, one thread per pixel. Each pixel
// walks its candidate entries in order, one entry (two per step) at a time;
// an entry lands in its worker's part of its group of 4 (an item's entries
// 4g .. 4g+3 from the item start), and a group is blended when the walk
// reaches the next one, as the reference's four workers do: (w0 over w1) over
// (w2 over w3), then final over group, the same float operations in the same
// order, computed in one thread. A group without a candidate contributes
// transparent black and depth 0, which leaves the blend unchanged, so skipping
// it keeps the result.
// ===========================================================================
constexpr uint32_t kCamThreads = 64;  // = kPixelSlots
constexpr uint32_t kCamCap = 128;
constexpr uint32_t kCamWords = kCamCap / 32;
constexpr uint16_t kEntryInvalid = 0x8000u;

__global__ void __launch_bounds__(kCamThreads, 14) k_raster(const FrameParams* __restrict__ Pp,
                                                        const InstanceView* __restrict__ inst, RenderArgs R) {
    if (frame_failed(R.counters)) return;
    const FrameParams& P = *Pp;
    // Per staged entry: 68 B of projection (x, y, z, w of both end points),
    // radii and shading texels, the run item and position in it (bit 15:
    // behind the camera, never a candidate). The words of sinv, srmin, srmax
    // and svis first receive the reference's task, instance, segment and
    // material index (the first copy level); s_hist receives the history
    // texel pair (visibility, current).
    __shared__ float4 sa[kCamCap], sb[kCamCap];
    __shared__ float sinv[kCamCap], srmin[kCamCap], srmax[kCamCap], svis[kCamCap];
    __shared__ uint32_t s_hist[kCamCap];
    __shared__ uint2 ss0[kCamCap], ss1[kCamCap];
    __shared__ uint16_t s_item[kCamCap];
    __shared__ uint32_t s_pmask[kCamWords * kPixelSlots];  // [word][pixel] candidate bits
    __shared__ uint32_t s_wbase[kMaxRunItems], s_wcount[kMaxRunItems], s_prefix[kMaxRunItems + 1];
    __shared__ RoundPlan s_plan;
    __shared__ uint32_t s_more, s_run;

    const uint32_t n_runs = *((volatile uint32_t*)&R.counters->camera_active);
    const uint32_t slot = threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t cap = P.atlas_cap;
    const __half* hist = R.history[(P.hist_in & 1u) ^ 1u];
    // Blocks claim runs from a counter, so long runs do not pile up on one block.
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_run = atomicAdd(&R.counters->tile_counter[kCameraRunCounter], 1u);
        __syncthreads();
        const uint32_t r = s_run;
        if (r >= n_runs) break;
        const fiber_raster_tile_run run = R.runs[r];
        const uint32_t f = run.frustum_id;
        if (run.work_count == 0u || f >= P.camera_frustum_end) continue;
        const uint32_t n_items = min(run.work_count, kMaxRunItems);
        const fiber_frustum_desc& d = P.frusta[f];
        const uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x);
        const uint32_t tx = run.screen_tile_id % ftx, ty = run.screen_tile_id / ftx;
        const uint32_t px = tx * d.froxel_size_x + slot % d.froxel_size_x;
        const uint32_t py = ty * d.froxel_size_y + slot / d.froxel_size_x;
        const bool active = slot < d.froxel_size_x * d.froxel_size_y && px < d.screen_width && py < d.screen_height;
        const size_t pi = (size_t)P.out_base[f] + (size_t)py * d.screen_width + px;  // this pixel's output
        const float pcx = u2f(px) + 0.5f, pcy = u2f(py) + 0.5f;
        const float tile_max = fmaxf(u2f((tx + 1u) * d.froxel_size_x), u2f((ty + 1u) * d.froxel_size_y)) + 1.0f;
        for (uint32_t i = threadIdx.x; i < n_items; i += blockDim.x) {
            const fiber_raster_work_item wi = R.work[run.work_base + i];
            s_wbase[i] = wi.seg_ref_base;
            s_wcount[i] = wi.seg_ref_count;
        }
        const float x0 = u2f(tx * d.froxel_size_x) + 0.5f, y0 = u2f(ty * d.froxel_size_y) + 0.5f;
        __syncthreads();
        float4 fin = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float gdepth = 0.0f;
        bool done = !active;
        uint32_t frags = 0;
        uint32_t pending = kInvalid;  // last item blended into, whose end test is still due
        uint32_t cur_item = 0u, cur_off = 0u;
        // Early out (alpha > 0.98) at the end of an item.
        auto end_of_item = [&]() {
            if (!done && fin.w > 0.98f) {
                fin = make_float4(fin.x / fin.w, fin.y / fin.w, fin.z / fin.w, 1.0f);
                done = true;
            }
            pending = kInvalid;
        };
        for (;;) {
            if (threadIdx.x == 0) {
                s_more = cur_item < n_items ? 1u : 0u;
                if (s_more) s_plan = plan_round(s_wcount, n_items, kCamCap, cur_item, cur_off, s_prefix);
            }
            __syncthreads();
            if (!s_more) break;
            const RoundPlan rp = s_plan;
            // The entries arrive by asynchronous copies in two levels: the
            // reference (task, instance, segment, material index), then the
            // task's projected end points (as k_fine projected them for this
            // frustum) and the segment's shading and history texels.
            uint32_t* s_task = reinterpret_cast<uint32_t*>(sinv);
            uint32_t* s_inst = reinterpret_cast<uint32_t*>(srmin);
            uint32_t* s_seg = reinterpret_cast<uint32_t*>(srmax);
            uint32_t* s_midx = reinterpret_cast<uint32_t*>(svis);
            for (uint32_t s = threadIdx.x; s < rp.n; s += blockDim.x) {
                uint32_t item, j;
                slot_source(s_prefix, rp, s, item, j);
                const uint32_t g = s_wbase[item] + j;
                cp_async4(s_task + s, R.ref_task + g);
                cp_async4(s_inst + s, &R.refs[g].inst_id);
                cp_async4(s_seg + s, &R.refs[g].seg_id);
                cp_async4(s_midx + s, &R.refs[g].material_idx);
                s_item[s] = (uint16_t)((item << 2) | (j & 3u));
            }
            cp_async_wait_all();
            for (uint32_t s = threadIdx.x; s < rp.n; s += blockDim.x) {
                const size_t t = s_task[s];
                const uint32_t ii = s_inst[s], i0 = min(s_seg[s], cap - 1u), i1 = min(i0 + 1u, cap - 1u);
                const fiber_strand_material& m = inst[ii].materials[s_midx[s]];
                const size_t t0 = (size_t)ii * cap + i0, t1 = (size_t)ii * cap + i1;
                cp_async16(sa + s, R.task_proj + 2u * t);
                cp_async16(sb + s, R.task_proj + 2u * t + 1u);
                cp_async8(ss0 + s, R.atlas + t0 * 4);
                cp_async8(ss1 + s, R.atlas + t1 * 4);
                cp_async4(s_hist + s, hist + t0 * 2);
                // min_radius = max(rmin, 1e-4) and max(rmax, min_radius) are
                // idempotent on these values, so they are applied once here.
                const float rmin = wmax(m.min_radius_pixels, 1e-4f);
                srmin[s] = rmin;
                srmax[s] = wmax(m.max_radius_pixels, rmin);
            }
            cp_async_wait_all();
            for (uint32_t s = threadIdx.x; s < rp.n; s += blockDim.x) {
                const float4 a = sa[s], b = sb[s];
                if (!(a.x < 0.0f && b.x < 0.0f)) {
                    const float abx = b.x - a.x, aby = b.y - a.y;
                    sinv[s] = 1.0f / (abx * abx + aby * aby);
                    svis[s] = __low2float(*reinterpret_cast<const __half2*>(s_hist + s));
                } else {
                    s_item[s] |= kEntryInvalid;
                }
            }
            __syncthreads();
            // Candidate bits: warp per 32-entry word. The radius bound uses the
            // normalised depth the exact test clamps.
            const uint32_t nq = (rp.n + 31u) >> 5;
            for (uint32_t q = warp; q < nq; q += blockDim.x >> 5) {
                const uint32_t s = q * 32u + lane;
                const bool v = s < rp.n && !(s_item[s] & kEntryInvalid);
                const uint32_t e = v ? s : 0u;
                const float4 ea = sa[e], eb = sb[e];
                const Band B = make_band(ea.x, ea.y, eb.x, eb.y, normalize_depth01(ea.z), normalize_depth01(eb.z),
                                         srmin[e], srmax[e], tile_max);
                candidate_word(B, v, x0, y0, d.froxel_size_x, d.froxel_size_y, lane, s_pmask + q * kPixelSlots);
            }
            __syncthreads();
            // The walk takes one candidate entry per step, so every live lane
            // runs the coverage and shading arithmetic on each step; the
            // entry lands in its worker's part of the current group, and the
            // group is blended when the walk reaches the next group.
            uint32_t cur_lead = kInvalid;  // first entry of the group being gathered
            float4 g0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), g1 = g0, g2 = g0, g3 = g0;
            float e0 = 0.0f, e1 = 0.0f, e2 = 0.0f, e3 = 0.0f;
            // (w0 over w1) over (w2 over w3), depth max.
            auto flush_group = [&]() {
                if (cur_lead == kInvalid) return;
                fin = over(fin, over(over(g0, g1), over(g2, g3)));
                gdepth = wmax(gdepth, wmax(wmax(e0, e1), wmax(e2, e3)));
                g0 = g1 = g2 = g3 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                e0 = e1 = e2 = e3 = 0.0f;
                cur_lead = kInvalid;
            };
            // Candidates are taken two at a time: both entries' arithmetic
            // runs side by side, then they land in entry order.
            uint32_t q = 0u, m = 0u;
            auto next = [&]() -> uint32_t {
                while (m == 0u && q < nq) {
                    m = s_pmask[q * kPixelSlots + slot];
                    ++q;
                }
                if (m == 0u) return kInvalid;
                const uint32_t bit = (uint32_t)(__ffs(m) - 1);
                m &= m - 1u;
                return (q - 1u) * 32u + bit;
            };
            // Coverage and shaded, premultiplied colour of entry bi at this pixel.
            auto eval = [&](uint32_t bi, float4& v, float& pz) -> bool {
                const float4 ea = sa[bi], eb = sb[bi];
                const float ax = ea.x, ay = ea.y, bx = eb.x, by = eb.y;
                const float rmax = srmax[bi];
                const bool in_box = !((pcx < wmin(ax, bx) - rmax || pcy < wmin(ay, by) - rmax) ||
                                      (pcx > wmax(ax, bx) + rmax || pcy > wmax(ay, by) + rmax));
                const float abx = bx - ax, aby = by - ay;
                const float t = ((pcx - ax) * abx + (pcy - ay) * aby) * sinv[bi];
                const float fx = ax + abx * t, fy = ay + aby * t;
                pz = wmix(ea.z, eb.z, t);
                const float rr = wmix(srmin[bi], rmax, wclamp(normalize_depth01(pz), 0.0f, 1.0f));
                const float dx = pcx - fx, dy = pcy - fy;
                const float d2 = dx * dx + dy * dy;
                const float cov = wclamp(1.0f - sqrtf(d2) / rr, 0.0f, 1.0f);
                // perspective_correct_line_t (:149-154)
                const float aw0 = wmax(fabsf(ea.w), 1e-6f), aw1 = wmax(fabsf(eb.w), 1e-6f);
                const float tw = (t * aw0) / ((1.0f - t) * aw1 + t * aw0);
                const float4 c0 = load_half4(reinterpret_cast<const __half*>(&ss0[bi]));
                const float4 c1 = load_half4(reinterpret_cast<const __half*>(&ss1[bi]));
                const float sr = wmix(c0.x, c1.x, tw), sg = wmix(c0.y, c1.y, tw);
                const float sbl = wmix(c0.z, c1.z, tw), sa_ = wmix(c0.w, c1.w, tw);
                const float alpha = sa_ * cov;
                const float vsb = svis[bi];
                v = make_float4(sr * vsb * alpha, sg * vsb * alpha, sbl * vsb * alpha, alpha);
                return in_box && t >= 0.0f && t <= 1.0f && d2 < rr * rr;
            };
            // Entry bi into its worker's part of the current group; false once
            // the pixel is done (early out at the end of an item).
            auto land = [&](uint32_t bi, bool covered, const float4& v, float pz) -> bool {
                const uint32_t tag = s_item[bi];
                const uint32_t w = tag & 3u;
                const uint32_t lead = bi - w;
                if (lead != cur_lead) {
                    flush_group();
                    const uint32_t item = (tag >> 2) & 0x3FFu;
                    if (pending != kInvalid && item > pending) {
                        end_of_item();
                        if (done) return false;
                    }
                    cur_lead = lead;
                    pending = item;
                }
                if (covered) {
                    if (w == 0u) { g0 = v; e0 = pz; }
                    else if (w == 1u) { g1 = v; e1 = pz; }
                    else if (w == 2u) { g2 = v; e2 = pz; }
                    else { g3 = v; e3 = pz; }
                    ++frags;
                }
                return true;
            };
            while (!done) {
                const uint32_t b0 = next();
                if (b0 == kInvalid) break;
                const uint32_t b1 = next();
                const bool two = b1 != kInvalid;
                const uint32_t c1 = two ? b1 : b0;
                float4 v0, v1;
                float z0, z1;
                const bool h0 = eval(b0, v0, z0);
                const bool h1 = eval(c1, v1, z1);
                if (!land(b0, h0, v0, z0) || !two) break;
                if (!land(c1, h1, v1, z1)) break;
            }
            flush_group();
            // The last item blended into ends in this round unless the round
            // stops inside it.
            if (pending != kInvalid && (pending + 1u < rp.hi || rp.completes)) end_of_item();
            if (!__syncthreads_or(!done)) break;
        }
        if (active) {
            float4 o = fin;
            if (o.w > 1e-6f && o.w < 1.0f) o = make_float4(o.x / o.w, o.y / o.w, o.z / o.w, o.w);
            reinterpret_cast<uint2*>(R.color)[pi] = pack_half4(o.x, o.y, o.z, o.w);
            R.depth[pi] = gdepth;
            if (P.fragment_counts) R.fragments[pi] = frags;
        }
    }
}

void launch_shadow(const LaunchCtx& L, const RenderArgs& R, uint32_t K) {
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t max_bytes = shadow_smem_bytes(kMaxDomSlices);
    if (dev < 0 || dev >= 64 || !configured[dev]) {
        cudaFuncSetAttribute(k_shadow, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_bytes);
        if (dev >= 0 && dev < 64) configured[dev] = true;
    }
    k_shadow<<<L.sm_count * 16, kShadowThreads, shadow_smem_bytes(K), L.stream>>>(L.P, L.inst, R);
}

void launch_raster(const LaunchCtx& L, const RenderArgs& R) {
    k_raster<<<L.sm_count * 16, kCamThreads, 0, L.stream>>>(L.P, L.inst, R);
}

}  // namespace fiber
