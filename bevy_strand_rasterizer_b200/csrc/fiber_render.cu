// fiber_render.cu — deep shadow + stampback, shading, camera raster and
// composite: the reference's strand_shadow_rasterizer_pass
// (src/nodes/shadows.rs:29-221), strand_shading_pass (src/nodes/shading.rs:25-155),
// strand_rasterizer_pass (src/nodes/raster.rs:26-179) and composition_pass
// (src/nodes/composite.rs:19-131).
#include "fiber_kernels.cuh"

namespace fiber {

// ---------------------------------------------------------------------------
// Segment fetch (get_segment_vertices_from_index_unchecked,
// strand_rasterizer.wgsl:289-303): 128-bit vertex loads through the read-only
// path, world transform in the reference's evaluation order.
// ---------------------------------------------------------------------------
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

// ===========================================================================
// K16 deep-opacity shadow raster (strand_rasterizer.wgsl:391-711) with the
// stampback (shadow_dom_stampback.wgsl:74-123) fused into its epilogue.
// One block per shadow tile run: 64 pixel slots x 4 depth workers.
// ===========================================================================
constexpr int kShadowBatch = 256;
constexpr int kMaxDomSlices = 16;

__global__ void __launch_bounds__(256) k_shadow(const FrameParams* __restrict__ Pp,
                                                const InstanceView* __restrict__ inst, RenderArgs R) {
    const FrameParams& P = *Pp;
    __shared__ float s_p0x[kShadowBatch], s_p0y[kShadowBatch], s_p0z[kShadowBatch];
    __shared__ float s_p1x[kShadowBatch], s_p1y[kShadowBatch], s_p1z[kShadowBatch];
    __shared__ float s_rmin[kShadowBatch], s_rmax[kShadowBatch], s_abs[kShadowBatch];
    __shared__ uint32_t s_valid[kShadowBatch];
    __shared__ float s_partial[256 * kMaxDomSlices];
    const uint32_t first = *((volatile uint32_t*)&R.counters->camera_active);
    const uint32_t last = *((volatile uint32_t*)&R.counters->active_tiles);
    const uint32_t K = P.K, D = P.dom_size, S = P.shadow_map_size;
    const uint32_t slot = threadIdx.x >> 2, worker = threadIdx.x & 3u;
    for (uint32_t r = first + blockIdx.x; r < last; r += gridDim.x) {
        const fiber_raster_tile_run run = R.runs[r];
        if (run.work_count == 0u) continue;
        const uint32_t f = run.frustum_id;
        const uint32_t layer = light_layer(P, f);
        if (layer == kInvalid) continue;
        const fiber_frustum_desc& d = P.frusta[f];
        const float* clip = P.clip[f];
        const float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
        const uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x);
        const uint32_t tx = run.screen_tile_id % ftx, ty = run.screen_tile_id / ftx;
        const uint32_t px = tx * d.froxel_size_x + slot % d.froxel_size_x;
        const uint32_t py = ty * d.froxel_size_y + slot / d.froxel_size_x;
        const bool active = slot < d.froxel_size_x * d.froxel_size_y && px < d.screen_width && py < d.screen_height;
        const float pfx = u2f(px) + 0.5f, pfy = u2f(py) + 0.5f;
        // Pass 1: nearest covered depth, searched work item by work item until
        // the first item with a hit; the 4 workers split each batch and take
        // the max (exact, order independent).
        float z0 = -1.0f;
        bool found = false;
        for (uint32_t w = 0; w < run.work_count; ++w) {
            const fiber_raster_work_item wi = R.work[run.work_base + w];
            const bool valid_item = wi.frustum_id == f && wi.screen_tile_id == run.screen_tile_id;
            bool hit = false;
            float zi = -1.0f;
            for (uint32_t bb = 0; bb < wi.seg_ref_count; bb += kShadowBatch) {
                const uint32_t bc = min((uint32_t)kShadowBatch, wi.seg_ref_count - bb);
                __syncthreads();
                if (threadIdx.x < bc) {
                    uint32_t v = 0u;
                    if (valid_item) {
                        fiber_fine_seg_ref ref = R.refs[wi.seg_ref_base + bb + threadIdx.x];
                        const InstanceView& in = inst[ref.inst_id];
                        float4 w0, w1;
                        segment_world(in, ref.seg_id, w0, w1);
                        float4 a = world_to_screen_raw(w0, clip, vw, vh), b = world_to_screen_raw(w1, clip, vw, vh);
                        fiber_strand_material m = in.materials[ref.material_idx];
                        s_p0x[threadIdx.x] = a.x; s_p0y[threadIdx.x] = a.y; s_p0z[threadIdx.x] = normalize_depth01(a.z);
                        s_p1x[threadIdx.x] = b.x; s_p1y[threadIdx.x] = b.y; s_p1z[threadIdx.x] = normalize_depth01(b.z);
                        float rmin = wmax(m.min_radius_pixels, 1e-4f);
                        s_rmin[threadIdx.x] = rmin;
                        s_rmax[threadIdx.x] = wmax(m.max_radius_pixels, rmin);
                        s_abs[threadIdx.x] = m.absorption_color[3];
                        v = 1u;
                    }
                    s_valid[threadIdx.x] = v;
                }
                __syncthreads();
                if (active && !found) {
                    for (uint32_t bi = worker; bi < bc; bi += 4u) {
                        if (!s_valid[bi]) continue;
                        float t = line_t(pfx, pfy, s_p0x[bi], s_p0y[bi], s_p1x[bi], s_p1y[bi]);
                        if (t < 0.0f || t > 1.0f) continue;
                        float qx = wmix(s_p0x[bi], s_p1x[bi], t), qy = wmix(s_p0y[bi], s_p1y[bi], t);
                        float qz = wmix(s_p0z[bi], s_p1z[bi], t);
                        float rr = wmix(s_rmin[bi], s_rmax[bi], wclamp(qz, 0.0f, 1.0f));
                        float dx = pfx - qx, dy = pfy - qy;
                        float cov = wclamp(1.0f - sqrtf(dx * dx + dy * dy) / rr, 0.0f, 1.0f);
                        if (cov > 0.0f) { zi = wmax(zi, qz); hit = true; }
                    }
                }
            }
            // Combine the 4 workers of each pixel (adjacent lanes).
            float zm = zi;
            zm = wmax(zm, __shfl_xor_sync(0xFFFFFFFFu, zm, 1));
            zm = wmax(zm, __shfl_xor_sync(0xFFFFFFFFu, zm, 2));
            unsigned hm = __ballot_sync(0xFFFFFFFFu, hit);
            bool any_hit = ((hm >> (threadIdx.x & 28u)) & 0xFu) != 0u;
            if (active && !found && any_hit) {
                z0 = wmax(z0, zm);
                found = true;
            }
            if (__syncthreads_and(found || !active)) break;
        }
        const size_t dom_px = (size_t)py * D + px;
        float* partial = s_partial + threadIdx.x * kMaxDomSlices;
        for (uint32_t i = 0; i < K; ++i) partial[i] = 0.0f;
        // No opaque directional shadow map is bound on this path (opaque depth 0).
        const bool alpha_active = active && found;
        const float alpha_z0 = alpha_active ? z0 : 1.0f;
        const float inv_span = 1.0f / wmax(1e-6f, alpha_z0);
        const bool any_alpha = __syncthreads_or(alpha_active);
        // Pass 2: opacity partials; worker w takes entries w, w+4, ... of each item.
        for (uint32_t w = 0; any_alpha && w < run.work_count; ++w) {
            const fiber_raster_work_item wi = R.work[run.work_base + w];
            const bool valid_item = wi.frustum_id == f && wi.screen_tile_id == run.screen_tile_id;
            for (uint32_t bb = 0; bb < wi.seg_ref_count; bb += kShadowBatch) {
                const uint32_t bc = min((uint32_t)kShadowBatch, wi.seg_ref_count - bb);
                __syncthreads();
                if (threadIdx.x < bc) {
                    uint32_t v = 0u;
                    if (valid_item) {
                        fiber_fine_seg_ref ref = R.refs[wi.seg_ref_base + bb + threadIdx.x];
                        const InstanceView& in = inst[ref.inst_id];
                        float4 w0, w1;
                        segment_world(in, ref.seg_id, w0, w1);
                        float4 a = world_to_screen_raw(w0, clip, vw, vh), b = world_to_screen_raw(w1, clip, vw, vh);
                        fiber_strand_material m = in.materials[ref.material_idx];
                        s_p0x[threadIdx.x] = a.x; s_p0y[threadIdx.x] = a.y; s_p0z[threadIdx.x] = normalize_depth01(a.z);
                        s_p1x[threadIdx.x] = b.x; s_p1y[threadIdx.x] = b.y; s_p1z[threadIdx.x] = normalize_depth01(b.z);
                        float rmin = wmax(m.min_radius_pixels, 1e-4f);
                        s_rmin[threadIdx.x] = rmin;
                        s_rmax[threadIdx.x] = wmax(m.max_radius_pixels, rmin);
                        s_abs[threadIdx.x] = m.absorption_color[3];
                        v = 1u;
                    }
                    s_valid[threadIdx.x] = v;
                }
                __syncthreads();
                if (!alpha_active) continue;
                for (uint32_t bi = worker; bi < bc; bi += 4u) {
                    if (!s_valid[bi]) continue;
                    float t = line_t(pfx, pfy, s_p0x[bi], s_p0y[bi], s_p1x[bi], s_p1y[bi]);
                    if (t < 0.0f || t > 1.0f) continue;
                    float qx = wmix(s_p0x[bi], s_p1x[bi], t), qy = wmix(s_p0y[bi], s_p1y[bi], t);
                    float qz = wmix(s_p0z[bi], s_p1z[bi], t);
                    float rr = wmix(s_rmin[bi], s_rmax[bi], wclamp(qz, 0.0f, 1.0f));
                    float dx = pfx - qx, dy = pfy - qy;
                    float cov = wclamp(1.0f - sqrtf(dx * dx + dy * dy) / rr, 0.0f, 1.0f);
                    if (cov <= 0.0f) continue;
                    float dzp = wmax(0.0f, alpha_z0 - qz) * inv_span;
                    float u = wclamp(dzp, 0.0f, 1.0f);  // pow(u, DOM_GAMMA = 1)
                    float tl = u * u2f(K);
                    uint32_t si = min(f2u(floorf(tl)), K - 1u);
                    float wf = tl - floorf(tl);
                    float a = cov * s_abs[bi] * 0.5f;
                    float a0 = partial[si];
                    partial[si] = wclamp(a0 + (1.0f - a0) * (1.0f - wf) * a, 0.0f, 1.0f);
                    if (si + 1u < K) {
                        float a1 = partial[si + 1u];
                        partial[si + 1u] = wclamp(a1 + (1.0f - a1) * wf * a, 0.0f, 1.0f);
                    }
                }
            }
        }
        __syncthreads();
        if (worker == 0u && active) {
            if (!found) {
                R.dom_depth[(size_t)layer * D * D + dom_px] = 0.0f;
                for (uint32_t i = 0; i < K; ++i) R.dom_opacity[((size_t)layer * K + i) * D * D + dom_px] = 0.0f;
            } else {
                R.dom_depth[(size_t)layer * D * D + dom_px] = z0;
                float acc = 0.0f;
                for (uint32_t i = 0; i < K; ++i) {
                    float a = 0.0f;
                    for (uint32_t wk = 0; wk < 4u; ++wk) {
                        float pv = s_partial[(threadIdx.x + wk) * kMaxDomSlices + i];
                        a = a + (1.0f - a) * pv;
                    }
                    acc = acc + (1.0f - acc) * a;  // opaque_terminal_slice = K without opaque depth
                    R.dom_opacity[((size_t)layer * K + i) * D * D + dom_px] = acc;
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
        __syncthreads();
    }
}

// ===========================================================================
// K18 shading: per camera segment, DOM visibility at the midpoint, temporal
// blend, Marschner-style R/TT/TRT (strand_shading.wgsl:173-695).
// ===========================================================================
__constant__ float c_leg_roots[10] = {-9.739065170e-01f, -8.650633693e-01f, -6.794095635e-01f, -4.333953857e-01f,
                                      -1.488743424e-01f, 1.488743424e-01f,  4.333953857e-01f,  6.794095635e-01f,
                                      8.650633693e-01f,  9.739065170e-01f};
__constant__ float c_leg_weights[10] = {6.667134166e-02f, 1.494513452e-01f, 2.190863639e-01f, 2.692667246e-01f,
                                        2.955242395e-01f, 2.955242395e-01f, 2.692667246e-01f, 2.190863639e-01f,
                                        1.494513452e-01f, 6.667134166e-02f};
__constant__ float c_factorials[10] = {1.0f, 1.0f, 2.0f, 6.0f, 24.0f, 120.0f, 720.0f, 5040.0f, 40320.0f, 362880.0f};
constexpr float kPi = 3.14159265359f;
constexpr float kPiHalf = kPi / 2.0f;

__device__ __forceinline__ F3 nrm3(F3 v) {
    float l = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return f3(v.x / l, v.y / l, v.z / l);
}
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ float sample_dom(const FrameParams& P, const RenderArgs& R, F3 pw, uint32_t layer) {
    uint32_t f = kInvalid;
    for (uint32_t i = 0, l = 0; i < P.F; ++i) {
        if (P.frusta[i].kind != 1u) continue;
        if (l == layer) { f = i; break; }
        ++l;
    }
    if (f == kInvalid) return 1.0f;
    const fiber_frustum_desc& d = P.frusta[f];
    float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
    float4 raw = world_to_screen_raw(make_float4(pw.x, pw.y, pw.z, 1.0f), P.clip[f], vw, vh);
    if (raw.x < 0.0f || raw.y < 0.0f || raw.x >= vw || raw.y >= vh || raw.z < 0.0f || raw.z > 1.0f) return 1.0f;
    uint32_t px = f2u(raw.x), py = f2u(raw.y);
    const uint32_t D = P.dom_size, K = P.K;
    float z0 = R.dom_depth[(size_t)layer * D * D + (size_t)py * D + px];
    if (z0 <= 0.0f) return 1.0f;
    float z = normalize_depth01(raw.z);
    if (z > z0 - 1e-3f) return 1.0f;
    float u = wclamp(wmax(0.0f, z0 - z) / wmax(z0, 1e-6f), 0.0f, 1.0f);  // pow(., DOM_GAMMA = 1)
    uint32_t slice = min(f2u(floorf(u * u2f(K))), K - 1u);
    float op = R.dom_opacity[((size_t)layer * K + slice) * D * D + (size_t)py * D + px];
    return wclamp(1.0f - op, 0.08f, 1.0f);
}

__device__ __forceinline__ float fresnel_reflectance(float eta_i, float eta_t, float cos_theta_i) {
    float ci = fabsf(cos_theta_i);
    float cic = wclamp(0.0f, 1.0f, ci);  // WGSL clamp(0.0, 1.0, x) = min(1.0, x)
    float sin_i_sq = 1.0f - cic * cic;
    float ratio = eta_i / eta_t;
    float cos_t = sqrtf(1.0f - ratio * ratio * sin_i_sq);
    float rpar = ((eta_t * ci) - (eta_i * cos_t)) / ((eta_t * ci) + (eta_i * cos_t));
    float rper = ((eta_i * ci) - (eta_t * cos_t)) / ((eta_i * ci) + (eta_t * cos_t));
    return (rpar * rpar + rper * rper) * 0.5f;
}

// Sum of the 21 wrapped Gaussians (k = -10..10). Terms whose exponent is below
// -110 are exactly zero in binary32 and are skipped without changing the sum.
__device__ __forceinline__ float gaussian_detector(float beta, float phi_delta) {
    float var = beta * beta;
    if (var < 1e-6f) {
        float two_pi = 2.0f * kPi;
        float m = phi_delta - two_pi * truncf(phi_delta / two_pi);
        return fabsf(m) < 1e-3f ? 0.0f : 1e6f;
    }
    float norm = 1.0f / (sqrtf(2.0f * kPi) * beta);
    float two_var = 2.0f * var;
    float total = 0.0f;
    for (int k = -10; k <= 10; ++k) {
        float angle = phi_delta - 2.0f * kPi * (float)k;
        float e = -angle * angle / two_var;
        if (e > -110.0f) total = total + expf(e);
    }
    return norm * total;
}

__device__ F3 marschner(F3 L, F3 V, F3 U, const fiber_strand_material& m, float occlusion) {
    float theta_i = acosf(dot3(L, U));
    float theta_r = acosf(dot3(L, V));
    float dUL = dot3(U, L), dVL = dot3(V, L);
    F3 lp = nrm3(f3(U.x - L.x * dUL, U.y - L.y * dUL, U.z - L.z * dUL));
    F3 vp = nrm3(f3(V.x - L.x * dVL, V.y - L.y * dVL, V.z - L.z * dVL));
    float ang = acosf(dot3(nrm3(lp), nrm3(vp)));
    float sd = dot3(cross3(lp, vp), L);
    float phi = ang * (sd > 0.0f ? 1.0f : (sd < 0.0f ? -1.0f : 0.0f));
    float sig[3] = {1.0f - m.absorption_color[0], 1.0f - m.absorption_color[1], 1.0f - m.absorption_color[2]};
    float v_long = m.alpha * m.alpha;
    float v_azim = m.beta * m.beta;
    float beta_azim = sqrtf(v_azim);
    float vis = wclamp(1.0f - occlusion, 0.0f, 1.0f);
    float direct = wmix(0.18f, 1.0f, vis);
    // Mp (:470-523): I0 series (5 terms) x exp(), without the csch factor.
    float mp;
    {
        float trs = theta_r + m.shift;
        float ti = wclamp(-kPiHalf + 1e-6f, kPiHalf - 1e-6f, theta_i);
        trs = wclamp(-kPiHalf + 1e-6f, kPiHalf - 1e-6f, trs);
        float cti = cosf(-ti), ctr = cosf(trs), sti = sinf(-ti), strs = sinf(trs);
        if (v_long < 1e-6f) {
            float tol = 0.1f * (kPi / 180.0f);
            mp = fabsf(trs + ti) < tol ? 0.0f : 1e6f / tol;
        } else {
            float x = (cti * ctr) / v_long;
            float y = 0.0f;
            for (uint32_t i = 0; i < 5u; ++i) {
                float num = powf(x, 2.0f * u2f(i));
                float den = powf(4.0f, u2f(i)) * c_factorials[i] * c_factorials[i];
                y = y + num / den;
            }
            mp = y * expf((sti * strs) / v_long);
        }
    }
    float tot[3];
    for (int q = 0; q < 3; ++q) tot[q] = mp * m.specular_color[q] * m.specular_color[3] * direct;
    // Np (:525-562) for p = 0, 1, 2.
    float theta_d = (theta_r - theta_i) * 0.5f;
    float sti = sinf(theta_i);
    float ctd = cosf(theta_d);
    float eta_prime = sqrtf(wmax(0.0f, m.eta * m.eta - sti * sti)) / ctd;
    float mup[3] = {sig[0] / ctd, sig[1] / ctd, sig[2] / ctd};
    float cos_td = cosf(theta_d);
    for (uint32_t p = 0; p < 3u; ++p) {
        float acc[3] = {0.0f, 0.0f, 0.0f};
        for (uint32_t i = 0; i < 10u; ++i) {
            float h = wclamp(-1.0f + 1e-6f, 1.0f - 1e-6f, c_leg_roots[i]);
            // A (:383-413)
            float gamma_t = asinf(h / eta_prime);
            float gamma_i = asinf(h);
            float fr = fresnel_reflectance(1.0f, m.eta, acosf(cos_td * cosf(gamma_i)));
            float c2 = 1.0f + cosf(2.0f * gamma_t);
            float T[3] = {expf(-2.0f * mup[0] * c2), expf(-2.0f * mup[1] * c2), expf(-2.0f * mup[2] * c2)};
            float A[3];
            if (p == 0u) {
                for (int q = 0; q < 3; ++q) A[q] = fr * T[q] * T[q];
            } else {
                float f_ = 1.0f - fr;
                float k = (f_ * f_) * powf(fr, u2f(p - 1u));
                for (int q = 0; q < 3; ++q) A[q] = k * powf(T[q], u2f(p));
            }
            // Phi (:464-468)
            float gt2 = asinf(wclamp(h / eta_prime, -1.0f, 1.0f));
            float shift = 2.0f * u2f(p) * gt2 - 2.0f * asinf(h) + u2f(p) * kPi;
            float det = gaussian_detector(beta_azim, phi - shift);
            for (int q = 0; q < 3; ++q) acc[q] = acc[q] + A[q] * det * c_leg_weights[i];
        }
        float wgt = (u2f(p + 1u) * vis) / 3.0f;
        for (int q = 0; q < 3; ++q) tot[q] = tot[q] + (acc[q] * 0.5f) * wgt;
    }
    return f3(tot[0], tot[1], tot[2]);
}

__global__ void __launch_bounds__(128) k_shade(const FrameParams* __restrict__ Pp,
                                               const InstanceView* __restrict__ inst, RenderArgs R) {
    const FrameParams& P = *Pp;
    const uint32_t n = *((volatile uint32_t*)&R.counters->frustum_task_base[P.camera_frustum_end]);
    const uint32_t cap = P.atlas_cap;
    const uint32_t nl = min(P.L, 4u);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint4 t = reinterpret_cast<const uint4*>(R.tasks)[k];
        const uint32_t i = t.x, seg = t.z;
        const InstanceView& in = inst[i];
        const fiber_strand_meta sm = in.meta[t.y];
        float4 v0, v1;
        segment_world(in, seg, v0, v1);
        F3 U = nrm3(f3(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z));
        F3 cam = nrm3(f3(P.camera_pos[0] - v0.x, P.camera_pos[1] - v0.y, P.camera_pos[2] - v0.z));
        F3 B = nrm3(cross3(U, cam));
        F3 V = nrm3(cross3(B, U));
        const fiber_strand_material mat = in.materials[sm.material_idx];
        float accum[4] = {0.0f, 0.0f, 0.0f, mat.absorption_color[3]};
        const uint32_t atlas_idx = sm.offset + (seg - sm.offset);
        F3 mid = f3(wmix(v0.x, v1.x, 0.5f), wmix(v0.y, v1.y, 0.5f), wmix(v0.z, v1.z, 0.5f));
        float cur = 1.0f;
        if (nl != 0u) {
            float vs = 0.0f;
            for (uint32_t l = 0; l < nl; ++l) vs = vs + sample_dom(P, R, mid, l);
            cur = vs / u2f(nl);
        }
        const size_t hidx = (size_t)i * cap + atlas_idx;
        const __half* hist_prev = R.history[P.hist_in & 1u];
        __half* hist_next = R.history[(P.hist_in & 1u) ^ 1u];
        float prev = P.history_valid ? __half2float(hist_prev[hidx * 2]) : 0.0f;
        float vis = prev > 0.0f ? wmix(cur, prev, 0.88f) : cur;
        reinterpret_cast<__half2*>(hist_next)[hidx] = __halves2half2(__float2half_rn(vis), __float2half_rn(cur));
        float occ = 1.0f - vis;
        for (uint32_t j = 0; j < P.L; ++j) {
            const float* ld = P.light_dir[j];
            F3 L = nrm3(f3(ld[0], ld[1], ld[2]));
            F3 b = marschner(L, V, U, mat, occ);
            float bb[3] = {b.x, b.y, b.z};
            for (int q = 0; q < 3; ++q) {
                float c = bb[q] * (P.light_color[j][q] / 255.0f);
                float ambient = mat.absorption_color[q] * mat.ambient_factor + (P.ambient[q] / 255.0f) * mat.ambient_factor;
                c = wmix(c, ambient, mat.ambient_factor);
                accum[q] = accum[q] + c;
            }
        }
        __half2 lo = __halves2half2(__float2half_rn(wclamp(accum[0], 0.0f, 1.0f)), __float2half_rn(wclamp(accum[1], 0.0f, 1.0f)));
        __half2 hi = __halves2half2(__float2half_rn(wclamp(accum[2], 0.0f, 1.0f)), __float2half_rn(wclamp(accum[3], 0.0f, 1.0f)));
        uint2 packed = make_uint2(*reinterpret_cast<uint32_t*>(&lo), *reinterpret_cast<uint32_t*>(&hi));
        uint2* atlas = reinterpret_cast<uint2*>(R.atlas);
        atlas[hidx] = packed;
        // Texel seg + 1 belongs to segment seg + 1 when that segment is shaded
        // this frame (the next camera task); otherwise segment seg writes it.
        bool next_shades = false;
        if (k + 1u < n) {
            const uint4 tn = reinterpret_cast<const uint4*>(R.tasks)[k + 1u];
            next_shades = tn.x == i && tn.z == seg + 1u;
        }
        if (!next_shades && atlas_idx + 1u < cap) atlas[hidx + 1] = packed;
    }
}

// ===========================================================================
// K19 camera colour raster (strand_rasterizer.wgsl:855-1044). One block per
// camera tile run: 64 pixel slots x 4 segment workers, batches of 16
// references, premultiplied "over" reduced as (w0 over w1) over (w2 over w3),
// early out after each work item once alpha > 0.98.
// ===========================================================================
constexpr int kColorBatch = 16;

struct ColorBatch {
    float p0x[kColorBatch], p0y[kColorBatch], abx[kColorBatch], aby[kColorBatch], inv_len[kColorBatch];
    float z0[kColorBatch], z1[kColorBatch], w0[kColorBatch], w1[kColorBatch];
    float rmin[kColorBatch], rmax[kColorBatch];
    float mnx[kColorBatch], mny[kColorBatch], mxx[kColorBatch], mxy[kColorBatch];
    float4 s0[kColorBatch], s1[kColorBatch];
    float vis[kColorBatch];
    uint32_t valid[kColorBatch];
};

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

__global__ void __launch_bounds__(256) k_raster(const FrameParams* __restrict__ Pp,
                                                const InstanceView* __restrict__ inst, RenderArgs R) {
    const FrameParams& P = *Pp;
    __shared__ ColorBatch sb;
    const uint32_t n_runs = *((volatile uint32_t*)&R.counters->camera_active);
    const uint32_t slot = threadIdx.x >> 2, worker = threadIdx.x & 3u;
    const uint32_t lane = threadIdx.x & 31u, wbase = lane & ~3u;
    const uint32_t cap = P.atlas_cap;
    for (uint32_t r = blockIdx.x; r < n_runs; r += gridDim.x) {
        const fiber_raster_tile_run run = R.runs[r];
        const uint32_t f = run.frustum_id;
        if (run.work_count == 0u || f >= P.camera_frustum_end) continue;
        const fiber_frustum_desc& d = P.frusta[f];
        const float* clip = P.clip[f];
        const float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
        const uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x);
        const uint32_t tx = run.screen_tile_id % ftx, ty = run.screen_tile_id / ftx;
        const uint32_t px = tx * d.froxel_size_x + slot % d.froxel_size_x;
        const uint32_t py = ty * d.froxel_size_y + slot / d.froxel_size_x;
        const bool active = slot < d.froxel_size_x * d.froxel_size_y && px < d.screen_width && py < d.screen_height;
        const float pcx = u2f(px) + 0.5f, pcy = u2f(py) + 0.5f;
        float4 fin = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float gdepth = 0.0f;
        bool done = !active;
        uint32_t frags = 0;
        for (uint32_t w = 0; w < run.work_count; ++w) {
            const fiber_raster_work_item wi = R.work[run.work_base + w];
            for (uint32_t bb = 0; bb < wi.seg_ref_count; bb += kColorBatch) {
                __syncthreads();
                if (threadIdx.x < kColorBatch) {
                    const uint32_t j = threadIdx.x;
                    uint32_t v = 0u;
                    if (bb + j < wi.seg_ref_count) {
                        fiber_fine_seg_ref ref = R.refs[wi.seg_ref_base + bb + j];
                        const InstanceView& in = inst[ref.inst_id];
                        float4 w0, w1;
                        segment_world(in, ref.seg_id, w0, w1);
                        float4 a = world_to_screen_raw(w0, clip, vw, vh), b = world_to_screen_raw(w1, clip, vw, vh);
                        if (!(a.x < 0.0f && b.x < 0.0f)) {
                            fiber_strand_material m = in.materials[ref.material_idx];
                            float rmin = wmax(m.min_radius_pixels, 1e-4f);
                            float rmax = wmax(m.max_radius_pixels, rmin);
                            uint32_t i0 = ref.seg_id, i1 = min(i0 + 1u, cap - 1u);
                            size_t t0 = (size_t)ref.inst_id * cap + i0, t1 = (size_t)ref.inst_id * cap + i1;
                            float abx = b.x - a.x, aby = b.y - a.y;
                            sb.p0x[j] = a.x; sb.p0y[j] = a.y; sb.abx[j] = abx; sb.aby[j] = aby;
                            sb.inv_len[j] = 1.0f / (abx * abx + aby * aby);
                            sb.z0[j] = a.z; sb.z1[j] = b.z; sb.w0[j] = a.w; sb.w1[j] = b.w;
                            sb.rmin[j] = rmin; sb.rmax[j] = rmax;
                            sb.mnx[j] = wmin(a.x, b.x) - rmax; sb.mny[j] = wmin(a.y, b.y) - rmax;
                            sb.mxx[j] = wmax(a.x, b.x) + rmax; sb.mxy[j] = wmax(a.y, b.y) + rmax;
                            sb.s0[j] = load_half4(R.atlas + t0 * 4);
                            sb.s1[j] = load_half4(R.atlas + t1 * 4);
                            sb.vis[j] = __half2float(R.history[(P.hist_in & 1u) ^ 1u][t0 * 2]);
                            v = 1u;
                        }
                    }
                    sb.valid[j] = v;
                }
                __syncthreads();
                for (uint32_t g = 0; g < kColorBatch; g += 4u) {
                    float4 part = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    float pd = 0.0f;
                    const uint32_t bi = g + worker;
                    if (!done && sb.valid[bi] && !(pcx < sb.mnx[bi] || pcy < sb.mny[bi]) &&
                        !(pcx > sb.mxx[bi] || pcy > sb.mxy[bi])) {
                        float t = ((pcx - sb.p0x[bi]) * sb.abx[bi] + (pcy - sb.p0y[bi]) * sb.aby[bi]) * sb.inv_len[bi];
                        if (t >= 0.0f && t <= 1.0f) {
                            float fx = sb.p0x[bi] + sb.abx[bi] * t, fy = sb.p0y[bi] + sb.aby[bi] * t;
                            float pz = wmix(sb.z0[bi], sb.z1[bi], t);
                            float rmin = wmax(sb.rmin[bi], 1e-4f);
                            float rr = wmix(rmin, wmax(sb.rmax[bi], rmin), wclamp(normalize_depth01(pz), 0.0f, 1.0f));
                            float dx = pcx - fx, dy = pcy - fy;
                            float d2 = dx * dx + dy * dy;
                            if (d2 < rr * rr) {
                                float cov = wclamp(1.0f - sqrtf(d2) / rr, 0.0f, 1.0f);
                                // perspective_correct_line_t (:149-154)
                                float aw0 = wmax(fabsf(sb.w0[bi]), 1e-6f), aw1 = wmax(fabsf(sb.w1[bi]), 1e-6f);
                                float tw = (t * aw0) / ((1.0f - t) * aw1 + t * aw0);
                                float4 s0 = sb.s0[bi], s1 = sb.s1[bi];
                                float sr = wmix(s0.x, s1.x, tw), sg = wmix(s0.y, s1.y, tw);
                                float sbl = wmix(s0.z, s1.z, tw), sa = wmix(s0.w, s1.w, tw);
                                float alpha = sa * cov;
                                float vsb = sb.vis[bi];
                                part = make_float4(sr * vsb * alpha, sg * vsb * alpha, sbl * vsb * alpha, alpha);
                                pd = pz;
                                ++frags;
                            }
                        }
                    }
                    // (w0 over w1) over (w2 over w3), depth max.
                    float4 rhs;
                    rhs.x = __shfl_sync(0xFFFFFFFFu, part.x, wbase + (worker | 1u));
                    rhs.y = __shfl_sync(0xFFFFFFFFu, part.y, wbase + (worker | 1u));
                    rhs.z = __shfl_sync(0xFFFFFFFFu, part.z, wbase + (worker | 1u));
                    rhs.w = __shfl_sync(0xFFFFFFFFu, part.w, wbase + (worker | 1u));
                    float rd = __shfl_sync(0xFFFFFFFFu, pd, wbase + (worker | 1u));
                    float4 pair = part;
                    float pdd = pd;
                    if ((worker & 1u) == 0u) {
                        pair = over(part, rhs);
                        pdd = wmax(pd, rd);
                    }
                    float4 second;
                    second.x = __shfl_sync(0xFFFFFFFFu, pair.x, wbase + 2u);
                    second.y = __shfl_sync(0xFFFFFFFFu, pair.y, wbase + 2u);
                    second.z = __shfl_sync(0xFFFFFFFFu, pair.z, wbase + 2u);
                    second.w = __shfl_sync(0xFFFFFFFFu, pair.w, wbase + 2u);
                    float sdp = __shfl_sync(0xFFFFFFFFu, pdd, wbase + 2u);
                    if (worker == 0u && !done) {
                        fin = over(fin, over(pair, second));
                        gdepth = wmax(gdepth, wmax(pdd, sdp));
                    }
                }
            }
            if (worker == 0u && !done && fin.w > 0.98f) {
                fin = make_float4(fin.x / fin.w, fin.y / fin.w, fin.z / fin.w, 1.0f);
                done = true;
            }
            done = __shfl_sync(0xFFFFFFFFu, done, wbase);
            if (__syncthreads_and(done)) break;
        }
        // Sum the fragment counts of the 4 workers.
        frags += __shfl_xor_sync(0xFFFFFFFFu, frags, 1);
        frags += __shfl_xor_sync(0xFFFFFFFFu, frags, 2);
        if (worker == 0u && active) {
            float4 o = fin;
            if (o.w > 1e-6f && o.w < 1.0f) o = make_float4(o.x / o.w, o.y / o.w, o.z / o.w, o.w);
            size_t pi = (size_t)py * P.width + px;
            __half2 lo = __halves2half2(__float2half_rn(o.x), __float2half_rn(o.y));
            __half2 hi = __halves2half2(__float2half_rn(o.z), __float2half_rn(o.w));
            reinterpret_cast<uint2*>(R.color)[pi] = make_uint2(*reinterpret_cast<uint32_t*>(&lo), *reinterpret_cast<uint32_t*>(&hi));
            R.depth[pi] = gdepth;
            if (P.fragment_counts) R.fragments[pi] = frags;
        }
    }
}

// ===========================================================================
// K20 composite (strand_composite.wgsl:12-33) with BlendState::ALPHA_BLENDING
// onto the loaded destination (pipelines/composite.rs:115-124).
// ===========================================================================
__device__ __forceinline__ float4 load_px(const void* base, uint32_t pitch, uint32_t fmt, uint32_t x, uint32_t y) {
    const char* row = static_cast<const char*>(base) + (size_t)y * pitch;
    if (fmt == FIBER_FMT_RGBA32F) return reinterpret_cast<const float4*>(row)[x];
    return load_half4(reinterpret_cast<const __half*>(row) + 4 * x);
}
__device__ __forceinline__ void store_px(void* base, uint32_t pitch, uint32_t fmt, uint32_t x, uint32_t y, float4 v) {
    char* row = static_cast<char*>(base) + (size_t)y * pitch;
    if (fmt == FIBER_FMT_RGBA32F) {
        reinterpret_cast<float4*>(row)[x] = v;
        return;
    }
    __half2 lo = __halves2half2(__float2half_rn(v.x), __float2half_rn(v.y));
    __half2 hi = __halves2half2(__float2half_rn(v.z), __float2half_rn(v.w));
    reinterpret_cast<uint2*>(row)[x] = make_uint2(*reinterpret_cast<uint32_t*>(&lo), *reinterpret_cast<uint32_t*>(&hi));
}

__global__ void k_composite(CompositeArgs C) {
    const uint32_t n = C.width * C.height;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t x = i % C.width, y = i / C.width;
        float4 sc = load_px(C.scene_color, C.scene_pitch, C.scene_format, x, y);
        float sd = C.scene_depth ? reinterpret_cast<const float*>(reinterpret_cast<const char*>(C.scene_depth) + (size_t)y * C.depth_pitch)[x] : 0.0f;
        float4 st = load_half4(C.strand_color + (size_t)i * 4);
        float sdp = C.strand_depth[i];
        float4 frag;
        if (sd > sdp) frag = sc;
        else frag = make_float4(wmix(sc.x, st.x, st.w), wmix(sc.y, st.y, st.w), wmix(sc.z, st.z, st.w), sc.w);
        float4 dst = load_px(C.out, C.out_pitch, C.out_format, x, y);
        float oma = 1.0f - frag.w;
        float4 o = make_float4(frag.x * frag.w + dst.x * oma, frag.y * frag.w + dst.y * oma,
                               frag.z * frag.w + dst.z * oma, frag.w * 1.0f + dst.w * oma);
        store_px(C.out, C.out_pitch, C.out_format, x, y, o);
    }
}

void launch_shadow(const LaunchCtx& L, const RenderArgs& R) {
    k_shadow<<<L.sm_count * 4, 256, 0, L.stream>>>(L.P, L.inst, R);
}
void launch_shade(const LaunchCtx& L, const RenderArgs& R) {
    k_shade<<<L.sm_count * 16, 128, 0, L.stream>>>(L.P, L.inst, R);
}
void launch_raster(const LaunchCtx& L, const RenderArgs& R) {
    k_raster<<<L.sm_count * 6, 256, 0, L.stream>>>(L.P, L.inst, R);
}
void launch_composite(cudaStream_t s, const CompositeArgs& C) {
    unsigned blocks = ceil_div_host((uint64_t)C.width * C.height, 256);
    if (blocks > 148u * 16u) blocks = 148u * 16u;
    if (blocks) k_composite<<<blocks, 256, 0, s>>>(C);
}

}  // namespace fiber
