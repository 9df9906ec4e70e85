// fiber_render.cu — shading and composite: the reference's strand_shading_pass
// (src/nodes/shading.rs:25-155) and composition_pass
// (src/nodes/composite.rs:19-131). The rasters live in fiber_raster.cu.
#include "fiber_kernels.cuh"

namespace fiber {

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
__constant__ float c_mp_den[5] = {1.0f, 4.0f, 64.0f, 2304.0f, 147456.0f};  // 4^i (i!)^2
constexpr float kPi = 3.14159265359f;
constexpr float kPiHalf = kPi / 2.0f;

// This file is compiled with contraction and approximate division. The
// shading frame (tangent, view and light directions, their projections and
// the angles between them) is spelt with correctly rounded intrinsics, so an
// acos argument lands on the same side of +-1 as the reference's and an
// antiparallel or degenerate frame gives the same NaN; the smooth terms after
// it (the Mp series, the quadrature, the detectors) run on the fast path.
__device__ __forceinline__ float dot3(F3 a, F3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ F3 nrm3(F3 v) {
    const float l = __fsqrt_rn(dot3(v, v));
    return f3(__fdiv_rn(v.x, l), __fdiv_rn(v.y, l), __fdiv_rn(v.z, l));
}
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
// v - w * s, per component.
__device__ __forceinline__ F3 sub_scaled3(F3 v, F3 w, float s) {
    return f3(__fsub_rn(v.x, __fmul_rn(w.x, s)), __fsub_rn(v.y, __fmul_rn(w.y, s)), __fsub_rn(v.z, __fmul_rn(w.z, s)));
}

__device__ float sample_dom(const FrameParams& P, const RenderArgs& R, F3 pw, uint32_t layer) {
    const uint32_t f = layer < P.L ? P.layer_frustum[layer] : kInvalid;
    if (f == kInvalid) return 1.0f;
    const fiber_frustum_desc& d = P.frusta[f];
    float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
    float4 raw = world_to_screen_raw(make_float4(pw.x, pw.y, pw.z, 1.0f), P.clip[f], vw, vh);
    if (raw.x < 0.0f || raw.y < 0.0f || raw.x >= vw || raw.y >= vh || raw.z < 0.0f || raw.z > 1.0f) return 1.0f;
    uint32_t px = f2u(raw.x), py = f2u(raw.y);
    const uint32_t K = P.K;
    float* dz;
    float* dop;
    size_t ds;
    if (!dom_texel(P, R, layer, px, py, dz, dop, ds)) return 1.0f;  // page not resident: nothing there
    float z0 = *dz;
    if (z0 <= 0.0f) return 1.0f;
    float z = normalize_depth01(raw.z);
    if (z > z0 - 1e-3f) return 1.0f;
    float u = wclamp(__fdiv_rn(wmax(0.0f, z0 - z), wmax(z0, 1e-6f)), 0.0f, 1.0f);  // pow(., DOM_GAMMA = 1)
    uint32_t slice = min(f2u(floorf(u * u2f(K))), K - 1u);
    float op = dop[slice * ds];
    return wclamp(1.0f - op, 0.08f, 1.0f);
}

// fresnel_reflectance (:370-381) with eta_i = 1; ratio = 1 / eta_t is passed
// in. The quotients use the hardware reciprocal path (__fdividef): shading is
// compared within a tolerance, not bit for bit, and is stored as binary16.
__device__ __forceinline__ float fresnel_reflectance(float eta_t, float ratio, float cos_theta_i) {
    float ci = fabsf(cos_theta_i);
    float cic = wclamp(0.0f, 1.0f, ci);  // WGSL clamp(0.0, 1.0, x) = min(1.0, x)
    float sin_i_sq = 1.0f - cic * cic;
    float cos_t = sqrtf(1.0f - ratio * ratio * sin_i_sq);
    float rpar = __fdividef((eta_t * ci) - cos_t, (eta_t * ci) + cos_t);
    float rper = __fdividef(ci - (eta_t * cos_t), ci + (eta_t * cos_t));
    return (rpar * rpar + rper * rper) * 0.5f;
}

// gaussian_detector (:425-462) for one azimuthal width beta: the terms that
// depend on beta alone, evaluated once per shaded segment.
struct Detector {
    float var, norm, neg_inv_two_var, reach;
    bool near3;  // var < 2: the three wrapped terms nearest to phi carry the sum
    bool near1;  // var < 0.26: the nearest term alone does
};

__device__ __forceinline__ Detector make_detector(float beta) {
    Detector g;
    g.var = beta * beta;
    const float two_var = 2.0f * g.var;
    g.norm = 1.0f / (sqrtf(2.0f * kPi) * beta);
    g.neg_inv_two_var = -1.0f / two_var;
    g.reach = sqrtf(110.0f * two_var) * 1.001f + 1e-3f;
    g.near3 = g.var < 2.0f;
    g.near1 = g.var < 0.26f;
    return g;
}

// Sum of the 21 wrapped Gaussians (k = -10..10). Terms whose exponent is below
// -110 are zero in binary32 and are skipped without changing the sum; the test
// is written so that a NaN exponent is not skipped and still poisons the sum,
// as exp(NaN) does in the reference. Only k with |phi - 2 pi k| below
// sqrt(110 * 2 var) can pass it, so the loop runs over that window (its reach
// widened by 1e-3 relative + 1e-3 absolute), in the same increasing k order; a
// NaN phi takes the full range. The exponent is a product with -1 / (2 var)
// and exp is the hardware exp2 path (__expf), within the shading tolerance.
__device__ __forceinline__ float gaussian_detector(const Detector& g, float phi_delta) {
    if (g.var < 1e-6f) {
        float two_pi = 2.0f * kPi;
        float m = phi_delta - two_pi * truncf(phi_delta / two_pi);
        return fabsf(m) < 1e-3f ? 0.0f : 1e6f;
    }
    // Let k_c be the wrap nearest to phi (|phi - 2 pi k_c| <= pi; |phi| < 56
    // keeps k_c +- 1 inside k = -10..10). Nearest term alone: with var < 0.26
    // every other term is below exp(-pi^2 / (2 var)) < 5.8e-9 (|phi - 2 pi k|
    // >= pi), and the 20 of them change the detector by less than 1.2e-8 norm.
    if (g.near1 && fabsf(phi_delta) < 56.0f) {
        const float a = phi_delta - (2.0f * kPi) * rintf(phi_delta * (1.0f / (2.0f * kPi)));
        return g.norm * __expf((a * a) * g.neg_inv_two_var);
    }
    // Three nearest terms: every k other than k_c and k_c +- 1 has
    // |phi - 2 pi k| >= 3 pi, so its term is below exp(-9 pi^2 / (2 var)) <
    // 2.3e-10 for var < 2; the at most 18 such terms change the detector by
    // less than 4.2e-9 norm, far inside the shading tolerance. Summed in
    // increasing k, as the full loop does.
    if (g.near3 && fabsf(phi_delta) < 56.0f) {
        const float two_pi = 2.0f * kPi;
        const float kc = rintf(phi_delta * (1.0f / two_pi));
        const float a0 = phi_delta - two_pi * (kc - 1.0f), a1 = phi_delta - two_pi * kc,
                    a2 = phi_delta - two_pi * (kc + 1.0f);
        const float total = (__expf((a0 * a0) * g.neg_inv_two_var) + __expf((a1 * a1) * g.neg_inv_two_var)) +
                            __expf((a2 * a2) * g.neg_inv_two_var);
        return g.norm * total;
    }
    int k0 = -10, k1 = 10;
    if (phi_delta == phi_delta) {
        const float inv_two_pi = 1.0f / (2.0f * kPi);
        const float lo = wclamp(floorf((phi_delta - g.reach) * inv_two_pi), -11.0f, 11.0f);
        const float hi = wclamp(ceilf((phi_delta + g.reach) * inv_two_pi), -11.0f, 11.0f);
        k0 = max(k0, (int)lo);
        k1 = min(k1, (int)hi);
    }
    float total = 0.0f;
    for (int k = k0; k <= k1; ++k) {
        float angle = phi_delta - 2.0f * kPi * (float)k;
        float e = (angle * angle) * g.neg_inv_two_var;
        if (!(e <= -110.0f)) total = total + __expf(e);
    }
    return g.norm * total;
}

// Per quadrature point i, terms that depend on the root alone: h (the clamped
// root), asin(h) and cos(asin(h)). A block fills them once.
struct QuadTable {
    float h[10], gi[10], cgi[10];
};

__device__ __forceinline__ void fill_quad_table(QuadTable& t) {
    if (threadIdx.x < 10u) {
        const float h = wclamp(-1.0f + 1e-6f, 1.0f - 1e-6f, c_leg_roots[threadIdx.x]);
        const float gi = asinf(h);
        t.h[threadIdx.x] = h;
        t.gi[threadIdx.x] = gi;
        t.cgi[threadIdx.x] = cosf(gi);
    }
}

__device__ F3 marschner(F3 L, F3 V, F3 U, const fiber_strand_material& m, float occlusion, const QuadTable& qt,
                        const Detector& det_azim) {
    float theta_i = acosf(dot3(L, U));
    float theta_r = acosf(dot3(L, V));
    float dUL = dot3(U, L), dVL = dot3(V, L);
    F3 lp = nrm3(sub_scaled3(U, L, dUL));
    F3 vp = nrm3(sub_scaled3(V, L, dVL));
    float ang = acosf(dot3(nrm3(lp), nrm3(vp)));
    float sd = dot3(cross3(lp, vp), L);
    float phi = ang * (sd > 0.0f ? 1.0f : (sd < 0.0f ? -1.0f : 0.0f));
    float sig[3] = {1.0f - m.absorption_color[0], 1.0f - m.absorption_color[1], 1.0f - m.absorption_color[2]};
    float v_long = m.alpha * m.alpha;
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
            // sum_i x^(2i) / (4^i (i!)^2), i = 0..4: the powers of x as running
            // products, the denominators as their exact values 1, 4, 64, 2304,
            // 147456.
            float x = (cti * ctr) / v_long;
            const float x2 = x * x;
            float y = 0.0f, num = 1.0f;
            for (uint32_t i = 0; i < 5u; ++i) {
                y = y + num / c_mp_den[i];
                num = num * x2;
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
    const float inv_eta_prime = 1.0f / eta_prime;
    const float inv_eta = 1.0f / m.eta;
    float mup[3] = {sig[0] / ctd, sig[1] / ctd, sig[2] / ctd};
    const float cos_td = ctd;  // cos(theta_d), the same evaluation
    // The quadrature point's Fresnel, absorption and azimuth terms depend on
    // the segment only, not on the path p, so they are evaluated once per point
    // and reused by the three paths; each path's sum keeps its order (i = 0..9).
    // asin(h) serves gamma_i and the azimuth shift alike, and asin(clamp(x))
    // equals asin(x) whenever |x| <= 1. The path powers are exact products:
    // pow(x, 0) = 1, pow(x, 1) = x and pow(x, 2) = x * x correctly rounded.
    float acc[3][3] = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}};
    for (uint32_t i = 0; i < 10u; ++i) {
        const float h = qt.h[i];
        // A (:383-413)
        const float x_t = h * inv_eta_prime;
        float gamma_t = asinf(x_t);
        float gamma_i = qt.gi[i];
        float fr = fresnel_reflectance(m.eta, inv_eta, acosf(cos_td * qt.cgi[i]));
        float c2 = 1.0f + __cosf(2.0f * gamma_t);
        float T[3] = {__expf(-2.0f * mup[0] * c2), __expf(-2.0f * mup[1] * c2), __expf(-2.0f * mup[2] * c2)};
        float f_ = 1.0f - fr;
        // Phi (:464-468)
        float gt2 = fabsf(x_t) <= 1.0f ? gamma_t : asinf(wclamp(x_t, -1.0f, 1.0f));
        float asin_h = gamma_i;
        for (uint32_t p = 0; p < 3u; ++p) {
            float A[3];
            if (p == 0u) {
                for (int q = 0; q < 3; ++q) A[q] = fr * T[q] * T[q];
            } else if (p == 1u) {
                float k = (f_ * f_) * 1.0f;
                for (int q = 0; q < 3; ++q) A[q] = k * T[q];
            } else {
                float k = (f_ * f_) * fr;
                for (int q = 0; q < 3; ++q) A[q] = k * (T[q] * T[q]);
            }
            float shift = 2.0f * u2f(p) * gt2 - 2.0f * asin_h + u2f(p) * kPi;
            float det = gaussian_detector(det_azim, phi - shift);
            for (int q = 0; q < 3; ++q) acc[p][q] = acc[p][q] + A[q] * det * c_leg_weights[i];
        }
    }
    for (uint32_t p = 0; p < 3u; ++p) {
        float wgt = (u2f(p + 1u) * vis) / 3.0f;
        for (int q = 0; q < 3; ++q) tot[q] = tot[q] + (acc[p][q] * 0.5f) * wgt;
    }
    return f3(tot[0], tot[1], tot[2]);
}

__global__ void __launch_bounds__(128, 8) k_shade(const FrameParams* __restrict__ Pp,
                                               const InstanceView* __restrict__ inst, RenderArgs R) {
    if (frame_failed(R.counters)) return;
    const FrameParams& P = *Pp;
    __shared__ QuadTable s_quad;
    fill_quad_table(s_quad);
    __syncthreads();
    const uint32_t n = *((volatile uint32_t*)&R.counters->frustum_task_base[P.camera_frustum_end]);
    const uint32_t cap = P.atlas_cap;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint4 t = reinterpret_cast<const uint4*>(R.tasks)[k];
        const uint32_t i = t.x, seg = t.z;
        // The task's view: its camera position and its own lights.
        const uint32_t view = P.fview[min(t.w >> 3, kMaxFrusta - 1u)];
        const float* camera_pos = P.view_cam_pos[view];
        const uint32_t l0 = P.view_layer0[view], nlv = P.view_layers[view];
        const uint32_t nl = min(nlv, 4u);
        const InstanceView& in = inst[i];
        const fiber_strand_meta sm = in.meta[t.y];
        float4 v0, v1;
        segment_world(in, seg, v0, v1);
        F3 U = nrm3(f3(__fsub_rn(v1.x, v0.x), __fsub_rn(v1.y, v0.y), __fsub_rn(v1.z, v0.z)));
        F3 cam = nrm3(f3(__fsub_rn(camera_pos[0], v0.x), __fsub_rn(camera_pos[1], v0.y),
                         __fsub_rn(camera_pos[2], v0.z)));
        F3 B = nrm3(cross3(U, cam));
        F3 V = nrm3(cross3(B, U));
        const fiber_strand_material mat = in.materials[sm.material_idx];
        float accum[4] = {0.0f, 0.0f, 0.0f, mat.absorption_color[3]};
        const uint32_t atlas_idx = sm.offset + (seg - sm.offset);
        F3 mid = f3(wmix(v0.x, v1.x, 0.5f), wmix(v0.y, v1.y, 0.5f), wmix(v0.z, v1.z, 0.5f));
        float cur = 1.0f;
        if (nl != 0u) {
            float vs = 0.0f;
            for (uint32_t l = 0; l < nl; ++l) vs = vs + sample_dom(P, R, mid, l0 + l);
            cur = vs / u2f(nl);
        }
        const size_t hidx = (size_t)i * cap + atlas_idx;
        const __half* hist_prev = R.history[P.hist_in & 1u];
        __half* hist_next = R.history[(P.hist_in & 1u) ^ 1u];
        float prev = P.history_valid ? __half2float(hist_prev[hidx * 2]) : 0.0f;
        float vis = prev > 0.0f ? wmix(cur, prev, 0.88f) : cur;
        reinterpret_cast<__half2*>(hist_next)[hidx] = __halves2half2(__float2half_rn(vis), __float2half_rn(cur));
        float occ = 1.0f - vis;
        const Detector det_azim = make_detector(sqrtf(mat.beta * mat.beta));
        for (uint32_t j = l0; j < l0 + nlv; ++j) {
            const float* ld = P.light_dir[j];
            F3 L = nrm3(f3(ld[0], ld[1], ld[2]));
            F3 b = marschner(L, V, U, mat, occ, s_quad, det_azim);
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

void launch_shade(const LaunchCtx& L, const RenderArgs& R) {
    k_shade<<<L.sm_count * 16, 128, 0, L.stream>>>(L.P, L.inst, R);
}
void launch_composite(cudaStream_t s, const CompositeArgs& C) {
    unsigned blocks = ceil_div_host((uint64_t)C.width * C.height, 256);
    if (blocks > 148u * 16u) blocks = 148u * 16u;
    if (blocks) k_composite<<<blocks, 256, 0, s>>>(C);
}

}  // namespace fiber
