// fiber_ref.cpp — ORACLE (test infrastructure only; see fiber_ref.h).
//
// CPU restatement of the reference's strand software-raster path. Each stage
// cites the WGSL it restates (paths inside RostigerDagmer/bevy_strand_rasterizer).
// Built with -ffp-contract=off and no fast-math: every + - * / sqrt is one
// IEEE-754 binary32 operation in source order, and a matrix-vector product is
// c0*x + c1*y + c2*z + c3*w left to right. The integer-deciding stages use only
// those operations plus floor / round-half-even, so the CUDA path (built with
// --fmad=false) must reproduce them bit for bit.
//
// Canonical orders (the reference appends with atomics):
//   binning tasks  (frustum, instance, strand, segment)
//   coarse ranges  dense [instance][frustum]; LUT intervals merged in instance order
//   count pages    page-table order (coarse tile, coarse z)
//   ref bases      prefix over pages in page order
//   refs in a cell (depth key of the projected segment descending, inst, seg)
//   tile runs      active fine-tile order (coarse tile * 16 + local fine tile)
//   work items     run order, then near-to-far lanes

#include "fiber_ref.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t kCoarseExtent = 4;    // COARSE_FINE_TILE_EXTENT, src/plugin.rs:58
constexpr uint32_t kDepthSlices = 16;    // COARSE_DEPTH_SLICES, src/plugin.rs:59
constexpr uint32_t kPageSize = 256;      // COARSE_COUNT_PAGE_SIZE, src/plugin.rs:61
constexpr uint32_t kDepthQuantMax = 16777215u;  // strand_prepass.wgsl:65
constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kMarked = 0xFFFFFFFEu;       // strand_prepass.wgsl:69
constexpr uint32_t kMaxTexture = 8192;          // MAX_TEXTURE_EXTENT, src/plugin.rs:57
constexpr float kPi = 3.14159265359f;           // strand_shading.wgsl:52
constexpr float kPiHalf = kPi / 2.0f;
constexpr uint32_t kPixelSlots = 64;            // strand_rasterizer.wgsl:309,839
constexpr uint32_t kShadowWorkers = 4;          // :310
constexpr uint32_t kShadowBatch = 256;          // :311
constexpr uint32_t kColorWorkers = 4;           // :840
constexpr uint32_t kColorBatch = 16;            // :841

struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };

// ---- WGSL builtin semantics -------------------------------------------------
inline float wmin(float a, float b) { return std::fmin(a, b); }
inline float wmax(float a, float b) { return std::fmax(a, b); }
// WGSL clamp(e, lo, hi) = min(max(e, lo), hi) (also for the swapped-argument
// calls in strand_shading.wgsl:307,364,386,465,491-492).
inline float wclamp(float e, float lo, float hi) { return wmin(wmax(e, lo), hi); }
inline int32_t iclamp(int32_t e, int32_t lo, int32_t hi) { return std::min(std::max(e, lo), hi); }
inline float wmix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline float wfract(float x) { return x - std::floor(x); }
// Saturating float -> integer conversions (WGSL clamps out-of-range values).
inline uint32_t f2u(float f) {
    if (!(f > 0.0f)) return 0u;
    if (f >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)f;
}
inline int32_t f2i(float f) {
    if (f != f) return 0;
    if (f <= -2147483648.0f) return INT32_MIN;
    if (f >= 2147483648.0f) return INT32_MAX;
    return (int32_t)f;
}
inline float u2f(uint32_t u) { return (float)u; }  // round to nearest even

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 sub3(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 add3(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 mul3s(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot2(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline V3 cross3(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline V3 normalize3(V3 v) {
    float l = std::sqrt(dot3(v, v));
    return v3(v.x / l, v.y / l, v.z / l);
}
inline V3 mix3(V3 a, V3 b, float t) { return v3(wmix(a.x, b.x, t), wmix(a.y, b.y, t), wmix(a.z, b.z, t)); }

inline V4 matvec(const float* m, V4 v) {
    V4 r;
    r.x = ((m[0] * v.x + m[4] * v.y) + m[8] * v.z) + m[12] * v.w;
    r.y = ((m[1] * v.x + m[5] * v.y) + m[9] * v.z) + m[13] * v.w;
    r.z = ((m[2] * v.x + m[6] * v.y) + m[10] * v.z) + m[14] * v.w;
    r.w = ((m[3] * v.x + m[7] * v.y) + m[11] * v.z) + m[15] * v.w;
    return r;
}

// common.wgsl:206-212
inline float normalize_depth01(float z) {
    if (z >= 0.0f && z <= 1.0f) return z;
    return wclamp(z * 0.5f + 0.5f, 0.0f, 1.0f);
}
// common.wgsl:93-107
inline V4 world_to_screen_raw(V4 p, const float* clip_from_world, float vw, float vh) {
    V4 c = matvec(clip_from_world, p);
    if (c.w <= 0.0f) return V4{-1.0f, -1.0f, -1.0f, -1.0f};
    float nx = c.x / c.w, ny = c.y / c.w, nz = c.z / c.w;
    float sx = 0.0f + (nx * 0.5f + 0.5f) * vw;
    float sy = 0.0f + (ny * -0.5f + 0.5f) * vh;
    return V4{sx, sy, nz, c.w};
}
// common.wgsl:229-242
inline uint32_t wang_hash(uint32_t x) {
    x = (x ^ 61u) ^ (x >> 16u);
    x = x + (x << 3u);
    x = x ^ (x >> 4u);
    x = x * 0x27d4eb2du;
    x = x ^ (x >> 15u);
    return x;
}
inline float hash_to_unit_float(uint32_t x) { return u2f(x) / 4294967296.0f; }
// strand_prepass.wgsl:533-539
inline uint32_t quantize_depth01(float z) {
    return f2u(std::nearbyint(wclamp(z, 0.0f, 1.0f) * (float)kDepthQuantMax));
}
inline float dequantize_depth01(uint32_t q) { return u2f(q) / (float)kDepthQuantMax; }
// WGSL pack2x16unorm: floor(0.5 + 65535 * clamp(e, 0, 1)), x in the low half.
inline uint32_t unorm16(float e) {
    float t = 65535.0f * wmin(1.0f, wmax(0.0f, e));
    return f2u(std::floor(0.5f + t));
}
inline uint32_t pack2x16unorm(float a, float b) { return unorm16(a) | (unorm16(b) << 16u); }
inline V2 unpack2x16unorm(uint32_t p) {
    return V2{u2f(p & 0xFFFFu) / 65535.0f, u2f(p >> 16u) / 65535.0f};
}
inline int32_t sgn_i32(float f) {  // strand_prepass.wgsl:523-527
    if (f > 1e-6f) return 1;
    if (f < -1e-6f) return -1;
    return 0;
}
inline uint16_t to_half_bits(float f) {
    _Float16 h = (_Float16)f;
    uint16_t b;
    std::memcpy(&b, &h, 2);
    return b;
}
inline float from_half_bits(uint16_t b) {
    _Float16 h;
    std::memcpy(&h, &b, 2);
    return (float)h;
}
inline uint32_t ceil_div(uint32_t x, uint32_t y) { return (x + y - 1u) / y; }

// ---- clip_axis_to_range / clip_segment_to_box (strand_prepass.wgsl:1356-1410)
struct Clipped { bool ok; V3 p0, p1; };
inline bool clip_axis(float p, float d, float mn, float mx, float& tmin, float& tmax) {
    if (std::fabs(d) < 1e-6f) return !(p < mn || p > mx);
    float inv_d = 1.0f / d;
    float a = (mn - p) * inv_d;
    float b = (mx - p) * inv_d;
    if (a > b) std::swap(a, b);
    tmin = wmax(tmin, a);
    tmax = wmin(tmax, b);
    return !(tmin > tmax);
}
inline Clipped clip_segment(V3 p0, V3 p1, V3 bmin, V3 bmax) {
    V3 d = sub3(p1, p0);
    float tmin = 0.0f, tmax = 1.0f;
    if (!clip_axis(p0.x, d.x, bmin.x, bmax.x, tmin, tmax)) return Clipped{false, p0, p1};
    if (!clip_axis(p0.y, d.y, bmin.y, bmax.y, tmin, tmax)) return Clipped{false, p0, p1};
    if (!clip_axis(p0.z, d.z, bmin.z, bmax.z, tmin, tmax)) return Clipped{false, p0, p1};
    return Clipped{true, add3(p0, mul3s(d, tmin)), add3(p0, mul3s(d, tmax))};
}

// ---- depth-warp LUT (build_depth_warp_lut, strand_prepass.wgsl:884-1014)
inline uint32_t interval_gap(uint32_t amin, uint32_t amax, uint32_t bmin, uint32_t bmax) {
    if (amax < bmin) return bmin - amax;
    if (bmax < amin) return amin - bmax;
    return 0u;
}
struct LutBuilder {
    uint32_t mins[kDepthSlices], maxs[kDepthSlices];
    uint32_t count = 0;
    void add(uint32_t a, uint32_t b) {
        uint32_t zmin = std::min(a, b), zmax = std::max(a, b);
        bool merged = false;
        for (uint32_t i = 0; i < count; ++i) {
            if (zmin <= maxs[i] + 1u && zmax + 1u >= mins[i]) {
                mins[i] = std::min(mins[i], zmin);
                maxs[i] = std::max(maxs[i], zmax);
                merged = true;
            }
        }
        if (merged) return;
        if (count < kDepthSlices) {
            mins[count] = zmin;
            maxs[count] = zmax;
            ++count;
            return;
        }
        uint32_t best = 0, best_gap = 0xFFFFFFFFu;
        for (uint32_t i = 0; i < kDepthSlices; ++i) {
            uint32_t g = interval_gap(mins[i], maxs[i], zmin, zmax);
            if (g < best_gap) { best_gap = g; best = i; }
        }
        mins[best] = std::min(mins[best], zmin);
        maxs[best] = std::max(maxs[best], zmax);
    }
    void emit(fiber_coarse_depth_lut_entry* out) {
        for (uint32_t i = 0; i < kDepthSlices; ++i) out[i] = {0u, 0u, 0u, 0u};
        if (count == 0) return;
        for (uint32_t i = 1; i < count; ++i) {  // insertion sort by z_min
            uint32_t j = i, kmin = mins[i], kmax = maxs[i];
            while (j != 0 && mins[j - 1] > kmin) {
                mins[j] = mins[j - 1];
                maxs[j] = maxs[j - 1];
                --j;
            }
            mins[j] = kmin;
            maxs[j] = kmax;
        }
        uint32_t out_slice = 0;
        for (uint32_t k = 0; k < count; ++k) {
            uint32_t base_slices = std::max(1u, kDepthSlices / count);
            uint32_t rem = kDepthSlices % count;
            uint32_t slices = base_slices + (k < rem ? 1u : 0u);
            uint32_t zmin = mins[k], zmax = maxs[k];
            uint32_t span = std::max(1u, zmax - zmin + 1u);
            for (uint32_t s = 0; s < slices && out_slice < kDepthSlices; ++s) {
                uint32_t start = zmin + (span * s) / slices;
                uint32_t excl_end = zmin + (span * (s + 1u)) / slices;
                uint32_t end = std::min(excl_end > start ? excl_end - 1u : start, zmax);
                out[out_slice++] = {start, end, start, std::max(1u, end - start + 1u)};
            }
        }
    }
};

// ---- frame state -------------------------------------------------------------
struct Inst {
    const fref_instance* src;
    uint32_t strand_count;  // min(meta count, geo.strand_count)
};

struct ShadowRunOut;

}  // namespace

struct fref_frame {
    uint32_t F = 0, I = 0, L = 0, K = 0;
    std::vector<fiber_frustum_desc> frusta;
    std::vector<const float*> clip;  // clip_from_world per frustum
    uint32_t total_coarse_tiles = 0;
    std::vector<uint32_t> range_valid;
    std::vector<fiber_coarse_asset_range> ranges;
    std::vector<float> keep;
    std::vector<uint32_t> inst_visible, inst_strands;
    std::vector<float> inst_cam_keep, inst_shadow_keep;
    std::vector<fiber_coarse_depth_lut_entry> lut;
    std::vector<fiber_binning_task> tasks;
    std::vector<fiber_projected_segment> projected;
    std::vector<uint32_t> frustum_task_base;  // F+1
    std::vector<uint32_t> page_table;
    std::vector<fiber_fine_page_meta> page_meta;
    std::vector<uint32_t> counts, offsets;
    std::vector<fiber_fine_seg_ref> refs;
    std::vector<uint32_t> ref_keys;
    std::vector<uint32_t> active_tiles;
    std::vector<fiber_raster_work_item> work;
    std::vector<fiber_raster_tile_run> runs;  // camera runs, then shadow runs
    uint32_t camera_runs = 0, shadow_runs = 0;
    uint32_t D = 0, S = 0;
    std::vector<float> dom_depth, dom_opacity, shadow_map;
    uint32_t atlas_w = 1, atlas_h = 1, atlas_cap = 1;
    std::vector<uint16_t> atlas, history;
    uint32_t W = 0, H = 0;
    std::vector<uint16_t> color;
    std::vector<float> depth;
    std::vector<uint32_t> fragments;
    std::vector<float> composite;
    std::vector<uint32_t> opaque_tiles;  // (covered, farthest q) per camera fine tile
    // Prepass telemetry (PrepassTelemetrySettings): per-frustum visibility and
    // retention counts, candidate tasks per page, the reference tail, and the
    // fiber_telemetry image built from them after the emit.
    std::vector<uint32_t> tel_visible_instances = std::vector<uint32_t>(16, 0u);
    std::vector<uint32_t> tel_visible_strands = std::vector<uint32_t>(16, 0u);
    std::vector<uint32_t> tel_retained = std::vector<uint32_t>(16, 0u);
    std::vector<uint32_t> page_candidates;
    uint64_t refs_tail = 0;
    std::vector<uint32_t> telemetry;
    bool opaque_bound = false;
    uint32_t overflow = 0;
    uint32_t n_cam_tasks = 0;
    uint64_t total_segments = 0, total_points = 0, total_strands = 0;
    float stage_ms[8] = {0};
};

namespace {

struct Ctx {
    fref_frame* fr;
    std::vector<Inst> inst;
    const fiber_settings* st;
    const fiber_camera* cam;
    const fiber_light* lights;
    fref_capacities caps;
};

inline uint32_t frustum_for_tile(const fref_frame* fr, uint32_t tile) {
    for (uint32_t f = 0; f < fr->F; ++f) {
        const auto& d = fr->frusta[f];
        if (tile >= d.coarse_depth_tile_base && tile < d.coarse_depth_tile_base + d.coarse_depth_tile_count)
            return f;
    }
    return kInvalid;
}
// light_layer_from_frustum (strand_prepass.wgsl:408-425)
inline uint32_t light_layer(const fref_frame* fr, uint32_t f) {
    if (f >= fr->F || fr->frusta[f].kind != 1u) return kInvalid;
    uint32_t layer = 0;
    for (uint32_t i = 0; i < f; ++i)
        if (fr->frusta[i].kind == 1u) ++layer;
    return layer >= fr->L ? kInvalid : layer;
}

// ---- K1 broad_prepass (strand_prepass.wgsl:295-392, 575-760) ----------------
void aabb_corners(const fiber_aabb& a, const float* w, V4 out[8]) {
    const float* mn = a.min;
    const float* mx = a.max;
    V4 c[8] = {{mn[0], mn[1], mn[2], 1}, {mn[0], mn[1], mx[2], 1}, {mn[0], mx[1], mn[2], 1},
               {mn[0], mx[1], mx[2], 1}, {mx[0], mn[1], mn[2], 1}, {mx[0], mn[1], mx[2], 1},
               {mx[0], mx[1], mn[2], 1}, {mx[0], mx[1], mx[2], 1}};
    for (int i = 0; i < 8; ++i) out[i] = matvec(w, c[i]);
}

struct CornerScan {
    V2 smin{1e30f, 1e30f}, smax{-1e30f, -1e30f};
    float zmin = 1.0f, zmax = 0.0f;
    bool any = false, near_clip = false;
};
CornerScan scan_corners(const V4 corners[8], const float* clip, float vw, float vh) {
    CornerScan s;
    for (int i = 0; i < 8; ++i) {
        V4 c = matvec(clip, corners[i]);
        if (c.w <= 1e-6f) { s.near_clip = true; continue; }
        float nx = c.x / c.w, ny = c.y / c.w, nz = c.z / c.w;
        if (nz < 0.0f) s.near_clip = true;
        float rx = 0.0f + (nx * 0.5f + 0.5f) * vw;
        float ry = 0.0f + (ny * -0.5f + 0.5f) * vh;
        s.any = true;
        s.smin = V2{wmin(s.smin.x, rx), wmin(s.smin.y, ry)};
        s.smax = V2{wmax(s.smax.x, rx), wmax(s.smax.y, ry)};
        float z = normalize_depth01(nz);
        s.zmin = wmin(s.zmin, z);
        s.zmax = wmax(s.zmax, z);
    }
    return s;
}

float aabb_area(const fref_frame* fr, uint32_t f, const V4 corners[8]) {
    const auto& d = fr->frusta[f];
    float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
    CornerScan s = scan_corners(corners, fr->clip[f], vw, vh);
    if (s.near_clip) return vw * vh;
    if (!s.any) return -1.0f;
    if (s.smax.x < 0.0f || s.smax.y < 0.0f || s.smin.x >= vw || s.smin.y >= vh) return -1.0f;
    if (s.zmax < 0.0f || s.zmin > 1.0f) return -1.0f;
    float cminx = wclamp(s.smin.x, 0.0f, vw - 1.0f), cminy = wclamp(s.smin.y, 0.0f, vh - 1.0f);
    float cmaxx = wclamp(s.smax.x, 0.0f, vw - 1.0f), cmaxy = wclamp(s.smax.y, 0.0f, vh - 1.0f);
    float ex = wmax(cmaxx - cminx, 1.0f), ey = wmax(cmaxy - cminy, 1.0f);
    return ex * ey;
}

bool emit_range(Ctx& c, uint32_t inst, uint32_t f, const V4 corners[8]) {
    fref_frame* fr = c.fr;
    const auto& d = fr->frusta[f];
    if (d.coarse_depth_tile_count == 0u) return false;
    if (d.kind == 1u && light_layer(fr, f) == kInvalid) return false;
    float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
    CornerScan s = scan_corners(corners, fr->clip[f], vw, vh);
    if (s.near_clip) {
        s.smin = V2{0.0f, 0.0f};
        s.smax = V2{vw - 1.0f, vh - 1.0f};
        s.zmax = 1.0f;
        if (!s.any) s.zmin = 0.0f;
        s.any = true;
    }
    if (!s.any) return false;
    if (s.smax.x < 0.0f || s.smax.y < 0.0f || s.smin.x >= vw || s.smin.y >= vh) return false;
    if (s.zmax < 0.0f || s.zmin > 1.0f) return false;
    uint32_t cpx = std::max(1u, d.froxel_size_x * kCoarseExtent);
    uint32_t cpy = std::max(1u, d.froxel_size_y * kCoarseExtent);
    float cminx = wclamp(s.smin.x, 0.0f, vw - 1.0f), cminy = wclamp(s.smin.y, 0.0f, vh - 1.0f);
    float cmaxx = wclamp(s.smax.x, 0.0f, vw - 1.0f), cmaxy = wclamp(s.smax.y, 0.0f, vh - 1.0f);
    fiber_coarse_asset_range r;
    r.geo_id = inst;
    r.frustum_id = f;
    r.min_x = std::min(f2u(cminx) / cpx, d.coarse_tiles_x - 1u);
    r.max_x = std::min(f2u(cmaxx) / cpx, d.coarse_tiles_x - 1u);
    r.min_y = std::min(f2u(cminy) / cpy, d.coarse_tiles_y - 1u);
    r.max_y = std::min(f2u(cmaxy) / cpy, d.coarse_tiles_y - 1u);
    r.z_min_q = quantize_depth01(s.zmin);
    r.z_max_q = quantize_depth01(s.zmax);
    fr->ranges[inst * fr->F + f] = r;
    fr->range_valid[inst * fr->F + f] = 1u;
    return true;
}

float camera_keep(const fiber_settings* st, uint32_t n, float area) {
    if (st->stochastic_cull_enabled == 0u) return 1.0f;
    if (area < 0.0f) return 0.0f;
    float density = wmax(st->target_strands_per_pixel, 1e-5f);
    float min_keep = wclamp(st->min_keep_probability, 0.0f, 1.0f);
    return wclamp(area * density / wmax(u2f(n), 1.0f), min_keep, 1.0f);
}
float shadow_keep(const fiber_settings* st, uint32_t n, float area, uint32_t cascade) {
    if (st->stochastic_cull_enabled == 0u) return 1.0f;
    if (area < 0.0f) return 0.0f;
    float density = wmax(st->target_strands_per_pixel, 1e-5f);
    float min_keep = wclamp(st->min_keep_probability, 0.0f, 1.0f);
    float cap = wclamp(st->shadow_keep_probability, 0.0f, 1.0f);
    float area_keep = wclamp(area * density / wmax(u2f(n), 1.0f), min_keep, 1.0f);
    float curved = area_keep * area_keep;
    float scale = 1.0f / std::exp2(u2f(cascade));
    return wclamp(curved * scale * cap, min_keep, 1.0f);
}

void stage_broad(Ctx& c) {
    fref_frame* fr = c.fr;
    for (uint32_t i = 0; i < fr->I; ++i) {
        const fref_instance* in = c.inst[i].src;
        uint32_t strand_count = c.inst[i].strand_count;
        V4 corners[8];
        aabb_corners(in->geo.aabb, in->world_from_local, corners);
        bool visible = false;
        float cam_k = 0.0f, sh_k = 0.0f;
        for (uint32_t f = 0; f < fr->F; ++f) {
            const auto& d = fr->frusta[f];
            float k = 0.0f;
            if (d.kind <= 1u) {
                bool vis = emit_range(c, i, f, corners);
                visible = vis || visible;
                if (vis && f < 16u) {  // FRUSTUM_TELEMETRY_VISIBLE_* (:735-738)
                    fr->tel_visible_instances[f] += 1u;
                    fr->tel_visible_strands[f] += strand_count;
                }
                if (vis && d.kind == 0u) {
                    k = camera_keep(c.st, strand_count, aabb_area(fr, f, corners));
                    cam_k = wmax(cam_k, k);
                } else if (vis && d.kind == 1u) {
                    k = shadow_keep(c.st, strand_count, aabb_area(fr, f, corners), d.cascade_index);
                    sh_k = wmax(sh_k, k);
                }
            }
            fr->keep[i * fr->F + f] = k;
        }
        fr->inst_visible[i] = visible ? 1u : 0u;
        fr->inst_strands[i] = strand_count;
        fr->inst_cam_keep[i] = cam_k;
        fr->inst_shadow_keep[i] = sh_k;
    }
}

// ---- K4/K5 coarse intervals + depth-warp LUT --------------------------------
void stage_lut(Ctx& c) {
    fref_frame* fr = c.fr;
    fr->lut.assign((size_t)fr->total_coarse_tiles * kDepthSlices, {0, 0, 0, 0});
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < (int64_t)fr->total_coarse_tiles; ++t) {
        uint32_t f = frustum_for_tile(fr, (uint32_t)t);
        if (f == kInvalid) continue;
        const auto& d = fr->frusta[f];
        uint32_t local = (uint32_t)t - d.coarse_depth_tile_base;
        uint32_t cx = local % d.coarse_tiles_x, cy = local / d.coarse_tiles_x;
        LutBuilder b;
        for (uint32_t i = 0; i < fr->I; ++i) {
            if (!fr->range_valid[i * fr->F + f]) continue;
            const auto& r = fr->ranges[i * fr->F + f];
            if (r.max_x < r.min_x || r.max_y < r.min_y) continue;
            if (cx < r.min_x || cx > r.max_x || cy < r.min_y || cy > r.max_y) continue;
            b.add(r.z_min_q, r.z_max_q);
        }
        b.emit(&fr->lut[(size_t)t * kDepthSlices]);
    }
}

// ---- K2 + K6 fine prepass (strand_prepass.wgsl:762-782, 1016-1140) ----------
struct SegEmit { fiber_binning_task task; fiber_projected_segment proj; };

void fine_strand(Ctx& c, uint32_t f, uint32_t inst, uint32_t strand, std::vector<SegEmit>& out) {
    fref_frame* fr = c.fr;
    const fref_instance* in = c.inst[inst].src;
    const auto& d = fr->frusta[f];
    if (d.kind > 1u) return;
    if (strand >= in->n_meta) return;
    const fiber_strand_meta& m = in->meta[strand];
    if (m.count < 2u) return;
    float strand_random = hash_to_unit_float(wang_hash((inst * 16777619u) ^ strand));
    float k = fr->keep[inst * fr->F + f];
    if (strand_random > k) return;
    if (d.kind == 1u && light_layer(fr, f) == kInvalid) return;
    if (f < 16u) __atomic_fetch_add(&fr->tel_retained[f], 1u, __ATOMIC_RELAXED);  // :1085
    uint32_t is_shadow = d.kind == 1u ? 1u : 0u;
    uint32_t packed = 0u | (is_shadow << 2u) | (f << 3u);
    const float* clip = fr->clip[f];
    float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
    V3 box_max = v3(wmax(0.0f, vw - 1e-3f), wmax(0.0f, vh - 1e-3f), 1.0f);
    float ssx = wmax(1.0f, vw), ssy = wmax(1.0f, vh);
    const float* W = in->world_from_local;
    for (uint32_t i = 0; i < m.count - 1u; ++i) {
        uint32_t seg = m.offset + i;
        if (seg + 1u >= in->n_indices) continue;
        uint32_t vi0 = in->indices[seg], vi1 = in->indices[seg + 1u];
        const float* a = in->vertices4 + 4ull * vi0;
        const float* b = in->vertices4 + 4ull * vi1;
        V4 w0 = matvec(W, V4{a[0], a[1], a[2], 1.0f});
        V4 w1 = matvec(W, V4{b[0], b[1], b[2], 1.0f});
        V4 r0 = world_to_screen_raw(w0, clip, vw, vh);
        V4 r1 = world_to_screen_raw(w1, clip, vw, vh);
        V3 p0 = v3(r0.x, r0.y, normalize_depth01(r0.z));
        V3 p1 = v3(r1.x, r1.y, normalize_depth01(r1.z));
        Clipped cl = clip_segment(p0, p1, v3(0, 0, 0), box_max);
        if (!cl.ok) continue;
        SegEmit e;
        e.task = {inst, strand, seg, packed};
        e.proj.p0_xy = pack2x16unorm(wclamp(cl.p0.x / ssx, 0.0f, 1.0f), wclamp(cl.p0.y / ssy, 0.0f, 1.0f));
        e.proj.p1_xy = pack2x16unorm(wclamp(cl.p1.x / ssx, 0.0f, 1.0f), wclamp(cl.p1.y / ssy, 0.0f, 1.0f));
        e.proj.depths = pack2x16unorm(wclamp(cl.p0.z, 0.0f, 1.0f), wclamp(cl.p1.z, 0.0f, 1.0f));
        out.push_back(e);
    }
}

void stage_fine(Ctx& c) {
    fref_frame* fr = c.fr;
    // K2: fine tasks in (instance, strand) order.
    std::vector<std::pair<uint32_t, uint32_t>> fine;
    for (uint32_t i = 0; i < fr->I; ++i) {
        if (!fr->inst_visible[i]) continue;
        float keep = wmax(fr->inst_cam_keep[i], fr->inst_shadow_keep[i]);
        for (uint32_t s = 0; s < fr->inst_strands[i]; ++s) {
            if (hash_to_unit_float(wang_hash((i * 16777619u) ^ s)) > keep) continue;
            fine.emplace_back(i, s);
        }
    }
    fr->tasks.clear();
    fr->projected.clear();
    fr->frustum_task_base.assign(fr->F + 1, 0);
    const int64_t n = (int64_t)fine.size();
    for (uint32_t f = 0; f < fr->F; ++f) {
        fr->frustum_task_base[f] = (uint32_t)fr->tasks.size();
        std::vector<std::vector<SegEmit>> per(n);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t k = 0; k < n; ++k) fine_strand(c, f, fine[k].first, fine[k].second, per[k]);
        for (int64_t k = 0; k < n; ++k) {
            for (const auto& e : per[k]) {
                if (fr->tasks.size() >= c.caps.task_capacity) { fr->overflow |= 1u; break; }
                fr->tasks.push_back(e.task);
                fr->projected.push_back(e.proj);
            }
        }
    }
    fr->frustum_task_base[fr->F] = (uint32_t)fr->tasks.size();
    fr->n_cam_tasks = 0;
    for (uint32_t f = 0; f < fr->F; ++f)
        if (fr->frusta[f].kind == 0u) fr->n_cam_tasks += fr->frustum_task_base[f + 1] - fr->frustum_task_base[f];
}

// ---- K0 reduce_opaque_depth (opaque_depth_reduce.wgsl:36-86) ---------------
// depth: the camera's opaque depth, reversed-Z, `samples` floats per pixel,
// rows of width * samples floats. Without one the tiles stay cleared
// (src/nodes/prepass.rs:140-145) and nothing is culled.
void stage_opaque(Ctx& c, const float* depth, uint32_t samples) {
    fref_frame* fr = c.fr;
    const fiber_frustum_desc& d = fr->frusta[0];  // the camera, kind 0
    const uint32_t tx = ceil_div(d.screen_width, d.froxel_size_x), ty = ceil_div(d.screen_height, d.froxel_size_y);
    fr->opaque_tiles.assign((size_t)tx * ty * 2, 0u);
    fr->opaque_bound = depth != nullptr;
    if (!depth) return;
    for (uint32_t t = 0; t < tx * ty; ++t) {
        const uint32_t x0 = (t % tx) * d.froxel_size_x, y0 = (t / tx) * d.froxel_size_y;
        const uint32_t x1 = std::min(x0 + d.froxel_size_x, d.screen_width);
        const uint32_t y1 = std::min(y0 + d.froxel_size_y, d.screen_height);
        uint32_t covered = 0, total = 0;
        float farthest = 1.0f;
        for (uint32_t y = y0; y < y1; ++y) {
            for (uint32_t x = x0; x < x1; ++x) {
                ++total;
                const float* px = depth + ((size_t)y * d.screen_width + x) * samples;
                float z = px[0];
                for (uint32_t q = 1; q < samples; ++q) z = wmin(z, px[q]);
                if (z > 0.0f) {
                    ++covered;
                    farthest = wmin(farthest, z);
                }
            }
        }
        fr->opaque_tiles[(size_t)t * 2] = covered == total && total > 0u ? 1u : 0u;
        fr->opaque_tiles[(size_t)t * 2 + 1] = quantize_depth01(farthest);
    }
}

// fine_tile_occluded_by_opaque (strand_prepass.wgsl:551-573); the tiles hold
// the camera's fine tiles only, whose fine_depth_tile_base is 0.
bool fine_tile_occluded(const fref_frame* fr, const fiber_frustum_desc& d, uint32_t fx, uint32_t fy,
                        float nearest_depth) {
    if (!fr->opaque_bound || d.kind != 0u) return false;
    const uint32_t tx = ceil_div(d.screen_width, d.froxel_size_x), ty = ceil_div(d.screen_height, d.froxel_size_y);
    if (fx >= tx || fy >= ty) return false;
    const size_t idx = (size_t)d.fine_depth_tile_base + (size_t)fy * tx + fx;
    if (idx * 2 >= fr->opaque_tiles.size()) return false;
    if (fr->opaque_tiles[idx * 2] == 0u) return false;
    return nearest_depth <= dequantize_depth01(fr->opaque_tiles[idx * 2 + 1]) - 1e-4f;
}

// ---- K7/K9/K11 coarse + fine traversal (strand_prepass.wgsl:1251-1696) ------
enum class Pass { Mark, Count, Fill };

inline uint32_t lut_slice(const fref_frame* fr, uint32_t tile, float z) {
    uint32_t zq = quantize_depth01(z);
    const fiber_coarse_depth_lut_entry* e = &fr->lut[(size_t)tile * kDepthSlices];
    uint32_t best = kInvalid, best_d = 0xFFFFFFFFu;
    for (uint32_t i = 0; i < kDepthSlices; ++i) {
        if (e[i].virtual_count_q == 0u) continue;
        if (zq >= e[i].z_min_q && zq <= e[i].z_max_q) return i;
        uint32_t dist = zq > e[i].z_max_q ? zq - e[i].z_max_q : e[i].z_min_q - zq;
        if (dist < best_d) { best_d = dist; best = i; }
    }
    return best;
}

// canonical_min_mask (common.wgsl:249-262): 0 = x, 1 = y, 2 = z
inline int min_axis(V3 t) {
    float m = wmin(wmin(t.x, t.y), t.z);
    if (t.x == m) return 0;
    if (t.y == m) return 1;
    return 2;
}

struct Visit {
    Pass pass;
    uint32_t task_idx;
    fiber_fine_seg_ref ref;
    uint32_t key;
};

struct Traverse {
    fref_frame* fr;
    uint32_t* cursors;  // fill pass
    void cell(const Visit& v, uint32_t page, uint32_t cx, uint32_t cy, uint32_t cz) {
        uint32_t cell = (cz * kCoarseExtent + cy) * kCoarseExtent + cx;
        size_t g = (size_t)page * kPageSize + cell;
        if (v.pass == Pass::Count) {
            __atomic_fetch_add(&fr->counts[g], 1u, __ATOMIC_RELAXED);
        } else {
            const auto& pm = fr->page_meta[page];
            if (pm.seg_ref_count == 0u) return;
            uint32_t lw = __atomic_fetch_add(&cursors[g], 1u, __ATOMIC_RELAXED);
            size_t dst = (size_t)pm.seg_ref_base + fr->offsets[g] + lw;
            if (dst >= fr->refs.size()) return;
            fr->refs[dst] = v.ref;
            fr->ref_keys[dst] = v.key;
        }
    }

    void trace_page(const Visit& v, V3 p0, V3 p1, const fiber_frustum_desc& d, uint32_t tile, uint32_t local) {
        uint32_t ccx = local % d.coarse_tiles_x, ccy = local / d.coarse_tiles_x;
        uint32_t cpx = std::max(1u, d.froxel_size_x * kCoarseExtent);
        uint32_t cpy = std::max(1u, d.froxel_size_y * kCoarseExtent);
        V2 origin{u2f(ccx * cpx), u2f(ccy * cpy)};
        V2 tmax_xy{wmin(origin.x + u2f(cpx), u2f(d.screen_width)) - 1e-3f,
                   wmin(origin.y + u2f(cpy), u2f(d.screen_height)) - 1e-3f};
        V3 bmin = v3(origin.x, origin.y, 0.0f);
        V3 bmax = v3(wmax(origin.x, tmax_xy.x), wmax(origin.y, tmax_xy.y), 1.0f);
        Clipped cl = clip_segment(p0, p1, bmin, bmax);
        if (!cl.ok) return;
        uint32_t z0s = lut_slice(fr, tile, cl.p0.z), z1s = lut_slice(fr, tile, cl.p1.z);
        if (z0s == kInvalid || z1s == kInvalid) return;
        for (uint32_t cz = std::min(z0s, z1s); cz <= std::max(z0s, z1s); ++cz) {
            const auto& e = fr->lut[(size_t)tile * kDepthSlices + cz];
            if (e.virtual_count_q == 0u) continue;
            float zmin = dequantize_depth01(e.z_min_q), zmax = dequantize_depth01(e.z_max_q);
            Clipped dc = clip_segment(cl.p0, cl.p1, v3(origin.x, origin.y, zmin), v3(bmax.x, bmax.y, zmax));
            if (!dc.ok) continue;
            uint32_t pti = tile * kDepthSlices + cz;
            if (v.pass == Pass::Mark) {
                __atomic_store_n(&fr->page_table[pti], kMarked, __ATOMIC_RELAXED);
                continue;
            }
            uint32_t handle = fr->page_table[pti];
            if (handle == 0u || handle == kMarked) continue;
            uint32_t page = handle - 1u;
            // The count pass's per-page candidate counter (:1485-1490).
            if (v.pass == Pass::Count) __atomic_fetch_add(&fr->page_candidates[page], 1u, __ATOMIC_RELAXED);
            float zspan = wmax(zmax - zmin, 1.0f / (float)kDepthQuantMax);
            float fsx = u2f(d.froxel_size_x), fsy = u2f(d.froxel_size_y);
            V3 l0 = v3((dc.p0.x - origin.x) / fsx, (dc.p0.y - origin.y) / fsy,
                       wclamp((dc.p0.z - zmin) / zspan, 0.0f, 0.999999f) * 16.0f);
            V3 l1 = v3((dc.p1.x - origin.x) / fsx, (dc.p1.y - origin.y) / fsy,
                       wclamp((dc.p1.z - zmin) / zspan, 0.0f, 0.999999f) * 16.0f);
            int32_t f0[3] = {iclamp(f2i(std::floor(l0.x)), 0, 3), iclamp(f2i(std::floor(l0.y)), 0, 3),
                             iclamp(f2i(std::floor(l0.z)), 0, 15)};
            int32_t f1[3] = {iclamp(f2i(std::floor(l1.x)), 0, 3), iclamp(f2i(std::floor(l1.y)), 0, 3),
                             iclamp(f2i(std::floor(l1.z)), 0, 15)};
            V3 dir = sub3(l1, l0);
            int32_t step[3] = {sgn_i32(dir.x), sgn_i32(dir.y), sgn_i32(dir.z)};
            float sd[3] = {std::fabs(dir.x) < 1e-6f ? 1e-6f : dir.x, std::fabs(dir.y) < 1e-6f ? 1e-6f : dir.y,
                           std::fabs(dir.z) < 1e-6f ? 1e-6f : dir.z};
            float dd[3] = {std::fabs(1.0f / sd[0]), std::fabs(1.0f / sd[1]), std::fabs(1.0f / sd[2])};
            float pl[3] = {l0.x, l0.y, l0.z};
            float dv[3] = {dir.x, dir.y, dir.z};
            float tm[3];
            for (int a = 0; a < 3; ++a) {
                float fl = std::floor(pl[a]);
                tm[a] = step[a] > 0 ? ((fl + 1.0f) - pl[a]) / sd[a] : (fl - pl[a]) / sd[a];
                if (std::fabs(dv[a]) < 1e-6f) tm[a] = 1e38f;
            }
            int32_t fc[3] = {f0[0], f0[1], f0[2]};
            uint32_t safety = 0;
            for (;;) {
                if (safety > kCoarseExtent + kCoarseExtent + kDepthSlices + 3u) break;
                // Opaque fine-tile cull (:1539-1553 count/fill): the cell is
                // skipped, the walk goes on. zmax is the slice's nearest depth.
                if (!fine_tile_occluded(fr, d, ccx * kCoarseExtent + (uint32_t)fc[0],
                                        ccy * kCoarseExtent + (uint32_t)fc[1], zmax))
                    cell(v, page, (uint32_t)fc[0], (uint32_t)fc[1], (uint32_t)fc[2]);
                if (fc[0] == f1[0] && fc[1] == f1[1] && fc[2] == f1[2]) break;
                int a = min_axis(v3(tm[0], tm[1], tm[2]));
                fc[a] += step[a];
                tm[a] += dd[a];
                if (fc[0] < 0 || fc[1] < 0 || fc[2] < 0 || fc[0] >= 4 || fc[1] >= 4 || fc[2] >= 16) break;
                ++safety;
            }
        }
    }

    void visit(const Visit& v) {
        const fiber_binning_task& t = fr->tasks[v.task_idx];
        uint32_t f = t.packed_field >> 3u;
        if (f >= fr->F) return;
        const auto& d = fr->frusta[f];
        uint32_t inst = t.id_info;
        if (inst >= fr->I) return;
        const fiber_projected_segment& pr = fr->projected[v.task_idx];
        float sw = u2f(d.screen_width), sh = u2f(d.screen_height);
        V2 a = unpack2x16unorm(pr.p0_xy), b = unpack2x16unorm(pr.p1_xy), z = unpack2x16unorm(pr.depths);
        V3 p0 = v3(a.x * sw, a.y * sh, z.x);
        V3 p1 = v3(b.x * sw, b.y * sh, z.y);
        if (!fr->range_valid[inst * fr->F + f]) return;
        const auto& r = fr->ranges[inst * fr->F + f];
        uint32_t cpx = std::max(1u, d.froxel_size_x * kCoarseExtent);
        uint32_t cpy = std::max(1u, d.froxel_size_y * kCoarseExtent);
        float smin_x = wmin(p0.x, p1.x), smin_y = wmin(p0.y, p1.y);
        float smax_x = wmax(p0.x, p1.x), smax_y = wmax(p0.y, p1.y);
        uint32_t min_cx = std::max(r.min_x, std::min(f2u(wmax(smin_x, 0.0f)) / cpx, d.coarse_tiles_x - 1u));
        uint32_t max_cx = std::min(r.max_x, std::min(f2u(wmax(smax_x, 0.0f)) / cpx, d.coarse_tiles_x - 1u));
        uint32_t min_cy = std::max(r.min_y, std::min(f2u(wmax(smin_y, 0.0f)) / cpy, d.coarse_tiles_y - 1u));
        uint32_t max_cy = std::min(r.max_y, std::min(f2u(wmax(smax_y, 0.0f)) / cpy, d.coarse_tiles_y - 1u));
        if (max_cx < min_cx || max_cy < min_cy) return;
        V3 bmin = v3(u2f(min_cx * cpx), u2f(min_cy * cpy), 0.0f);
        V3 bmax = v3(wmin(u2f((max_cx + 1u) * cpx), sw) - 1e-3f, wmin(u2f((max_cy + 1u) * cpy), sh) - 1e-3f, 1.0f);
        Clipped cl = clip_segment(p0, p1, bmin, bmax);
        if (!cl.ok) return;
        V2 c0{cl.p0.x / u2f(cpx), cl.p0.y / u2f(cpy)};
        V2 c1{cl.p1.x / u2f(cpx), cl.p1.y / u2f(cpy)};
        int32_t fx = iclamp(f2i(std::floor(c0.x)), (int32_t)min_cx, (int32_t)max_cx);
        int32_t fy = iclamp(f2i(std::floor(c0.y)), (int32_t)min_cy, (int32_t)max_cy);
        int32_t ex = iclamp(f2i(std::floor(c1.x)), (int32_t)min_cx, (int32_t)max_cx);
        int32_t ey = iclamp(f2i(std::floor(c1.y)), (int32_t)min_cy, (int32_t)max_cy);
        V2 dir{c1.x - c0.x, c1.y - c0.y};
        int32_t sx = sgn_i32(dir.x), sy = sgn_i32(dir.y);
        float sdx = std::fabs(dir.x) < 1e-6f ? 1e-6f : dir.x;
        float sdy = std::fabs(dir.y) < 1e-6f ? 1e-6f : dir.y;
        float ddx = std::fabs(1.0f / sdx), ddy = std::fabs(1.0f / sdy);
        float fl_x = std::floor(c0.x), fl_y = std::floor(c0.y);
        float tx = sx > 0 ? ((fl_x + 1.0f) - c0.x) / sdx : (fl_x - c0.x) / sdx;
        float ty = sy > 0 ? ((fl_y + 1.0f) - c0.y) / sdy : (fl_y - c0.y) / sdy;
        if (std::fabs(dir.x) < 1e-6f) tx = 1e38f;
        if (std::fabs(dir.y) < 1e-6f) ty = 1e38f;
        uint32_t safety = 0;
        uint32_t max_steps = (max_cx - min_cx + 1u) + (max_cy - min_cy + 1u) + 2u;
        for (;;) {
            if (safety > max_steps) break;
            if (fx < (int32_t)min_cx || fx > (int32_t)max_cx || fy < (int32_t)min_cy || fy > (int32_t)max_cy) break;
            uint32_t local = (uint32_t)fy * d.coarse_tiles_x + (uint32_t)fx;
            if (local < d.coarse_depth_tile_count)
                trace_page(v, p0, p1, d, d.coarse_depth_tile_base + local, local);
            if (fx == ex && fy == ey) break;
            if (tx <= ty) { fx += sx; tx += ddx; } else { fy += sy; ty += ddy; }
            ++safety;
        }
    }
};

void stage_binning(Ctx& c) {
    fref_frame* fr = c.fr;
    const int64_t n = (int64_t)fr->tasks.size();
    const size_t table = (size_t)fr->total_coarse_tiles * kDepthSlices;
    fr->page_table.assign(table, 0u);
    Traverse tr{fr, nullptr};
    // K7 mark
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t k = 0; k < n; ++k) tr.visit(Visit{Pass::Mark, (uint32_t)k, {}, 0});
    // K8 allocate in page-table order (allocate_coarse_count_pages, :1934-1969)
    fr->page_meta.clear();
    for (size_t pti = 0; pti < table; ++pti) {
        if (fr->page_table[pti] != kMarked) continue;
        uint32_t idx = (uint32_t)fr->page_meta.size();
        if (idx >= c.caps.page_capacity) {
            fr->page_table[pti] = 0u;
            fr->overflow |= 2u;
            continue;
        }
        fr->page_meta.push_back({0, 0, 0, 0, (uint32_t)(pti / kDepthSlices), (uint32_t)(pti % kDepthSlices), 0, 0});
        fr->page_table[pti] = idx + 1u;
    }
    const size_t pages = fr->page_meta.size();
    // K9 count
    fr->counts.assign(pages * kPageSize, 0u);
    fr->page_candidates.assign(pages, 0u);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t k = 0; k < n; ++k) tr.visit(Visit{Pass::Count, (uint32_t)k, {}, 0});
    // K10 prefix (prefix_fine_pages, :2051-2143); ref bases in page order.
    fr->offsets.assign(pages * kPageSize, 0u);
    std::vector<uint32_t> active_flags(table, 0u);
    uint64_t tail = 0;
    for (size_t p = 0; p < pages; ++p) {
        uint32_t acc = 0;
        for (uint32_t cidx = 0; cidx < kPageSize; ++cidx) {
            fr->offsets[p * kPageSize + cidx] = acc;
            acc += fr->counts[p * kPageSize + cidx];
        }
        auto& pm = fr->page_meta[p];
        uint32_t base = 0, flags = 0;
        if (acc > 0u) {
            base = (uint32_t)tail;
            tail += acc;
            if ((uint64_t)base + acc > c.caps.ref_capacity) { flags = 1u; fr->overflow |= 4u; }
        }
        pm.seg_ref_base = base;
        pm.seg_ref_count = flags ? 0u : acc;
        pm.flags = flags;
        uint32_t f = frustum_for_tile(fr, pm.coarse_tile_id);
        if (flags != 0u || f == kInvalid) continue;
        const auto& d = fr->frusta[f];
        uint32_t local_coarse = pm.coarse_tile_id - d.coarse_depth_tile_base;
        uint32_t ccx = local_coarse % d.coarse_tiles_x, ccy = local_coarse / d.coarse_tiles_x;
        uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x), fty = ceil_div(d.screen_height, d.froxel_size_y);
        for (uint32_t lt = 0; lt < 16u; ++lt) {
            bool has = false;
            for (uint32_t z = 0; z < kDepthSlices; ++z) has = has || fr->counts[p * kPageSize + z * 16u + lt] > 0u;
            if (!has) continue;
            uint32_t fx = ccx * kCoarseExtent + lt % kCoarseExtent, fy = ccy * kCoarseExtent + lt / kCoarseExtent;
            if (fx >= ftx || fy >= fty) continue;  // append_active_fine_tile, :2207-2238
            active_flags[(size_t)pm.coarse_tile_id * 16u + lt] = 1u;
        }
    }
    fr->refs_tail = tail;
    // K11 fill; then the canonical within-cell order.
    uint64_t ref_total = 0;
    for (const auto& pm : fr->page_meta) ref_total += pm.seg_ref_count;
    uint64_t ref_extent = 0;
    for (const auto& pm : fr->page_meta)
        if (pm.seg_ref_count) ref_extent = std::max<uint64_t>(ref_extent, (uint64_t)pm.seg_ref_base + pm.seg_ref_count);
    fr->refs.assign(ref_extent, fiber_fine_seg_ref{0, 0, 0});
    fr->ref_keys.assign(ref_extent, 0u);
    std::vector<uint32_t> cursors(pages * kPageSize, 0u);
    tr.cursors = cursors.data();
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t k = 0; k < n; ++k) {
        const fiber_binning_task& t = fr->tasks[k];
        Visit v{Pass::Fill, (uint32_t)k, {t.id_info, t.seg_idx, 0u}, 0u};
        // make_fine_seg_ref (:1313-1327)
        const fref_instance* in = c.inst[t.id_info].src;
        if (t.chunk_id < in->n_meta) v.ref.material_idx = in->meta[t.chunk_id].material_idx;
        uint32_t dz = fr->projected[k].depths;
        v.key = (dz & 0xFFFFu) + (dz >> 16u);
        tr.visit(v);
    }
    (void)ref_total;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t p = 0; p < (int64_t)pages; ++p) {
        const auto& pm = fr->page_meta[p];
        if (pm.seg_ref_count == 0u) continue;
        for (uint32_t cidx = 0; cidx < kPageSize; ++cidx) {
            uint32_t cnt = fr->counts[p * kPageSize + cidx];
            if (cnt < 2u) continue;
            size_t base = (size_t)pm.seg_ref_base + fr->offsets[p * kPageSize + cidx];
            std::vector<uint32_t> order(cnt);
            for (uint32_t j = 0; j < cnt; ++j) order[j] = j;
            std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
                uint32_t kx = fr->ref_keys[base + x], ky = fr->ref_keys[base + y];
                if (kx != ky) return kx > ky;
                const auto& rx = fr->refs[base + x];
                const auto& ry = fr->refs[base + y];
                if (rx.inst_id != ry.inst_id) return rx.inst_id < ry.inst_id;
                if (rx.seg_id != ry.seg_id) return rx.seg_id < ry.seg_id;
                return rx.material_idx < ry.material_idx;
            });
            std::vector<fiber_fine_seg_ref> tmp(cnt);
            std::vector<uint32_t> tk(cnt);
            for (uint32_t j = 0; j < cnt; ++j) { tmp[j] = fr->refs[base + order[j]]; tk[j] = fr->ref_keys[base + order[j]]; }
            for (uint32_t j = 0; j < cnt; ++j) { fr->refs[base + j] = tmp[j]; fr->ref_keys[base + j] = tk[j]; }
        }
    }
    // K13 ordered active-tile compaction (:2581-2676)
    fr->active_tiles.clear();
    for (size_t i = 0; i < active_flags.size(); ++i)
        if (active_flags[i]) fr->active_tiles.push_back((uint32_t)i);
}

// ---- K14 emit_raster_work (:2509-2518, 2678-2834) ----------------------------
void stage_emit(Ctx& c) {
    fref_frame* fr = c.fr;
    fr->work.clear();
    std::vector<fiber_raster_tile_run> cam, sh;
    for (uint32_t packed : fr->active_tiles) {
        uint32_t lt = packed % 16u, tile = packed / 16u;
        uint32_t f = frustum_for_tile(fr, tile);
        if (f == kInvalid) continue;
        const auto& d = fr->frusta[f];
        uint32_t local = tile - d.coarse_depth_tile_base;
        uint32_t ccx = local % d.coarse_tiles_x, ccy = local / d.coarse_tiles_x;
        uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x);
        uint32_t lx = lt % kCoarseExtent, ly = lt / kCoarseExtent;
        uint32_t fx = ccx * kCoarseExtent + lx, fy = ccy * kCoarseExtent + ly;
        uint32_t screen_tile = fy * ftx + fx;
        std::vector<fiber_raster_work_item> items;
        uint32_t load = 0;
        for (uint32_t lane = 0; lane < kPageSize; ++lane) {
            uint32_t depth_lane = kPageSize - 1u - lane;
            uint32_t cz = depth_lane / kDepthSlices, fz = depth_lane % kDepthSlices;
            uint32_t pti = tile * kDepthSlices + cz;
            uint32_t handle = fr->page_table[pti];
            if (handle == 0u || handle == kMarked) continue;
            uint32_t page = handle - 1u;
            const auto& pm = fr->page_meta[page];
            uint32_t cell = (fz * kCoarseExtent + ly) * kCoarseExtent + lx;
            uint32_t cnt = 0, base = 0;
            if (pm.seg_ref_count > 0u && pm.flags == 0u) {
                cnt = fr->counts[(size_t)page * kPageSize + cell];
                if (cnt > 0u) base = pm.seg_ref_base + fr->offsets[(size_t)page * kPageSize + cell];
            }
            if (cnt == 0u) continue;
            const auto& lut = fr->lut[pti];
            uint32_t dkey = lut.virtual_count_q == 0u ? fz : lut.virtual_start_q + (lut.virtual_count_q * fz) / kDepthSlices;
            items.push_back({base, cnt, f, screen_tile, dkey, cnt, page, cell});
            load += cnt;
        }
        if (items.empty()) continue;
        if (fr->work.size() + items.size() > c.caps.work_capacity) { fr->overflow |= 8u; continue; }
        fiber_raster_tile_run run{(uint32_t)fr->work.size(), (uint32_t)items.size(), f, screen_tile, load, 0, 0, 0};
        fr->work.insert(fr->work.end(), items.begin(), items.end());
        (d.kind == 1u ? sh : cam).push_back(run);
    }
    fr->runs = cam;
    fr->runs.insert(fr->runs.end(), sh.begin(), sh.end());
    fr->camera_runs = (uint32_t)cam.size();
    fr->shadow_runs = (uint32_t)sh.size();
}

// ---- segment fetch (get_segment_vertices_from_index_unchecked, strand_rasterizer.wgsl:289-303)
inline void segment_world(const fref_instance* in, uint32_t seg, V4& w0, V4& w1) {
    uint32_t i0 = in->indices[seg], i1 = in->indices[seg + 1u];
    const float* a = in->vertices4 + 4ull * i0;
    const float* b = in->vertices4 + 4ull * i1;
    w0 = matvec(in->world_from_local, V4{a[0], a[1], a[2], 1.0f});
    w1 = matvec(in->world_from_local, V4{b[0], b[1], b[2], 1.0f});
}

// fragment_position_line_relative (strand_rasterizer.wgsl:138-147)
inline float line_t(V2 p, V2 a, V2 b) {
    V2 ab{b.x - a.x, b.y - a.y};
    float l2 = dot2(ab, ab);
    if (l2 == 0.0f) return 0.0f;
    V2 pa{p.x - a.x, p.y - a.y};
    return dot2(pa, ab) / l2;
}

// ---- K16 deep shadow raster (strand_rasterizer.wgsl:391-711) + K17 stampback
struct ShadowRef { bool valid; V3 p0, p1; float rmin, rmax, absorb; };

void stage_shadow(Ctx& c) {
    fref_frame* fr = c.fr;
    const uint32_t K = fr->K, D = fr->D;
    fr->dom_depth.assign((size_t)fr->L * D * D, 0.0f);
    fr->dom_opacity.assign((size_t)fr->L * K * D * D, 0.0f);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t r = 0; r < (int64_t)fr->shadow_runs; ++r) {
        const auto& run = fr->runs[fr->camera_runs + r];
        if (run.work_count == 0u) continue;
        uint32_t f = run.frustum_id;
        const auto& d = fr->frusta[f];
        uint32_t layer = light_layer(fr, f);
        if (layer == kInvalid) continue;
        const float* clip = fr->clip[f];
        float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
        uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x);
        uint32_t tx = run.screen_tile_id % ftx, ty = run.screen_tile_id / ftx;
        uint32_t tile_px = d.froxel_size_x * d.froxel_size_y;
        // Stage every reference of the run once (the workgroup batches hold the same values).
        std::vector<std::vector<ShadowRef>> items(run.work_count);
        for (uint32_t w = 0; w < run.work_count; ++w) {
            const auto& wi = fr->work[run.work_base + w];
            bool valid_item = wi.frustum_id == f && wi.screen_tile_id == run.screen_tile_id;
            items[w].resize(wi.seg_ref_count);
            for (uint32_t j = 0; j < wi.seg_ref_count; ++j) {
                ShadowRef& s = items[w][j];
                s.valid = false;
                if (!valid_item) continue;
                const auto& ref = fr->refs[wi.seg_ref_base + j];
                const fref_instance* in = c.inst[ref.inst_id].src;
                V4 w0, w1;
                segment_world(in, ref.seg_id, w0, w1);
                V4 r0 = world_to_screen_raw(w0, clip, vw, vh), r1 = world_to_screen_raw(w1, clip, vw, vh);
                const fiber_strand_material& m = in->materials[ref.material_idx];
                s.p0 = v3(r0.x, r0.y, normalize_depth01(r0.z));
                s.p1 = v3(r1.x, r1.y, normalize_depth01(r1.z));
                s.rmin = wmax(m.min_radius_pixels, 1e-4f);
                s.rmax = wmax(m.max_radius_pixels, s.rmin);
                s.absorb = m.absorption_color[3];
                s.valid = true;
            }
        }
        for (uint32_t slot = 0; slot < kPixelSlots; ++slot) {
            if (slot >= tile_px) continue;
            uint32_t px = tx * d.froxel_size_x + slot % d.froxel_size_x;
            uint32_t py = ty * d.froxel_size_y + slot / d.froxel_size_x;
            if (px >= d.screen_width || py >= d.screen_height) continue;
            V2 pf{u2f(px) + 0.5f, u2f(py) + 0.5f};
            const float opaque = 0.0f;  // no opaque directional shadow map bound
            // Pass 1: nearest depth, stopping after the first work item with a hit.
            float z0 = -1.0f;
            bool found = false;
            for (uint32_t w = 0; w < run.work_count && !found; ++w) {
                bool hit = false;
                for (const ShadowRef& s : items[w]) {
                    if (!s.valid) continue;
                    float t = line_t(pf, V2{s.p0.x, s.p0.y}, V2{s.p1.x, s.p1.y});
                    if (t < 0.0f || t > 1.0f) continue;
                    V3 p = mix3(s.p0, s.p1, t);
                    // in_front_of_opaque_shadow_depth (:371-377) with opaque depth 0
                    float rr = wmix(s.rmin, s.rmax, wclamp(p.z, 0.0f, 1.0f));
                    V2 dd{pf.x - p.x, pf.y - p.y};
                    float cov = wclamp(1.0f - std::sqrt(dot2(dd, dd)) / rr, 0.0f, 1.0f);
                    if (cov > 0.0f) { z0 = wmax(z0, p.z); hit = true; }
                }
                if (hit) found = true;
            }
            size_t dom_px = (size_t)py * D + px;
            if (!found && opaque <= 0.0f) {
                fr->dom_depth[(size_t)layer * D * D + dom_px] = 0.0f;
                for (uint32_t i = 0; i < K; ++i) fr->dom_opacity[((size_t)layer * K + i) * D * D + dom_px] = 0.0f;
                continue;
            }
            if (!found) z0 = opaque;
            // Pass 2: opacity partials per depth worker (strided batch entries).
            float inv_span = 1.0f / wmax(1e-6f, z0);
            std::vector<float> partial((size_t)kShadowWorkers * K, 0.0f);
            for (uint32_t w = 0; w < run.work_count; ++w) {
                const auto& refs = items[w];
                uint32_t n = (uint32_t)refs.size();
                for (uint32_t bb = 0; bb < n; bb += kShadowBatch) {
                    uint32_t bc = std::min(kShadowBatch, n - bb);
                    for (uint32_t wk = 0; wk < kShadowWorkers; ++wk) {
                        for (uint32_t bi = wk; bi < bc; bi += kShadowWorkers) {
                            const ShadowRef& s = refs[bb + bi];
                            if (!s.valid) continue;
                            float t = line_t(pf, V2{s.p0.x, s.p0.y}, V2{s.p1.x, s.p1.y});
                            if (t < 0.0f || t > 1.0f) continue;
                            V3 p = mix3(s.p0, s.p1, t);
                            float rr = wmix(s.rmin, s.rmax, wclamp(p.z, 0.0f, 1.0f));
                            V2 dd{pf.x - p.x, pf.y - p.y};
                            float cov = wclamp(1.0f - std::sqrt(dot2(dd, dd)) / rr, 0.0f, 1.0f);
                            if (cov <= 0.0f) continue;
                            float dzp = wmax(0.0f, z0 - p.z) * inv_span;
                            float u = wclamp(dzp, 0.0f, 1.0f);  // pow(u, DOM_GAMMA = 1)
                            float tl = u * u2f(K);
                            uint32_t si = std::min(f2u(std::floor(tl)), K - 1u);
                            float wf = wfract(tl);
                            float a = cov * s.absorb * 0.5f;
                            float* pp = &partial[(size_t)wk * K];
                            float a0 = pp[si];
                            pp[si] = wclamp(a0 + (1.0f - a0) * (1.0f - wf) * a, 0.0f, 1.0f);
                            if (si + 1u < K) {
                                float a1 = pp[si + 1u];
                                pp[si + 1u] = wclamp(a1 + (1.0f - a1) * wf * a, 0.0f, 1.0f);
                            }
                        }
                    }
                }
            }
            fr->dom_depth[(size_t)layer * D * D + dom_px] = z0;
            float acc = 0.0f;
            uint32_t terminal = K;  // opaque_terminal_slice with no opaque depth
            for (uint32_t i = 0; i < K; ++i) {
                float a = 0.0f;
                for (uint32_t wk = 0; wk < kShadowWorkers; ++wk) a = a + (1.0f - a) * partial[(size_t)wk * K + i];
                acc = acc + (1.0f - acc) * a;
                if (i >= terminal) acc = 1.0f;
                fr->dom_opacity[((size_t)layer * K + i) * D * D + dom_px] = acc;
            }
        }
    }
    // K17 stampback (shadow_dom_stampback.wgsl:74-123): max DOM depth over the
    // DOM texels each target texel covers; target cleared to 0.
    const uint32_t S = fr->S;
    fr->shadow_map.assign((size_t)fr->L * S * S, 0.0f);
    for (uint32_t l = 0; l < fr->L; ++l) {
        uint32_t f = kInvalid;
        for (uint32_t i = 0, layer = 0; i < fr->F; ++i) {
            if (fr->frusta[i].kind != 1u) continue;
            if (layer == l) { f = i; break; }
            ++layer;
        }
        if (f == kInvalid) continue;
        const auto& d = fr->frusta[f];
#pragma omp parallel for schedule(static)
        for (int64_t y = 0; y < (int64_t)S; ++y) {
            for (uint32_t x = 0; x < S; ++x) {
                uint32_t mnx = std::min((x * d.screen_width) / S, d.screen_width - 1u);
                uint32_t mny = std::min(((uint32_t)y * d.screen_height) / S, d.screen_height - 1u);
                uint32_t mxx = std::min(((x + 1u) * d.screen_width + S - 1u) / S, d.screen_width);
                uint32_t mxy = std::min((((uint32_t)y + 1u) * d.screen_height + S - 1u) / S, d.screen_height);
                float z = 0.0f;
                for (uint32_t yy = mny; yy < mxy; ++yy)
                    for (uint32_t xx = mnx; xx < mxx; ++xx)
                        z = wmax(z, fr->dom_depth[(size_t)l * D * D + (size_t)yy * D + xx]);
                if (z <= 0.0f) continue;
                fr->shadow_map[(size_t)l * S * S + (size_t)y * S + x] = z;
            }
        }
    }
}

// ---- K18 shading (strand_shading.wgsl:173-695) -------------------------------
// Gauss-Legendre n = 10 nodes/weights (shading_LUTs.wgsl LEG_*_10), regenerated
// with numpy.polynomial.legendre.leggauss(10) and rounded to binary32.
const float kLegRoots[10] = {-9.739065170e-01f, -8.650633693e-01f, -6.794095635e-01f, -4.333953857e-01f,
                             -1.488743424e-01f, 1.488743424e-01f,  4.333953857e-01f,  6.794095635e-01f,
                             8.650633693e-01f,  9.739065170e-01f};
const float kLegWeights[10] = {6.667134166e-02f, 1.494513452e-01f, 2.190863639e-01f, 2.692667246e-01f,
                               2.955242395e-01f, 2.955242395e-01f, 2.692667246e-01f, 2.190863639e-01f,
                               1.494513452e-01f, 6.667134166e-02f};
const float kFactorials[10] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880};

float sample_dom(const fref_frame* fr, V3 pw, uint32_t layer, const fiber_light* lights) {
    uint32_t f = kInvalid;
    for (uint32_t i = 0, l = 0; i < fr->F; ++i) {
        if (fr->frusta[i].kind != 1u) continue;
        if (l == layer) { f = i; break; }
        ++l;
    }
    if (f == kInvalid) return 1.0f;
    const auto& d = fr->frusta[f];
    float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
    V4 raw = world_to_screen_raw(V4{pw.x, pw.y, pw.z, 1.0f}, lights[layer].clip_from_world, vw, vh);
    if (raw.x < 0.0f || raw.y < 0.0f || raw.x >= vw || raw.y >= vh || raw.z < 0.0f || raw.z > 1.0f) return 1.0f;
    uint32_t px = f2u(raw.x), py = f2u(raw.y);
    const uint32_t D = fr->D, K = fr->K;
    float z0 = fr->dom_depth[(size_t)layer * D * D + (size_t)py * D + px];
    if (z0 <= 0.0f) return 1.0f;
    float z = normalize_depth01(raw.z);
    if (z > z0 - 1e-3f) return 1.0f;
    float u = wclamp(wmax(0.0f, z0 - z) / wmax(z0, 1e-6f), 0.0f, 1.0f);  // pow(., DOM_GAMMA = 1)
    float sf = u * u2f(K);
    uint32_t slice = std::min(f2u(std::floor(sf)), std::min(K, K) - 1u);
    float op = fr->dom_opacity[((size_t)layer * K + slice) * D * D + (size_t)py * D + px];
    return wclamp(1.0f - op, 0.08f, 1.0f);
}

float fresnel_reflectance(float eta_i, float eta_t, float cos_theta_i) {
    float ci = std::fabs(cos_theta_i);
    float cic = wclamp(0.0f, 1.0f, ci);  // clamp(0.0, 1.0, x) = min(max(0, 1), x)
    float sin_i_sq = 1.0f - cic * cic;
    float ratio = eta_i / eta_t;
    float sin_t_sq = ratio * ratio * sin_i_sq;
    float cos_t = std::sqrt(1.0f - sin_t_sq);
    float rpar = ((eta_t * ci) - (eta_i * cos_t)) / ((eta_t * ci) + (eta_i * cos_t));
    float rper = ((eta_i * ci) - (eta_t * cos_t)) / ((eta_i * ci) + (eta_t * cos_t));
    return (rpar * rpar + rper * rper) * 0.5f;
}

V3 attenuation(uint32_t p, float h_, float eta, float eta_prime, V3 mu, float theta_d) {
    float h = wclamp(-1.0f + 1e-6f, 1.0f - 1e-6f, h_);  // = min(1 - 1e-6, h_)
    float gamma_t = std::asin(h / eta_prime);
    float gamma_i = std::asin(h);
    float f = fresnel_reflectance(1.0f, eta, std::acos(std::cos(theta_d) * std::cos(gamma_i)));
    float c2 = 1.0f + std::cos(2.0f * gamma_t);
    V3 T = v3(std::exp(-2.0f * mu.x * c2), std::exp(-2.0f * mu.y * c2), std::exp(-2.0f * mu.z * c2));
    if (p == 0u) return v3(f * T.x * T.x, f * T.y * T.y, f * T.z * T.z);
    float f_ = 1.0f - f;
    float fp = std::pow(f, u2f(p - 1u));
    float k = (f_ * f_) * fp;
    return v3(k * std::pow(T.x, u2f(p)), k * std::pow(T.y, u2f(p)), k * std::pow(T.z, u2f(p)));
}

float gaussian_detector(float beta, float phi_delta, uint32_t k_limit) {
    float var = beta * beta;
    if (var < 1e-6f) {
        float two_pi = 2.0f * kPi;
        float m = phi_delta - two_pi * std::trunc(phi_delta / two_pi);
        return std::fabs(m) < 1e-3f ? 0.0f : 1e6f;  // select(1e6, 0.0, cond)
    }
    float norm = 1.0f / (std::sqrt(2.0f * kPi) * beta);
    float total = 0.0f;
    int32_t ik = (int32_t)k_limit;
    for (int32_t k = -ik; k <= ik; ++k) {
        float angle = phi_delta - 2.0f * kPi * (float)k;
        total = total + std::exp(-angle * angle / (2.0f * var));
    }
    return norm * total;
}

float phi_shift(uint32_t p, float h_, float eta_prime) {
    float h = wclamp(-1.0f + 1e-6f, 1.0f - 1e-6f, h_);
    float gamma_t = std::asin(wclamp(h / eta_prime, -1.0f, 1.0f));
    return 2.0f * u2f(p) * gamma_t - 2.0f * std::asin(h) + u2f(p) * kPi;
}

float bessel_first(float x, uint32_t steps) {
    float y = 0.0f;
    for (uint32_t i = 0; i < steps; ++i) {
        float num = std::pow(x, 2.0f * u2f(i));
        float den = std::pow(4.0f, u2f(i)) * kFactorials[i] * kFactorials[i];
        y = y + num / den;
    }
    return y;
}

float Mp(float v, float theta_i_, float theta_r, float alpha) {
    float trs = theta_r + alpha;
    float ti = wclamp(-kPiHalf + 1e-6f, kPiHalf - 1e-6f, theta_i_);
    trs = wclamp(-kPiHalf + 1e-6f, kPiHalf - 1e-6f, trs);
    float cti = std::cos(-ti), ctr = std::cos(trs), sti = std::sin(-ti), strs = std::sin(trs);
    if (v < 1e-6f) {
        float tol = 0.1f * (kPi / 180.0f);
        return std::fabs(trs + ti) < tol ? 0.0f : 1e6f / tol;
    }
    float bessel_arg = (cti * ctr) / v;
    float exp_arg = (sti * strs) / v;
    return bessel_first(bessel_arg, 5u) * std::exp(exp_arg);
}

V3 Np(uint32_t p, float phi, float theta_i, float theta_r, float eta, V3 mu, float beta) {
    float theta_d = (theta_r - theta_i) * 0.5f;
    float sti = std::sin(theta_i);
    float ctd = std::cos(theta_d);
    float arg_sq = eta * eta - sti * sti;
    float eta_prime = std::sqrt(wmax(0.0f, arg_sq)) / ctd;
    V3 mup = v3(mu.x / ctd, mu.y / ctd, mu.z / ctd);
    V3 acc = v3(0, 0, 0);
    for (uint32_t i = 0; i < 10u; ++i) {
        V3 A = attenuation(p, kLegRoots[i], eta, eta_prime, mup, theta_d);
        float det = gaussian_detector(beta, phi - phi_shift(p, kLegRoots[i], eta_prime), 10u);
        acc = add3(acc, mul3s(mul3s(A, det), kLegWeights[i]));
    }
    return mul3s(acc, 0.5f);
}

V3 marschner(V3 L, V3 V, V3 U, const fiber_strand_material& m, float occlusion) {
    // marschner(point, direction = L, view_normal = V, light_normal = U) (:579-605, call :686)
    float theta_i = std::acos(dot3(L, U));
    float theta_r = std::acos(dot3(L, V));
    V3 lp = normalize3(sub3(U, mul3s(L, dot3(U, L))));
    V3 vp = normalize3(sub3(V, mul3s(L, dot3(V, L))));
    float ang = std::acos(dot3(normalize3(lp), normalize3(vp)));
    float sdot = dot3(cross3(lp, vp), L);
    float phi = ang * (sdot > 0.0f ? 1.0f : (sdot < 0.0f ? -1.0f : 0.0f));
    V3 sigma = v3(1.0f - m.absorption_color[0], 1.0f - m.absorption_color[1], 1.0f - m.absorption_color[2]);
    float v_long = m.alpha * m.alpha;
    float v_azim = m.beta * m.beta;
    float beta_azim = std::sqrt(v_azim);
    float vis = wclamp(1.0f - occlusion, 0.0f, 1.0f);
    float direct = wmix(0.18f, 1.0f, vis);
    float mp = Mp(v_long, theta_i, theta_r, m.shift);
    V3 total = v3(mp * m.specular_color[0] * m.specular_color[3] * direct,
                  mp * m.specular_color[1] * m.specular_color[3] * direct,
                  mp * m.specular_color[2] * m.specular_color[3] * direct);
    for (uint32_t p = 0; p < 3u; ++p) {
        V3 n = Np(p, phi, theta_i, theta_r, m.eta, sigma, beta_azim);
        total = add3(total, mul3s(n, (u2f(p + 1u) * vis) / 3.0f));
    }
    return total;
}

void stage_shading(Ctx& c, const uint16_t* history_prev) {
    fref_frame* fr = c.fr;
    const uint32_t cap = fr->atlas_cap;
    fr->atlas.assign((size_t)fr->I * cap * 4, 0);
    fr->history.assign((size_t)fr->I * cap * 2, 0);
    const uint32_t n = fr->n_cam_tasks;  // camera frustum 0 owns tasks [0, n)
    const float* cp = c.cam->world_position;
    uint32_t nl = std::min(fr->L, 4u);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)n; ++k) {
        const fiber_binning_task& t = fr->tasks[k];
        uint32_t inst = t.id_info;
        const fref_instance* in = c.inst[inst].src;
        const fiber_strand_meta& m = in->meta[t.chunk_id];
        uint32_t seg = t.seg_idx;
        V4 v0, v1;
        segment_world(in, seg, v0, v1);
        V3 U = normalize3(v3(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z));
        V3 cam_dir = normalize3(v3(cp[0] - v0.x, cp[1] - v0.y, cp[2] - v0.z));
        V3 binormal = normalize3(cross3(U, cam_dir));
        V3 V = normalize3(cross3(binormal, U));
        const fiber_strand_material& mat = in->materials[m.material_idx];
        float accum[4] = {0.0f, 0.0f, 0.0f, mat.absorption_color[3]};
        uint32_t atlas_idx = m.offset + (seg - m.offset);
        V3 mid = mix3(v3(v0.x, v0.y, v0.z), v3(v1.x, v1.y, v1.z), 0.5f);
        float cur = 1.0f;
        if (nl != 0u) {
            float vis = 0.0f;
            for (uint32_t l = 0; l < nl; ++l) vis = vis + sample_dom(fr, mid, l, c.lights);
            cur = vis / u2f(nl);
        }
        size_t hidx = (size_t)inst * cap + atlas_idx;
        float prev = history_prev ? from_half_bits(history_prev[hidx * 2]) : 0.0f;
        float vis = prev > 0.0f ? wmix(cur, prev, 0.88f) : cur;
        fr->history[hidx * 2 + 0] = to_half_bits(vis);
        fr->history[hidx * 2 + 1] = to_half_bits(cur);
        float occ = 1.0f - vis;
        const float* amb = c.st->ambient_color;
        for (uint32_t j = 0; j < fr->L; ++j) {
            const fiber_light& lt = c.lights[j];
            V3 L = normalize3(v3(lt.direction_to_light[0], lt.direction_to_light[1], lt.direction_to_light[2]));
            V3 b = marschner(L, V, U, mat, occ);
            float cc[3] = {b.x * (lt.color[0] / 255.0f), b.y * (lt.color[1] / 255.0f), b.z * (lt.color[2] / 255.0f)};
            for (int q = 0; q < 3; ++q) {
                float ambient = mat.absorption_color[q] * mat.ambient_factor + (amb[q] / 255.0f) * mat.ambient_factor;
                cc[q] = wmix(cc[q], ambient, mat.ambient_factor);
                accum[q] = accum[q] + cc[q];
            }
        }
        // Rgba8Unorm storage semantics without the 8-bit rounding: clamp to [0, 1].
        uint16_t hv[4];
        for (int q = 0; q < 4; ++q) hv[q] = to_half_bits(wclamp(accum[q], 0.0f, 1.0f));
        size_t a0 = (size_t)inst * cap + atlas_idx;
        for (int q = 0; q < 4; ++q) fr->atlas[a0 * 4 + q] = hv[q];
        // Texel seg + 1: written unless the next camera task shades it (canonical
        // resolution of the reference's seg/seg+1 write race, :692-694).
        bool next_shades = (k + 1 < (int64_t)n) && fr->tasks[k + 1].id_info == inst &&
                           fr->tasks[k + 1].seg_idx == seg + 1u;
        if (!next_shades && atlas_idx + 1u < cap)
            for (int q = 0; q < 4; ++q) fr->atlas[(a0 + 1) * 4 + q] = hv[q];
    }
}

// ---- K19 camera colour raster (strand_rasterizer.wgsl:855-1044) --------------
struct ColorRef {
    bool valid;
    V2 p0, ab, mn, mx;
    float inv_len_sq, z0, z1, w0, w1, rmin, rmax;
    float s0[4], s1[4], vis;
};
struct RGBA { float r, g, b, a; };
inline RGBA over(RGBA fg, RGBA bg) {
    float oma = 1.0f - fg.a;
    return RGBA{fg.r + bg.r * oma, fg.g + bg.g * oma, fg.b + bg.b * oma, fg.a + bg.a * oma};
}
inline float persp_t(float t, float w0, float w1) {
    float aw0 = wmax(std::fabs(w0), 1e-6f), aw1 = wmax(std::fabs(w1), 1e-6f);
    float denom = (1.0f - t) * aw1 + t * aw0;
    return (t * aw0) / denom;
}

void stage_raster(Ctx& c) {
    fref_frame* fr = c.fr;
    const uint32_t W = fr->W, H = fr->H;
    fr->color.assign((size_t)W * H * 4, 0);
    fr->depth.assign((size_t)W * H, 0.0f);
    fr->fragments.assign((size_t)W * H, 0u);
    const uint32_t cap = fr->atlas_cap;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t r = 0; r < (int64_t)fr->camera_runs; ++r) {
        const auto& run = fr->runs[r];
        if (run.work_count == 0u) continue;
        uint32_t f = run.frustum_id;
        const auto& d = fr->frusta[f];
        const float* clip = fr->clip[f];
        float vw = u2f(d.screen_width), vh = u2f(d.screen_height);
        uint32_t ftx = ceil_div(d.screen_width, d.froxel_size_x);
        uint32_t tx = run.screen_tile_id % ftx, ty = run.screen_tile_id / ftx;
        uint32_t tile_px = d.froxel_size_x * d.froxel_size_y;
        std::vector<std::vector<ColorRef>> items(run.work_count);
        for (uint32_t w = 0; w < run.work_count; ++w) {
            const auto& wi = fr->work[run.work_base + w];
            items[w].resize(wi.seg_ref_count);
            for (uint32_t j = 0; j < wi.seg_ref_count; ++j) {
                ColorRef& s = items[w][j];
                s.valid = false;
                const auto& ref = fr->refs[wi.seg_ref_base + j];
                const fref_instance* in = c.inst[ref.inst_id].src;
                V4 w0, w1;
                segment_world(in, ref.seg_id, w0, w1);
                V4 a = world_to_screen_raw(w0, clip, vw, vh), b = world_to_screen_raw(w1, clip, vw, vh);
                if (a.x < 0.0f && b.x < 0.0f) continue;
                const fiber_strand_material& m = in->materials[ref.material_idx];
                float rmin = wmax(m.min_radius_pixels, 1e-4f);
                float rmax = wmax(m.max_radius_pixels, rmin);
                uint32_t i0 = ref.seg_id, i1 = std::min(i0 + 1u, cap - 1u);
                s.valid = true;
                s.p0 = V2{a.x, a.y};
                s.ab = V2{b.x - a.x, b.y - a.y};
                s.inv_len_sq = 1.0f / dot2(s.ab, s.ab);
                s.z0 = a.z; s.z1 = b.z; s.w0 = a.w; s.w1 = b.w;
                s.rmin = rmin; s.rmax = rmax;
                s.mn = V2{wmin(a.x, b.x) - rmax, wmin(a.y, b.y) - rmax};
                s.mx = V2{wmax(a.x, b.x) + rmax, wmax(a.y, b.y) + rmax};
                size_t t0 = (size_t)ref.inst_id * cap + i0, t1 = (size_t)ref.inst_id * cap + i1;
                for (int q = 0; q < 4; ++q) {
                    s.s0[q] = from_half_bits(fr->atlas[t0 * 4 + q]);
                    s.s1[q] = from_half_bits(fr->atlas[t1 * 4 + q]);
                }
                s.vis = from_half_bits(fr->history[t0 * 2]);
            }
        }
        for (uint32_t slot = 0; slot < kPixelSlots; ++slot) {
            uint32_t px = tx * d.froxel_size_x + slot % d.froxel_size_x;
            uint32_t py = ty * d.froxel_size_y + slot / d.froxel_size_x;
            bool active = slot < tile_px && px < d.screen_width && py < d.screen_height;
            if (!active) continue;
            V2 pc{u2f(px) + 0.5f, u2f(py) + 0.5f};
            RGBA fin{0, 0, 0, 0};
            float gdepth = 0.0f;
            bool done = false;
            uint32_t frags = 0;
            for (uint32_t w = 0; w < run.work_count && !done; ++w) {
                const auto& refs = items[w];
                uint32_t n = (uint32_t)refs.size();
                for (uint32_t bb = 0; bb < n; bb += kColorBatch) {
                    for (uint32_t g = 0; g < kColorBatch; g += kColorWorkers) {
                        RGBA part[4] = {};
                        float pd[4] = {0, 0, 0, 0};
                        for (uint32_t wk = 0; wk < kColorWorkers; ++wk) {
                            uint32_t bi = bb + g + wk;
                            if (bi >= n) continue;
                            const ColorRef& s = refs[bi];
                            if (!s.valid) continue;
                            if (pc.x < s.mn.x || pc.y < s.mn.y || pc.x > s.mx.x || pc.y > s.mx.y) continue;
                            V2 pa{pc.x - s.p0.x, pc.y - s.p0.y};
                            float t = dot2(pa, s.ab) * s.inv_len_sq;
                            if (!(t >= 0.0f && t <= 1.0f)) continue;
                            V2 pfr{s.p0.x + s.ab.x * t, s.p0.y + s.ab.y * t};
                            float pz = wmix(s.z0, s.z1, t);
                            float rmin = wmax(s.rmin, 1e-4f);
                            float rr = wmix(rmin, wmax(s.rmax, rmin), wclamp(normalize_depth01(pz), 0.0f, 1.0f));
                            V2 dl{pc.x - pfr.x, pc.y - pfr.y};
                            float d2 = dot2(dl, dl);
                            if (!(d2 < rr * rr)) continue;
                            float cov = wclamp(1.0f - std::sqrt(d2) / rr, 0.0f, 1.0f);
                            float tw = persp_t(t, s.w0, s.w1);
                            float sh[4];
                            for (int q = 0; q < 4; ++q) sh[q] = wmix(s.s0[q], s.s1[q], tw);
                            float alpha = sh[3] * cov;
                            part[wk] = RGBA{sh[0] * s.vis * alpha, sh[1] * s.vis * alpha, sh[2] * s.vis * alpha, alpha};
                            pd[wk] = pz;
                            ++frags;
                        }
                        RGBA p01 = over(part[0], part[1]), p23 = over(part[2], part[3]);
                        float d01 = wmax(pd[0], pd[1]), d23 = wmax(pd[2], pd[3]);
                        fin = over(fin, over(p01, p23));
                        gdepth = wmax(gdepth, wmax(d01, d23));
                    }
                }
                if (fin.a > 0.98f) {
                    fin = RGBA{fin.r / fin.a, fin.g / fin.a, fin.b / fin.a, 1.0f};
                    done = true;
                }
            }
            RGBA o = fin;
            if (o.a > 1e-6f && o.a < 1.0f) o = RGBA{o.r / o.a, o.g / o.a, o.b / o.a, o.a};
            size_t pi = (size_t)py * W + px;
            fr->color[pi * 4 + 0] = to_half_bits(o.r);
            fr->color[pi * 4 + 1] = to_half_bits(o.g);
            fr->color[pi * 4 + 2] = to_half_bits(o.b);
            fr->color[pi * 4 + 3] = to_half_bits(o.a);
            fr->depth[pi] = gdepth;
            fr->fragments[pi] = frags;
        }
    }
}

// ---- finalize_telemetry (strand_prepass.wgsl:2145-2188) ----------------------
// The fiber_telemetry image: totals, the candidate statistics of every
// allocated page, and per frustum the visibility / retention counts, tasks,
// pages, candidates, references and the load of the tile runs with work.
void stage_telemetry(Ctx& c) {
    fref_frame* fr = c.fr;
    const uint32_t kHist = 8, kFr = 40, kStride = 11;
    std::vector<uint32_t>& t = fr->telemetry;
    t.assign(kFr + 16 * kStride, 0u);
    auto F = [&](uint32_t f, uint32_t field) -> uint32_t& { return t[kFr + f * kStride + field]; };
    t[0] = (uint32_t)fr->page_meta.size();
    t[1] = (uint32_t)fr->tasks.size();
    t[3] = (uint32_t)fr->refs_tail;
    t[6] = fr->F;
    for (uint32_t f = 0; f < fr->F && f < 16u; ++f) {
        F(f, 0) = fr->tel_visible_instances[f];
        F(f, 1) = fr->tel_visible_strands[f];
        F(f, 2) = fr->tel_retained[f];
        F(f, 3) = fr->frustum_task_base[f + 1] - fr->frustum_task_base[f];
    }
    for (size_t p = 0; p < fr->page_meta.size(); ++p) {
        const auto& pm = fr->page_meta[p];
        const uint32_t f = frustum_for_tile(fr, pm.coarse_tile_id);
        if (f != kInvalid) F(f, 4) += 1u;
        const uint32_t cand = fr->page_candidates[p];
        if (cand == 0u) continue;
        t[2] += cand;
        t[4] += 1u;
        t[5] = std::max(t[5], cand);
        uint32_t bin = 0, rem = cand;
        while (rem > 1u && bin + 1u < 32u) { rem >>= 1u; ++bin; }
        t[kHist + bin] += 1u;
        if (f != kInvalid) {
            F(f, 5) += cand;
            F(f, 6) += pm.seg_ref_count;
            F(f, 9) = std::max(F(f, 9), cand);
        }
    }
    for (const auto& run : fr->runs) {
        if (run.work_count == 0u || run.frustum_id >= fr->F) continue;
        F(run.frustum_id, 7) += 1u;
        F(run.frustum_id, 8) += run.load_score;
        F(run.frustum_id, 10) = std::max(F(run.frustum_id, 10), run.load_score);
    }
}

// ---- K20 composite (strand_composite.wgsl:12-33 + ALPHA_BLENDING) -----------
// One pixel. The fragment shader's output is `scene` where the scene depth is
// in front of the strand depth, else mix(scene.rgb, strand.rgb, strand.a) with
// the scene's alpha (strand_composite.wgsl:23-32). The colour target blends it
// with BlendState::ALPHA_BLENDING (src/pipelines/composite.rs:115-124) onto
// the destination loaded with LoadOp::Load (src/nodes/composite.rs:102-118):
// rgb = src.rgb * src.a + dst.rgb * (1 - src.a), a = src.a * 1 + dst.a * (1 - src.a).
// The destination is post_process_write().destination, an image of its own;
// it equals the scene colour only when the pass composites in place.
void composite_pixel(const float* sc, float sd, const float* st, float strand_depth, const float* dst, float* out) {
    float frag[4];
    if (sd > strand_depth) {
        for (int q = 0; q < 4; ++q) frag[q] = sc[q];
    } else {
        for (int q = 0; q < 3; ++q) frag[q] = wmix(sc[q], st[q], st[3]);
        frag[3] = sc[3];
    }
    const float oma = 1.0f - frag[3];
    for (int q = 0; q < 3; ++q) out[q] = frag[q] * frag[3] + dst[q] * oma;
    out[3] = frag[3] * 1.0f + dst[3] * oma;
}

// The frame's composite over one scene image. dest: the destination's
// contents before the pass (NULL = the scene colour, compositing in place);
// half_out rounds every channel to binary16 (an RGBA16F target).
void composite_image(const fref_frame* fr, const float* scene_color, const float* scene_depth, const float* dest,
                     bool half_out, float* out) {
    const size_t n = (size_t)fr->W * fr->H;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float* sc = scene_color + 4 * i;
        const float sd = scene_depth ? scene_depth[i] : 0.0f;
        float st[4];
        for (int q = 0; q < 4; ++q) st[q] = from_half_bits(fr->color[i * 4 + q]);
        float o[4];
        composite_pixel(sc, sd, st, fr->depth[i], dest ? dest + 4 * i : sc, o);
        for (int q = 0; q < 4; ++q) out[i * 4 + q] = half_out ? from_half_bits(to_half_bits(o[q])) : o[q];
    }
}

void stage_composite(Ctx& c, const float* scene_color, const float* scene_depth) {
    fref_frame* fr = c.fr;
    const size_t n = (size_t)fr->W * fr->H;
    fr->composite.assign(n * 4, 0.0f);
    if (!scene_color) return;
    composite_image(fr, scene_color, scene_depth, nullptr, true, fr->composite.data());
}

// Frustum table (use_prepass_buffers, src/plugin.rs:386-482): camera first,
// then the lights in order.
void build_frusta(fref_frame* fr, const fiber_froxel_config* cam_cfg, const fiber_froxel_config* lcfg,
                  uint32_t n_lights) {
    uint32_t bucket = 0, coarse = 0, fine = 0;
    for (uint32_t f = 0; f < 1u + n_lights; ++f) {
        const fiber_froxel_config& cfg = f == 0 ? *cam_cfg : lcfg[f - 1];
        uint32_t tx = ceil_div(cfg.screen_width, cfg.froxel_size_x);
        uint32_t ty = ceil_div(cfg.screen_height, cfg.froxel_size_y);
        uint32_t ctx_ = std::max(1u, ceil_div(tx, kCoarseExtent));
        uint32_t cty = std::max(1u, ceil_div(ty, kCoarseExtent));
        fiber_frustum_desc d{};
        d.screen_width = cfg.screen_width;
        d.screen_height = cfg.screen_height;
        d.froxel_size_x = cfg.froxel_size_x;
        d.froxel_size_y = cfg.froxel_size_y;
        d.depth_slices = cfg.depth_slices;
        d.bucket_base = bucket;
        d.bucket_count = tx * ty * cfg.depth_slices;
        d.kind = f == 0 ? 0u : 1u;
        d.coarse_depth_tile_base = coarse;
        d.coarse_depth_tile_count = ctx_ * cty;
        d.coarse_tiles_x = ctx_;
        d.coarse_tiles_y = cty;
        d.cascade_index = 0;
        d.fine_depth_tile_base = fine;
        fr->frusta.push_back(d);
        bucket += d.bucket_count;
        coarse += d.coarse_depth_tile_count;
        fine += tx * ty;
    }
    fr->total_coarse_tiles = coarse;
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
uint64_t copy_out(const std::vector<T>& v, void* host, uint64_t cap) {
    uint64_t bytes = (uint64_t)v.size() * sizeof(T);
    if (host && cap >= bytes && bytes) std::memcpy(host, v.data(), bytes);
    return bytes;
}

}  // namespace

extern "C" {

fref_frame* fref_run(const fref_instance* inst, uint32_t n_inst, const fiber_froxel_config* camera_cfg,
                     const fiber_camera* camera, const fiber_froxel_config* light_cfgs,
                     const fiber_light* lights, uint32_t n_lights, const fiber_settings* settings,
                     const fref_capacities* caps, const uint16_t* history_prev,
                     const float* scene_color, const float* scene_depth, int threads) {
    return fref_run_opaque(inst, n_inst, camera_cfg, camera, light_cfgs, lights, n_lights, settings, caps,
                           history_prev, scene_color, scene_depth, nullptr, 0u, threads);
}

fref_frame* fref_run_opaque(const fref_instance* inst, uint32_t n_inst, const fiber_froxel_config* camera_cfg,
                            const fiber_camera* camera, const fiber_froxel_config* light_cfgs,
                            const fiber_light* lights, uint32_t n_lights, const fiber_settings* settings,
                            const fref_capacities* caps, const uint16_t* history_prev,
                            const float* scene_color, const float* scene_depth, const float* opaque_depth,
                            uint32_t opaque_samples, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    fref_frame* fr = new fref_frame();
    Ctx c;
    c.fr = fr;
    c.st = settings;
    c.cam = camera;
    c.lights = lights;
    c.caps = *caps;
    fr->I = n_inst;
    fr->L = n_lights;
    fr->K = std::max(1u, settings->dom_slices);
    build_frusta(fr, camera_cfg, light_cfgs, n_lights);
    fr->F = (uint32_t)fr->frusta.size();
    fr->clip.push_back(camera->clip_from_world);
    for (uint32_t l = 0; l < n_lights; ++l) fr->clip.push_back(lights[l].clip_from_world);
    uint32_t max_texels = 0;
    for (uint32_t i = 0; i < n_inst; ++i) {
        Inst in;
        in.src = &inst[i];
        in.strand_count = std::min(inst[i].n_meta, inst[i].geo.strand_count);
        c.inst.push_back(in);
        max_texels = std::max(max_texels, inst[i].n_indices);
        fr->total_points += inst[i].n_indices;
        for (uint32_t s = 0; s < inst[i].n_meta; ++s)
            if (inst[i].meta[s].count >= 2u) { fr->total_segments += inst[i].meta[s].count - 1u; fr->total_strands += 1; }
    }
    // Shading atlas dims (create_shading_target_texture, pipelines/shading.rs:410-438).
    fr->atlas_w = std::min(std::max(max_texels, 1u), kMaxTexture);
    fr->atlas_h = std::min(std::max(ceil_div(max_texels, fr->atlas_w), 1u), kMaxTexture);
    fr->atlas_cap = fr->atlas_w * fr->atlas_h;
    fr->range_valid.assign((size_t)n_inst * fr->F, 0u);
    fr->ranges.assign((size_t)n_inst * fr->F, fiber_coarse_asset_range{});
    fr->keep.assign((size_t)n_inst * fr->F, 0.0f);
    fr->inst_visible.assign(n_inst, 0u);
    fr->inst_strands.assign(n_inst, 0u);
    fr->inst_cam_keep.assign(n_inst, 0.0f);
    fr->inst_shadow_keep.assign(n_inst, 0.0f);
    fr->W = camera_cfg->screen_width;
    fr->H = camera_cfg->screen_height;
    fr->D = n_lights ? light_cfgs[0].screen_width : 0u;
    fr->S = n_lights ? (settings->shadow_map_size ? settings->shadow_map_size : fr->D) : 0u;

    double t0 = now_ms();
    stage_opaque(c, opaque_depth, std::max(1u, opaque_samples));
    stage_broad(c);
    stage_lut(c);
    double t1 = now_ms();
    stage_fine(c);
    double t2 = now_ms();
    stage_binning(c);
    double t3 = now_ms();
    stage_emit(c);
    stage_telemetry(c);
    double t4 = now_ms();
    stage_shadow(c);
    double t5 = now_ms();
    stage_shading(c, history_prev);
    double t6 = now_ms();
    stage_raster(c);
    stage_composite(c, scene_color, scene_depth);
    double t7 = now_ms();
    fr->stage_ms[0] = (float)(t1 - t0);
    fr->stage_ms[1] = (float)(t2 - t1);
    fr->stage_ms[2] = (float)(t3 - t2);
    fr->stage_ms[3] = (float)(t4 - t3);
    fr->stage_ms[4] = (float)(t5 - t4);
    fr->stage_ms[5] = (float)(t6 - t5);
    fr->stage_ms[6] = (float)(t7 - t6);
    fr->stage_ms[7] = (float)(t7 - t0);
    return fr;
}

uint64_t fref_get(const fref_frame* f, uint32_t what, void* host, uint64_t cap) {
    switch (what) {
        case FIBER_DUMP_FRUSTA: return copy_out(f->frusta, host, cap);
        case FIBER_DUMP_RANGES: {
            std::vector<uint32_t> v;
            for (size_t i = 0; i < f->ranges.size(); ++i) {
                v.push_back(f->range_valid[i]);
                const uint32_t* r = reinterpret_cast<const uint32_t*>(&f->ranges[i]);
                if (f->range_valid[i]) v.insert(v.end(), r, r + 8);
                else v.insert(v.end(), 8, 0u);
            }
            return copy_out(v, host, cap);
        }
        case FIBER_DUMP_KEEP: return copy_out(f->keep, host, cap);
        case FIBER_DUMP_LUT: return copy_out(f->lut, host, cap);
        case FIBER_DUMP_TASKS: return copy_out(f->tasks, host, cap);
        case FIBER_DUMP_PROJECTED: return copy_out(f->projected, host, cap);
        case FIBER_DUMP_PAGE_TABLE: return copy_out(f->page_table, host, cap);
        case FIBER_DUMP_PAGE_META: return copy_out(f->page_meta, host, cap);
        case FIBER_DUMP_COUNTS: return copy_out(f->counts, host, cap);
        case FIBER_DUMP_OFFSETS: return copy_out(f->offsets, host, cap);
        case FIBER_DUMP_REFS: return copy_out(f->refs, host, cap);
        case FIBER_DUMP_ACTIVE_TILES: return copy_out(f->active_tiles, host, cap);
        case FIBER_DUMP_WORK: return copy_out(f->work, host, cap);
        case FIBER_DUMP_RUNS: return copy_out(f->runs, host, cap);
        case FIBER_DUMP_DOM_DEPTH: return copy_out(f->dom_depth, host, cap);
        case FIBER_DUMP_DOM_OPACITY: return copy_out(f->dom_opacity, host, cap);
        case FIBER_DUMP_SHADOW_MAP: return copy_out(f->shadow_map, host, cap);
        case FIBER_DUMP_ATLAS: return copy_out(f->atlas, host, cap);
        case FIBER_DUMP_HISTORY: return copy_out(f->history, host, cap);
        case FIBER_DUMP_COLOR: return copy_out(f->color, host, cap);
        case FIBER_DUMP_DEPTH: return copy_out(f->depth, host, cap);
        case FIBER_DUMP_FRAGMENTS: return copy_out(f->fragments, host, cap);
        case FIBER_DUMP_OPAQUE_TILES: return copy_out(f->opaque_tiles, host, cap);
        case FREF_COMPOSITE: return copy_out(f->composite, host, cap);
        case FREF_TELEMETRY: return copy_out(f->telemetry, host, cap);
        case FREF_REF_KEYS: return copy_out(f->ref_keys, host, cap);
        case FREF_STAGE_MS: {
            uint64_t bytes = sizeof(f->stage_ms);
            if (host && cap >= bytes) std::memcpy(host, f->stage_ms, bytes);
            return bytes;
        }
        default: return 0;
    }
}

void fref_stats(const fref_frame* f, fiber_stats* s) {
    std::memset(s, 0, sizeof(*s));
    s->frustum_count = f->F;
    s->instance_count = f->I;
    s->binning_tasks = (uint32_t)f->tasks.size();
    s->camera_tasks = f->n_cam_tasks;
    s->allocated_pages = (uint32_t)f->page_meta.size();
    uint64_t refs = 0;
    for (const auto& pm : f->page_meta) refs += pm.seg_ref_count;
    s->fine_refs = (uint32_t)std::min<uint64_t>(refs, 0xFFFFFFFFull);
    s->fine_refs_total = refs;
    s->refs_requested = f->refs_tail;
    s->active_tiles = (uint32_t)f->active_tiles.size();
    s->camera_runs = f->camera_runs;
    s->shadow_runs = f->shadow_runs;
    s->work_items = (uint32_t)f->work.size();
    s->overflow_flags = f->overflow;
    for (uint32_t i = 0; i < f->F && i < FIBER_MAX_FRUSTA; ++i)
        s->frustum_tasks[i] = f->frustum_task_base[i + 1] - f->frustum_task_base[i];
    for (const auto& pm : f->page_meta) {
        uint32_t fr = frustum_for_tile(f, pm.coarse_tile_id);
        if (fr < FIBER_MAX_FRUSTA) { s->frustum_pages[fr]++; s->frustum_refs[fr] += pm.seg_ref_count; }
    }
    for (const auto& r : f->runs)
        if (r.frustum_id < FIBER_MAX_FRUSTA) { s->frustum_work[r.frustum_id] += r.work_count; s->frustum_runs[r.frustum_id]++; }
    s->total_segments = f->total_segments;
    s->total_points = f->total_points;
    s->total_strands = f->total_strands;
}

void fref_free(fref_frame* f) { delete f; }

void fref_composite(const fref_frame* f, const float* scene_color, const float* scene_depth, const float* dest,
                    int half_out, float* out) {
    if (!f || !scene_color || !out) return;
    composite_image(f, scene_color, scene_depth, dest, half_out != 0, out);
}

uint32_t fref_wang_hash(uint32_t x) { return wang_hash(x); }
float fref_hash_to_unit_float(uint32_t x) { return hash_to_unit_float(x); }
uint32_t fref_pack2x16unorm(float a, float b) { return pack2x16unorm(a, b); }
uint32_t fref_quantize_depth01(float z) { return quantize_depth01(z); }
float fref_normalize_depth01(float z) { return normalize_depth01(z); }
uint32_t fref_clip_segment(const float* p0, const float* p1, const float* bmin, const float* bmax, float* out) {
    Clipped c = clip_segment(v3(p0[0], p0[1], p0[2]), v3(p1[0], p1[1], p1[2]), v3(bmin[0], bmin[1], bmin[2]),
                             v3(bmax[0], bmax[1], bmax[2]));
    out[0] = c.p0.x; out[1] = c.p0.y; out[2] = c.p0.z;
    out[3] = c.p1.x; out[4] = c.p1.y; out[5] = c.p1.z;
    return c.ok ? 1u : 0u;
}
void fref_build_lut(const uint32_t* mins, const uint32_t* maxs, uint32_t n, fiber_coarse_depth_lut_entry* out) {
    LutBuilder b;
    for (uint32_t i = 0; i < n; ++i) b.add(mins[i], maxs[i]);
    b.emit(out);
}

}  // extern "C"
