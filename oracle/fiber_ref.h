/*
 * fiber_ref.h — ORACLE (test infrastructure only).
 *
 * CPU restatement of the reference's WGSL strand-raster path, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker and
 * the timed CPU baseline. Nothing in the product links or calls this code.
 *
 * Parity status: UNPINNED. The reference (Rust + WGSL over wgpu/Vulkan)
 * cannot be built or run here and its tests hold no golden vectors for this
 * path; the only reference test (src/strand_cache.rs:238-281) pins the
 * `.strands` parser, which tests/test_strand_cache.py mirrors. Every stage
 * below follows the cited WGSL line by line with the WGSL-spec semantics of
 * its builtins; where the reference is nondeterministic (atomic append
 * orders) the oracle fixes a canonical order that the CUDA path reproduces.
 */
#ifndef FIBER_REF_H
#define FIBER_REF_H

#include <stdint.h>
#include "../include/fiber.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One registered instance: host copies of its slabs (one slab per kind). */
typedef struct fref_instance {
    const float* vertices4;              /* float4 per vertex (w = 1)     */
    uint32_t n_vertices;
    const uint32_t* indices;
    uint32_t n_indices;
    const fiber_strand_meta* meta;
    uint32_t n_meta;
    fiber_strand_geo geo;
    const fiber_strand_material* materials;
    uint32_t n_materials;
    float world_from_local[16];
} fref_instance;

typedef struct fref_capacities {
    uint32_t task_capacity;   /* binning queue entries        */
    uint32_t page_capacity;   /* allocatable count pages      */
    uint32_t ref_capacity;    /* fine segment references      */
    uint32_t work_capacity;   /* raster work items            */
} fref_capacities;

typedef struct fref_frame fref_frame;

/* Runs one frame. history_prev: half2 per atlas texel (may be NULL = cleared).
 * threads <= 0 uses every OpenMP thread. */
fref_frame* fref_run(const fref_instance* inst, uint32_t n_inst,
                     const fiber_froxel_config* camera_cfg, const fiber_camera* camera,
                     const fiber_froxel_config* light_cfgs, const fiber_light* lights,
                     uint32_t n_lights, const fiber_settings* settings,
                     const fref_capacities* caps, const uint16_t* history_prev,
                     const float* scene_color_rgba, const float* scene_depth,
                     int threads);

/* fref_run with the camera's opaque depth for the opaque-tile reduce and cull:
 * reversed-Z, `opaque_samples` (1 or 4) floats per pixel, rows of
 * width * samples floats; NULL culls nothing. */
fref_frame* fref_run_opaque(const fref_instance* inst, uint32_t n_inst,
                            const fiber_froxel_config* camera_cfg, const fiber_camera* camera,
                            const fiber_froxel_config* light_cfgs, const fiber_light* lights,
                            uint32_t n_lights, const fiber_settings* settings,
                            const fref_capacities* caps, const uint16_t* history_prev,
                            const float* scene_color_rgba, const float* scene_depth,
                            const float* opaque_depth, uint32_t opaque_samples, int threads);

/* Copies one output (fiber_dump_what numbering, plus FREF_* extras) into
 * host; returns the byte size (host may be NULL to query). */
uint64_t fref_get(const fref_frame* f, uint32_t what, void* host, uint64_t capacity);
void fref_stats(const fref_frame* f, fiber_stats* out);
void fref_free(fref_frame* f);

/* The composite of a finished frame's strand image over one scene image
 * (strand_composite.wgsl:12-33 with ALPHA_BLENDING onto the loaded
 * destination). scene_color and dest are float RGBA [H][W][4], scene_depth
 * float [H][W] (NULL: no opaque scene). dest holds the destination's contents
 * before the pass; NULL composites in place (dest = scene_color). half_out
 * rounds each output channel to binary16. out: float [H][W][4]. */
void fref_composite(const fref_frame* f, const float* scene_color, const float* scene_depth, const float* dest,
                    int half_out, float* out);

/* Extra oracle outputs beyond the fiber_dump_what set. */
#define FREF_COMPOSITE 100   /* float[W*H*4] composited output (fp16-rounded) */
#define FREF_REF_KEYS 101    /* u32[R] sort key of each reference             */
#define FREF_STAGE_MS 102    /* float[8] per-stage wall time                  */
#define FREF_TELEMETRY 103   /* fiber_telemetry image (u32 words)              */

/* Primitive known-answer helpers (tests/test_oracle_primitives.py). */
uint32_t fref_wang_hash(uint32_t x);
float fref_hash_to_unit_float(uint32_t x);
uint32_t fref_pack2x16unorm(float a, float b);
uint32_t fref_quantize_depth01(float z);
float fref_normalize_depth01(float z);
/* Clips segment p0->p1 (xyz) to a box; returns ok and writes the clipped
 * endpoints to out[6]. */
uint32_t fref_clip_segment(const float* p0, const float* p1, const float* bmin,
                           const float* bmax, float* out);
/* Builds a 16-entry depth-warp LUT from n intervals (z_min_q, z_max_q). */
void fref_build_lut(const uint32_t* mins, const uint32_t* maxs, uint32_t n,
                    fiber_coarse_depth_lut_entry* out16);

#ifdef __cplusplus
}
#endif
#endif
