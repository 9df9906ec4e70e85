/*
 * fiber.h — C ABI of the B200-native strand software-raster path.
 *
 * This library replaces the per-frame GPU work of the Fiber Bevy plugin
 * (RostigerDagmer/bevy_strand_rasterizer): work preparation (broad + fine
 * prepass, froxel binning), deep-opacity shadow maps with shadow-map
 * stampback, per-segment hair shading, tile-binned strand rasterisation and
 * compositing.  Every struct below is byte-for-byte the layout of the
 * reference's `#[repr(C)]` host mirrors (src/shader_types.rs,
 * src/pipelines/task_contract.rs, src/components.rs, src/plugin.rs) so a Rust
 * host can hand its own buffers across the FFI without repacking.
 *
 * Conventions
 *  - All entry points return fiber_status; nothing aborts or traps.
 *  - `stream` arguments are cudaStream_t passed as void* (NULL = legacy stream).
 *  - A context is single-threaded (callers synchronise externally); several
 *    contexts may share one device.
 *  - Matrices are column-major float[16] (glam Mat4 layout); a matrix-vector
 *    product is c0*x + c1*y + c2*z + c3*w evaluated left to right.
 */
#ifndef FIBER_H
#define FIBER_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Frusta of one frame: the camera plus up to 15 directional lights. */
#define FIBER_MAX_FRUSTA 16

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum fiber_status {
    FIBER_OK = 0,
    FIBER_EINVAL = 1,     /* bad argument, malformed slab or instance         */
    FIBER_ENOMEM = 2,     /* device allocation failed or HBM budget exceeded  */
    FIBER_EOVERFLOW = 3,  /* a device queue overflowed; work was dropped      */
    FIBER_ETIMEDOUT = 4,  /* a bounded device wait gave up                    */
    FIBER_ECUDA = 5,      /* a CUDA runtime call failed                       */
    FIBER_ENOTREADY = 6   /* a node ran before its inputs existed             */
} fiber_status;

/* ------------------------------------------------------------------------ */
/* Slab format (bevy_gpu_paging_allocator replacement)                       */
/* ------------------------------------------------------------------------ */
/* Slab kinds and their bind ids: src/plugin.rs:129-140 (Vert 0, Index 1,
 * StrandMaterial 5, StrandGeo 6, StrandMeta 7). */
typedef enum fiber_slab_kind {
    FIBER_SLAB_VERT = 0,
    FIBER_SLAB_INDEX = 1,
    FIBER_SLAB_MATERIAL = 5,
    FIBER_SLAB_GEO = 6,
    FIBER_SLAB_META = 7
} fiber_slab_kind;

/* DevicePtr: src/shaders/types.wgsl:23-27 ({slab, byte offset, byte size}). */
typedef struct fiber_devptr {
    uint32_t slab;
    uint32_t offset;
    uint32_t size;
} fiber_devptr;

/* StrandMeta: src/shader_types.rs:24-31 (16 B). */
typedef struct fiber_strand_meta {
    uint32_t count;        /* vertices in the strand                    */
    uint32_t offset;       /* first position in the index slab          */
    uint32_t material_idx; /* index into the instance's material slab   */
    uint32_t pad;
} fiber_strand_meta;

/* Aabb: src/shader_types.rs:44-51 (32 B). */
typedef struct fiber_aabb {
    float min[3];
    float pad_a;
    float max[3];
    float pad_b;
} fiber_aabb;

/* StrandGeo: src/shader_types.rs:64-73 (64 B). */
typedef struct fiber_strand_geo {
    uint32_t strand_count;
    uint32_t max_segments_in_strand;
    uint32_t offset;
    uint32_t pad_b;
    fiber_aabb aabb;
    uint32_t pad_c[4];
} fiber_strand_geo;

/* StrandMaterial: src/components.rs:61-72 (64 B); defaults :74-89. */
typedef struct fiber_strand_material {
    float absorption_color[4];
    float specular_color[4];
    float ambient_factor;
    float ao_factor;
    float eta;
    float beta;
    float alpha;
    float shift;
    float min_radius_pixels;
    float max_radius_pixels;
} fiber_strand_material;

/* StrandInstance: src/shader_types.rs:75-88 (160 B). The *_id fields are
 * allocation ids returned by fiber_slab_alloc for the matching slab kind. */
typedef struct fiber_strand_instance {
    uint32_t vertex_id;
    uint32_t index_id;
    uint32_t meta_id;
    uint32_t geo_id;
    uint32_t material_id;
    uint32_t pad0;
    uint32_t pad1;
    uint32_t pad2;
    float world_from_local[16];
    float local_from_world[16];
} fiber_strand_instance;

/* ------------------------------------------------------------------------ */
/* Views, lights and the frustum table                                       */
/* ------------------------------------------------------------------------ */
/* FroxelConfig: src/components.rs:93-110 (20 B). */
typedef struct fiber_froxel_config {
    uint32_t screen_width;
    uint32_t screen_height;
    uint32_t froxel_size_x;
    uint32_t froxel_size_y;
    uint32_t depth_slices;
} fiber_froxel_config;

/* GpuFrustumDesc: src/plugin.rs:1545-1562 (64 B). kind 0 = camera, 1 = light. */
typedef struct fiber_frustum_desc {
    uint32_t screen_width;
    uint32_t screen_height;
    uint32_t froxel_size_x;
    uint32_t froxel_size_y;
    uint32_t depth_slices;
    uint32_t bucket_base;
    uint32_t bucket_count;
    uint32_t kind;
    uint32_t coarse_depth_tile_base;
    uint32_t coarse_depth_tile_count;
    uint32_t coarse_tiles_x;
    uint32_t coarse_tiles_y;
    uint32_t cascade_index;
    uint32_t fine_depth_tile_base;
    uint32_t pad1;
    uint32_t pad2;
} fiber_frustum_desc;

/* The camera fields the path reads from Bevy's View uniform
 * (view.unjittered_clip_from_world, view.world_position:
 * src/shaders/strand_prepass.wgsl:446, src/shaders/strand_shading.wgsl:653). */
typedef struct fiber_camera {
    float clip_from_world[16];
    float world_position[3];
    float pad;
} fiber_camera;

/* The directional-light fields the path reads from Bevy's Lights uniform:
 * cascades[c].clip_from_world (one authoritative cascade per light),
 * direction_to_light and color (linear colour x illuminance)
 * (src/shaders/strand_prepass.wgsl:443, src/shaders/strand_shading.wgsl:684-688). */
typedef struct fiber_light {
    float clip_from_world[16];
    float direction_to_light[3];
    float pad0;
    float color[4];
} fiber_light;

/* ------------------------------------------------------------------------ */
/* Queue / task ABI (src/pipelines/task_contract.rs:45-135)                  */
/* ------------------------------------------------------------------------ */
typedef struct fiber_queue_header { uint32_t head, tail; } fiber_queue_header;
typedef struct fiber_fine_prepass_task { uint32_t inst_id, strand_local; } fiber_fine_prepass_task;
/* packed_field bits: [0..1] level, [2] is_shadow, [3..31] frustum. */
typedef struct fiber_binning_task { uint32_t id_info, chunk_id, seg_idx, packed_field; } fiber_binning_task;
typedef struct fiber_projected_segment { uint32_t p0_xy, p1_xy, depths; } fiber_projected_segment;
typedef struct fiber_raster_work_item {
    uint32_t seg_ref_base, seg_ref_count, frustum_id, screen_tile_id;
    uint32_t depth_key, load_score, page_idx, cell_idx;
} fiber_raster_work_item;
typedef struct fiber_raster_tile_run {
    uint32_t work_base, work_count, frustum_id, screen_tile_id;
    uint32_t load_score, flags, raster_run_reserved_a, raster_run_reserved_b;
} fiber_raster_tile_run;
typedef struct fiber_fine_seg_ref { uint32_t inst_id, seg_id, material_idx; } fiber_fine_seg_ref;
typedef struct fiber_fine_page_meta {
    uint32_t seg_ref_base, seg_ref_count, work_base, work_count;
    uint32_t coarse_tile_id, coarse_z, first_depth_key, flags;
} fiber_fine_page_meta;
/* GpuCoarseDepthLutEntry: src/plugin.rs:1566-1571. */
typedef struct fiber_coarse_depth_lut_entry {
    uint32_t z_min_q, z_max_q, virtual_start_q, virtual_count_q;
} fiber_coarse_depth_lut_entry;
/* GpuCoarseAssetRange: src/plugin.rs:1575-1584. */
typedef struct fiber_coarse_asset_range {
    uint32_t geo_id, frustum_id, min_x, max_x, min_y, max_y, z_min_q, z_max_q;
} fiber_coarse_asset_range;

/* ------------------------------------------------------------------------ */
/* Settings (StochasticCullSettings, PrepassTelemetrySettings,               */
/* FineBinningBackend: src/resources.rs:70-104; PushConstants                */
/* src/shader_types.rs:7-22)                                                 */
/* ------------------------------------------------------------------------ */
typedef struct fiber_settings {
    uint32_t stochastic_cull_enabled;   /* default 1                        */
    float target_strands_per_pixel;     /* default 2.0                      */
    float min_keep_probability;         /* default 0.02                     */
    float shadow_keep_probability;      /* default 1.0                      */
    uint32_t telemetry_enabled;         /* default 0                        */
    uint32_t fine_binning_backend;      /* 0 = SegmentScatter, 1 = PageCsr  */
    uint32_t dom_slices;                /* deep-opacity layers K (ref 12)   */
    uint32_t shadow_map_size;           /* stampback target side; 0 = DOM   */
    float ambient_color[4];             /* Lights.ambient_color (linear)    */
    uint32_t history_enabled;           /* temporal shadow history (1)      */
    uint32_t fragment_counts_enabled;   /* per-pixel fragment counter (0)   */
    uint32_t ref_capacity_factor;       /* refs = factor x tasks (4)        */
    uint32_t page_capacity_divisor;     /* pages = table / divisor (1)      */
    uint32_t dom_page_pool;             /* 0 = dense deep-opacity layers (default);
                                           N = sparse residency: the pages of
                                           256^2 texels that shadow tile runs
                                           request (with a one-page border)
                                           live in a pool of N pages          */
} fiber_settings;

/* ------------------------------------------------------------------------ */
/* Images (headless replacements for the swapchain / view targets)          */
/* ------------------------------------------------------------------------ */
typedef enum fiber_format {
    FIBER_FMT_RGBA16F = 0,  /* 8 B / px  */
    FIBER_FMT_R32F = 1,     /* 4 B / px  */
    FIBER_FMT_RGBA32F = 2   /* 16 B / px */
} fiber_format;

typedef struct fiber_image {
    void* ptr;          /* device pointer                */
    uint32_t width;
    uint32_t height;
    uint32_t pitch;     /* bytes per row                 */
    uint32_t format;    /* fiber_format                  */
} fiber_image;

/* ------------------------------------------------------------------------ */
/* Per-frame statistics (telemetry counters + overflow words)               */
/* ------------------------------------------------------------------------ */
typedef struct fiber_stats {
    uint32_t frustum_count;
    uint32_t instance_count;
    uint32_t binning_tasks;         /* N = sum_f N_f                          */
    uint32_t camera_tasks;          /* shading queue length                   */
    uint32_t allocated_pages;
    uint32_t fine_refs;             /* references kept (saturates at 2^32-1;
                                       fine_refs_total holds the full count)  */
    uint32_t active_tiles;
    uint32_t camera_runs;
    uint32_t shadow_runs;
    uint32_t work_items;
    uint32_t overflow_flags;        /* bit0 tasks, bit1 pages, bit2 refs, bit3 work,
                                       bit4 DOM page pool                     */
    uint32_t timeout_flags;         /* non-zero: a bounded device wait gave up */
    uint32_t frustum_tasks[FIBER_MAX_FRUSTA];  /* N_f per frustum (camera, then lights) */
    uint32_t frustum_pages[FIBER_MAX_FRUSTA];
    uint32_t frustum_refs[FIBER_MAX_FRUSTA];
    uint32_t frustum_work[FIBER_MAX_FRUSTA];
    uint32_t frustum_runs[FIBER_MAX_FRUSTA];
    uint64_t total_segments;        /* segments of all registered instances   */
    uint64_t total_points;
    uint64_t total_strands;
    uint64_t fine_refs_total;       /* references kept, 64-bit                */
    uint64_t refs_requested;        /* references the frame's cells asked for;
                                       above the kept count when refs overflowed */
} fiber_stats;

/* PrepassTelemetrySettings counters (src/resources.rs:77-84, collected by
 * strand_prepass.wgsl:271-292,2145-2188, read back by
 * src/pipelines/prepass.rs:1345-1396). Gathered only when
 * fiber_settings.telemetry_enabled is set: they add atomics to the prepass. */
#define FIBER_TELEMETRY_HISTOGRAM_BINS 32
#define FIBER_TELEMETRY_MAX_FRUSTA 16
typedef struct fiber_frustum_telemetry {
    uint32_t visible_instances;    /* instances whose AABB reaches the frustum       */
    uint32_t visible_strands;      /* their strand counts                            */
    uint32_t retained_strands;     /* strands kept by the stochastic cull            */
    uint32_t emitted_segments;     /* binning tasks                                  */
    uint32_t allocated_pages;
    uint32_t page_candidates;      /* (task, page) pairs over its allocated pages    */
    uint32_t fine_refs;
    uint32_t raster_runs;          /* tile runs with work                            */
    uint32_t raster_load;          /* sum of the runs' load scores (references)      */
    uint32_t max_page_candidates;
    uint32_t max_raster_load;
} fiber_frustum_telemetry;
typedef struct fiber_telemetry {
    uint32_t allocated_pages;
    uint32_t binning_tasks;
    uint32_t page_candidates;          /* tasks per allocated page, summed           */
    uint32_t fine_cell_hits;           /* fine references (the reference tail)       */
    uint32_t active_candidate_pages;   /* allocated pages with a candidate           */
    uint32_t max_candidates_per_page;
    uint32_t frustum_count;
    uint32_t pad;
    uint32_t candidate_histogram[FIBER_TELEMETRY_HISTOGRAM_BINS];  /* pages by floor(log2(candidates)) */
    fiber_frustum_telemetry frustum[FIBER_TELEMETRY_MAX_FRUSTA];
} fiber_telemetry;

/* What fiber_dump copies back (canonical forms used by parity tests). */
typedef enum fiber_dump_what {
    FIBER_DUMP_FRUSTA = 0,        /* fiber_frustum_desc[F]                      */
    FIBER_DUMP_RANGES = 1,        /* (valid u32 + fiber_coarse_asset_range)[I*F] */
    FIBER_DUMP_KEEP = 2,          /* float[I*F] per-frustum keep probability    */
    FIBER_DUMP_LUT = 3,           /* fiber_coarse_depth_lut_entry[T*16]         */
    FIBER_DUMP_TASKS = 4,         /* fiber_binning_task[N]                      */
    FIBER_DUMP_PROJECTED = 5,     /* fiber_projected_segment[N]                 */
    FIBER_DUMP_PAGE_TABLE = 6,    /* u32[T*16] (0 empty, idx+1 allocated)       */
    FIBER_DUMP_PAGE_META = 7,     /* fiber_fine_page_meta[pages]                */
    FIBER_DUMP_COUNTS = 8,        /* u32[pages*256] froxel counts               */
    FIBER_DUMP_OFFSETS = 9,       /* u32[pages*256] exclusive prefix offsets    */
    FIBER_DUMP_REFS = 10,         /* fiber_fine_seg_ref[R] (canonical order)    */
    FIBER_DUMP_ACTIVE_TILES = 11, /* u32[A] packed coarse_tile*16+local         */
    FIBER_DUMP_WORK = 12,         /* fiber_raster_work_item[W]                  */
    FIBER_DUMP_RUNS = 13,         /* fiber_raster_tile_run[runs] camera then shadow */
    FIBER_DUMP_DOM_DEPTH = 14,    /* float[L*D*D]                               */
    FIBER_DUMP_DOM_OPACITY = 15,  /* float[L*K*D*D]                             */
    FIBER_DUMP_SHADOW_MAP = 16,   /* float[L*S*S] stampback target              */
    FIBER_DUMP_ATLAS = 17,        /* half[I*cap*4] shading atlas                */
    FIBER_DUMP_HISTORY = 18,      /* half[I*cap*2] shadow history (next)        */
    FIBER_DUMP_COLOR = 19,        /* half[W*H*4] strand colour (RGBA16F)        */
    FIBER_DUMP_DEPTH = 20,        /* float[W*H] strand depth                    */
    FIBER_DUMP_FRAGMENTS = 21,    /* u32[W*H] per-pixel fragment counts         */
    FIBER_DUMP_OPAQUE_TILES = 22  /* (covered u32, farthest depth q u32)[camera fine
                                     tiles]; all zero when no opaque depth was given */
} fiber_dump_what;

typedef struct fiber_ctx fiber_ctx;

/* ------------------------------------------------------------------------ */
/* Plugin API (StrandRasterizerPlugin::build/finish, src/plugin.rs:162-262)  */
/* ------------------------------------------------------------------------ */
/* Create a context on `device`. hbm_budget bytes caps the context's device
 * allocations (0 = no cap). */
fiber_status fiber_ctx_create(int device, uint64_t hbm_budget, fiber_ctx** out);
fiber_status fiber_ctx_destroy(fiber_ctx* ctx);
/* Mirrors StochasticCullSettings / PrepassTelemetrySettings /
 * FineBinningBackend (src/resources.rs:70-104). */
fiber_status fiber_settings_default(fiber_settings* out);
fiber_status fiber_settings_set(fiber_ctx* ctx, const fiber_settings* settings);

/* ------------------------------------------------------------------------ */
/* Slabs (VirtualShaderStorageBuffer per SlabKind, src/plugin.rs:1395-1440)  */
/* ------------------------------------------------------------------------ */
/* Allocates `bytes` of slab `kind`; returns the allocation id (the id a
 * StrandInstance stores) and its DevicePtr. */
fiber_status fiber_slab_alloc(fiber_ctx* ctx, uint32_t kind, uint64_t bytes,
                              uint32_t* alloc_id, fiber_devptr* out);
fiber_status fiber_slab_upload(fiber_ctx* ctx, uint32_t kind, uint32_t alloc_id,
                               uint64_t dst_offset, const void* host, uint64_t bytes,
                               void* stream);
fiber_status fiber_slab_free(fiber_ctx* ctx, uint32_t kind, uint32_t alloc_id);

/* Registers the StrandInstance table (src/plugin.rs:284-315). Validates every
 * referenced slab on the device (indices < vertices, strand ranges inside the
 * index slab, material indices) and rejects malformed instances with EINVAL,
 * mirroring validate_cache (src/strand_cache.rs:174-209). */
fiber_status fiber_instance_set(fiber_ctx* ctx, const fiber_strand_instance* rows, uint32_t n);

/* ------------------------------------------------------------------------ */
/* Per-frame host preparation (use_prepass_buffers, src/plugin.rs:264-1209)  */
/* ------------------------------------------------------------------------ */
/* Builds the frustum table (camera first, then one frustum per light, in the
 * order given), sizes every queue, and uploads the frame tables on `stream`. */
fiber_status fiber_frame_begin(fiber_ctx* ctx,
                               const fiber_froxel_config* camera_cfg,
                               const fiber_camera* camera,
                               const fiber_froxel_config* light_cfgs,
                               const fiber_light* lights, uint32_t n_lights,
                               void* stream);

/* ------------------------------------------------------------------------ */
/* Render-graph node contracts (src/nodes/<node>.rs)                         */
/* ------------------------------------------------------------------------ */
/* reduce_opaque_depth (src/shaders/opaque_depth_reduce.wgsl:36-86, run by
 * src/nodes/prepass.rs:111-145 before the prepass dispatches): reduces the
 * camera's opaque depth to one (fully covered, farthest depth) pair per camera
 * fine tile. `depth` is R32F, reversed-Z (0 = nothing drawn), the camera's
 * width x height, with `samples` (1 or 4) consecutive floats per pixel, so a
 * row holds width * samples floats. Call after fiber_frame_begin and before
 * fiber_prepass; the prepass then drops the fine cells of a covered tile whose
 * depth slice lies wholly behind the farthest opaque depth
 * (fine_tile_occluded_by_opaque, src/shaders/strand_prepass.wgsl:551-573).
 * A frame without this call culls nothing. fiber_frame_fused and
 * fiber_render_host run it themselves on scene_depth (1 sample). */
fiber_status fiber_opaque_depth(fiber_ctx* ctx, const fiber_image* depth, uint32_t samples, void* stream);
/* work_preparation_pass (src/nodes/prepass.rs:27-233). */
fiber_status fiber_prepass(fiber_ctx* ctx, void* stream);
/* strand_shadow_rasterizer_pass incl. stampback (src/nodes/shadows.rs:29-221). */
fiber_status fiber_shadows(fiber_ctx* ctx, void* stream);
/* strand_shading_pass (src/nodes/shading.rs:25-155); flips the history. */
fiber_status fiber_shading(fiber_ctx* ctx, void* stream);
/* strand_rasterizer_pass (src/nodes/raster.rs:26-179). */
fiber_status fiber_raster(fiber_ctx* ctx, uint32_t view, void* stream);
/* composition_pass (src/nodes/composite.rs:19-131): per-pixel depth test and
 * alpha mix of the strand image into scene_color, ALPHA_BLENDING onto `out`
 * (loaded). scene_depth may be NULL (no opaque scene: depth 0). */
fiber_status fiber_composite(fiber_ctx* ctx, uint32_t view, const fiber_image* scene_color,
                             const fiber_image* scene_depth, fiber_image* out, void* stream);
/* One view of a multi-view frame: a camera, its lights and the instances it
 * sees. No counterpart in the reference, which records each view's nodes in
 * turn; it is the batched configuration of the path's specification. */
typedef struct fiber_view {
    fiber_froxel_config camera_cfg;
    fiber_camera camera;
    const fiber_froxel_config* light_cfgs;  /* n_lights square maps of one size  */
    const fiber_light* lights;
    uint32_t n_lights;
    uint32_t instance_first;   /* the view's instances: [first, first + count) of
                                  the instance table; views follow one another */
    uint32_t instance_count;
    uint32_t pad;
} fiber_view;

/* fiber_frame_begin for several independent views rendered by one frame: every
 * kernel of the frame covers all views, with each view's tasks, pages and
 * runs at offsets from the frame's single prefix sums, and each view seeing
 * only its own instances and lights. Frusta: the cameras (frustum v is view
 * v's camera), then each view's lights. The colour, depth and fragment images
 * of the views follow one another (view v's starts at the sum of the earlier
 * views' pixels); deep-opacity layer l is the l-th light, layers as large as
 * the largest map. At most 64 views and 128 frusta; dense deep-opacity layers
 * only, telemetry only up to 16 frusta, and no composite or opaque depth (those
 * are one camera's). Each view's images equal what the view renders alone. */
fiber_status fiber_frame_begin_views(fiber_ctx* ctx, const fiber_view* views, uint32_t n_views, void* stream);

/* All nodes of one frame in order, replayed from a CUDA graph after the first
 * call with the same frame shape. A scene_depth also feeds the opaque-tile
 * reduce (fiber_opaque_depth at 1 sample) ahead of the prepass. */
fiber_status fiber_frame_fused(fiber_ctx* ctx, const fiber_image* scene_color,
                               const fiber_image* scene_depth, fiber_image* out, void* stream);

/* One whole frame from host memory to host memory: copies the scene colour
 * (RGBA16F, width x height of the camera) and optional scene depth (R32F)
 * from host buffers (pinned for asynchronous copies), runs every node as
 * fiber_frame_fused does, and copies the composited RGBA16F image back into
 * out_rgba16f_host. Call after fiber_frame_begin; returns when the copies are
 * queued on `stream` (synchronise the stream before reading the output).
 * This is the whole render-graph slice of src/plugin.rs:240-260 seen from a
 * host that owns its images, e.g. a Rust caller over the FFI. */
fiber_status fiber_render_host(fiber_ctx* ctx, const void* scene_rgba16f_host,
                               const float* scene_depth_host, void* out_rgba16f_host,
                               void* stream);

/* ------------------------------------------------------------------------ */
/* Readback                                                                  */
/* ------------------------------------------------------------------------ */
/* Synchronises the context's last stream and returns the frame counters
 * (telemetry words, src/pipelines/prepass.rs:1345-1396). */
fiber_status fiber_stats_get(fiber_ctx* ctx, fiber_stats* out);

/* ------------------------------------------------------------------------ */
/* Test hook (no counterpart in the reference)                               */
/* ------------------------------------------------------------------------ */
/* Makes the next frame's bounded device waits run out, to exercise the
 * FIBER_ETIMEDOUT path without faulting or hanging anything. In the frame of
 * the next fiber_frame_begin, look-back stage `stage` (0 fine prepass, 1 page
 * allocation, 2 page prefix, 3 active-tile compaction, 4 raster work emit)
 * has a tile `tile` that never publishes its prefix, and every look-back wait
 * of that frame gives up after `spin_limit` polls (0: the default 2^21). The
 * waits behind that tile give up and set the frame's error word; the kernels
 * after the stage then do nothing, and fiber_stats_get returns
 * FIBER_ETIMEDOUT with timeout_flags set. The frame after it is normal. */
fiber_status fiber_debug_stall_lookback(fiber_ctx* ctx, uint32_t stage, uint32_t tile, uint32_t spin_limit);

/* The last frame's prepass telemetry; EINVAL unless telemetry is enabled. */
fiber_status fiber_telemetry_get(fiber_ctx* ctx, fiber_telemetry* out);
/* Copies one canonical buffer to host memory. With host == NULL only
 * *written receives the byte size. */
fiber_status fiber_dump(fiber_ctx* ctx, uint32_t what, void* host, uint64_t capacity,
                        uint64_t* written);
/* Device pointers of the context-owned outputs (strand colour RGBA16F, strand
 * depth R32F, DOM layers, stampback target) for zero-copy consumers. */
fiber_status fiber_output_image(fiber_ctx* ctx, uint32_t what, fiber_image* out);
/* Per-stage device times of the last frame in ms, named like the reference's
 * diagnostic spans; returns the number of spans written. */
uint32_t fiber_span_count(void);
const char* fiber_span_name(uint32_t i);
fiber_status fiber_span_times(fiber_ctx* ctx, float* ms, uint32_t n);
const char* fiber_status_string(fiber_status s);

/* ------------------------------------------------------------------------ */
/* Request server: continuous batching of render requests over resident      */
/* scenes. No counterpart in the reference (a Bevy app renders one frame per */
/* view per tick); it is the served mode of the path's specification.        */
/* ------------------------------------------------------------------------ */
typedef struct fiber_server fiber_server;

typedef struct fiber_server_config {
    uint32_t slots;        /* frames in flight at once (each slot is a context with
                              its own streams and worker thread); 0 = as many as
                              the HBM budget admits, at most 64 (8 without a
                              budget); a budget also caps a non-zero count     */
    uint32_t max_width;    /* largest request resolution; every slot is sized   */
    uint32_t max_height;   /* for it at fiber_server_start                      */
    uint32_t max_lights;   /* most lights of one request (<= 4)                 */
    uint32_t max_dom;      /* largest deep-shadow map side of one request       */
    uint32_t priority_levels; /* stream priorities the frames in flight take by
                              admission order (oldest highest): 0 = every level
                              the device offers, 1 = one priority for all   */
    uint64_t hbm_budget;   /* device bytes all slots may hold (0 = no cap)      */
    uint32_t priority_order; /* FIBER_PRIORITY_ARRIVAL: the oldest frame in flight
                              highest; FIBER_PRIORITY_COST: the costliest request
                              (segments x frusta + pixels + shadow texels)
                              highest, one level lower per halving of cost   */
    uint32_t pad;
} fiber_server_config;
#define FIBER_PRIORITY_ARRIVAL 0u
#define FIBER_PRIORITY_COST 1u

/* One resident scene: a strand instance in the reference's slab format
 * (pack_strands / pack_indexed_strands, src/plugin.rs:1315-1393), host memory. */
typedef struct fiber_server_scene {
    const float* vertices;           /* float4 per point (w = 1)          */
    uint32_t n_vertices;
    const uint32_t* indices;         /* u32 per point                     */
    uint32_t n_indices;
    const fiber_strand_meta* meta;   /* per strand                        */
    uint32_t n_meta;
    fiber_strand_geo geo;
    const fiber_strand_material* materials;
    uint32_t n_materials;
    float world_from_local[16];      /* column-major                      */
} fiber_server_scene;

#define FIBER_SERVER_MAX_LIGHTS 4
typedef struct fiber_server_request {
    uint32_t scene;                  /* id from fiber_server_add_scene    */
    uint32_t n_lights;
    fiber_froxel_config camera_cfg;
    fiber_camera camera;
    fiber_froxel_config light_cfgs[FIBER_SERVER_MAX_LIGHTS];
    fiber_light lights[FIBER_SERVER_MAX_LIGHTS];
    const void* scene_rgba16f;       /* host W x H RGBA16F under the strands, or NULL (transparent) */
    void* out_rgba16f;               /* host W x H RGBA16F result, written before the ticket completes */
    uint64_t arrival_ns;             /* arrival on fiber_server_now_ns's clock; 0 = at submit */
} fiber_server_request;

typedef struct fiber_server_result {
    fiber_status status;
    uint32_t slot;                   /* slot that rendered it             */
    uint64_t arrival_ns, admit_ns, done_ns;  /* fiber_server_now_ns clock  */
    uint32_t renders;                /* frames rendered: 1, or 2-3 when the
                                        slot's reference capacity had to grow
                                        (the image is never truncated)     */
    uint32_t priority;               /* stream priority level of its frame:
                                        0 = highest (admitted with no frame
                                        in flight)                         */
} fiber_server_result;

/* Creates a server on `device`; `settings` apply to every slot except that the
 * temporal shadow history is off, so a request's image does not depend on
 * which requests ran before it on the same slot. */
fiber_status fiber_server_create(int device, const fiber_settings* settings, const fiber_server_config* cfg,
                                 fiber_server** out);
/* Uploads a scene once (before fiber_server_start); every slot renders from
 * the same device-resident slabs. */
fiber_status fiber_server_add_scene(fiber_server* srv, const fiber_server_scene* scene, uint32_t* scene_id);
/* Sizes every slot for the largest scene at the configured maximum frame,
 * settles the slot count under the HBM budget and starts the workers. */
fiber_status fiber_server_start(fiber_server* srv, uint32_t* slots_started);
/* Queues a request; a free slot admits it at once, otherwise the first slot to
 * finish does (arrival order). Requests beyond the configured maximum shape
 * return FIBER_EINVAL. The request and its host buffers must stay valid until
 * its ticket completes. */
fiber_status fiber_server_submit(fiber_server* srv, const fiber_server_request* req, uint64_t* ticket);
/* Blocks until `ticket` completes. */
fiber_status fiber_server_wait(fiber_server* srv, uint64_t ticket, fiber_server_result* out);
/* Finishes queued requests, stops the workers and frees every slot. */
fiber_status fiber_server_destroy(fiber_server* srv);
/* The server's steady clock in nanoseconds. */
uint64_t fiber_server_now_ns(void);

/* ------------------------------------------------------------------------ */
/* Batched mode: many independent views rendered by one CUDA graph launch.   */
/* No counterpart in the reference (a Bevy app records each view's nodes in  */
/* turn); it is the batched configuration of the path's specification.       */
/* ------------------------------------------------------------------------ */
/* Each view is a context the caller creates and fills with the ordinary
 * calls (fiber_settings_set, slabs, fiber_instance_set, fiber_frame_begin).
 * fiber_batch_launch replays one frame of every view (prepass, shadows,
 * shading, raster; no composite) from a single graph captured on first use,
 * with the views spread over `branches` concurrent graph branches. Each
 * replayed frame advances its look-back epoch and shadow history on the
 * device, so replays repeat without host work per view. The graph is
 * recaptured when a view's frame shape changes (fiber_frame_begin with new
 * sizes, reallocated buffers) or the tuning changes. A context used in a
 * batch may still render alone; its next fiber_frame_begin restarts its
 * epoch. Outputs are read per view with fiber_dump / fiber_output_image. */
typedef struct fiber_batch fiber_batch;

typedef enum fiber_batch_order {
    FIBER_BATCH_ORDER_INDEX = 0,  /* view v on branch v mod branches, in index order   */
    FIBER_BATCH_ORDER_LPT = 1     /* longest predicted frame first, to the least loaded
                                     branch (frame cost: segments x frusta + pixels +
                                     DOM texels)                                        */
} fiber_batch_order;

typedef struct fiber_batch_tuning {
    uint32_t branches;  /* concurrent graph branches, 1..32                        */
    uint32_t order;     /* fiber_batch_order                                        */
    float ms;           /* fiber_batch_tune: measured batch time of this choice     */
    uint32_t pad;
} fiber_batch_tuning;

/* views: n contexts on one device, borrowed (they must outlive the batch).
 * The initial tuning is one branch in index order. */
fiber_status fiber_batch_create(fiber_ctx* const* views, uint32_t n, fiber_batch** out);
fiber_status fiber_batch_set_tuning(fiber_batch* batch, const fiber_batch_tuning* tuning);
fiber_status fiber_batch_get_tuning(const fiber_batch* batch, fiber_batch_tuning* tuning);
/* One frame of every view; `stream` must not be the legacy stream. */
fiber_status fiber_batch_launch(fiber_batch* batch, void* stream);
/* The autotuner: times every branch count (powers of two up to the view
 * count, at most 32) in both view orders over a few replays on `stream` with
 * CUDA events, keeps the fastest and returns it. Renders those frames. */
fiber_status fiber_batch_tune(fiber_batch* batch, void* stream, fiber_batch_tuning* best);
fiber_status fiber_batch_destroy(fiber_batch* batch);
/* Host only (no device): the branch of each view for the given frame costs,
 * branch count and order, as fiber_batch_launch assigns them. */
fiber_status fiber_batch_plan(const float* costs, uint32_t n, uint32_t branches, uint32_t order,
                              uint32_t* assign);

/* ------------------------------------------------------------------------ */
/* Page prefix without device allocation (no counterpart in the reference)   */
/* ------------------------------------------------------------------------ */
/* The froxel-page prefix of fiber_prepass as a standalone call for callers
 * that cannot allocate device memory where they run it: an engine that hands
 * out all GPU memory from its own pool, or code inside CUDA stream capture,
 * where cudaMalloc is not allowed. All buffers are the caller's device
 * memory: counts[pages * 256] (froxel counts, cell = (z * 4 + y) * 4 + x),
 * offsets[pages * 256] (exclusive prefix within each page), page_base[pages]
 * (first reference of each page, pages in order; 0 for an empty page) and
 * totals[2] (total references; non-zero if a bounded device wait gave up,
 * written by the last block to finish).
 * The only scratch is a fixed file-scope device array (8 B per page, for at
 * most 65536 pages = 512 KiB) that every GPU loading the library keeps until
 * exit; more pages return FIBER_EINVAL. Nothing is allocated or freed. The
 * first call on a device looks up the array's address with that device
 * current, so make it before any stream capture; the address is kept for the
 * life of the process, so after cudaDeviceReset (which may move the array)
 * reload the library before calling again. Every call shares the array
 * and clears the part it uses: calls that overlap on the GPU (two streams, or
 * two host threads on one device) race. Work is queued on `stream`. */
fiber_status fiber_prefix_pages_noalloc(const uint32_t* counts, uint32_t pages, uint32_t* offsets,
                                        uint32_t* page_base, uint32_t* totals, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FIBER_H */
