// fiber_internal.h — hooks between the context runtime (fiber_ctx.cu) and the
// request server (fiber_server.cu). Library-internal: not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fiber.h"

// A context's instance table with everything fiber_instance_set derives from
// it (validated device views, segment totals). Saving one per resident scene
// lets a context switch scenes between frames on the host alone: no
// validation kernel, no device synchronisation.
struct fiber_scene_state;

fiber_scene_state* fiber_ctx_save_scene(const fiber_ctx* c);
fiber_status fiber_ctx_load_scene(fiber_ctx* c, const fiber_scene_state* s);
void fiber_scene_state_free(fiber_scene_state* s);
uint64_t fiber_scene_segments(const fiber_scene_state* s);

// fiber_render_host with the node sequence launched directly on `s` (no graph
// capture), for callers whose frame shape changes from frame to frame.
fiber_status fiber_ctx_render_host_nodes(fiber_ctx* c, const void* scene_host, void* out_host, cudaStream_t s);

// Device bytes the context holds.
uint64_t fiber_ctx_allocated(const fiber_ctx* c);

// After a frame on `s` whose references overflowed: raises the context's
// reference capacity to what the frame's cells asked for, for the next
// fiber_frame_begin; returns true when it did (re-render the frame).
bool fiber_ctx_grow_refs(fiber_ctx* c, cudaStream_t s);

// After the frame on `s` completed: ETIMEDOUT if a bounded device wait gave
// up, EOVERFLOW if a queue dropped work, else OK. Reads two counter words.
fiber_status fiber_ctx_frame_status(fiber_ctx* c, cudaStream_t s);

// Batched mode (fiber_batch.cu). One replayable frame of a context on `s`,
// for capture into a batch graph: a device-side frame advance (next look-back
// epoch, shadow-history flip), the per-frame clears, then the prepass, shadow,
// shading and raster nodes. The frame tables are the ones the last
// fiber_frame_begin uploaded.
fiber_status fiber_ctx_enqueue_frame(fiber_ctx* c, cudaStream_t s);
// What the captured launches bake in (buffers, grid sizes, clear extents); a
// batch graph is recaptured when any of its views' keys changes.
constexpr int kFrameShapeWords = 6;
void fiber_ctx_shape_key(const fiber_ctx* c, uint64_t key[kFrameShapeWords]);
// After a batch graph ran a context's frame: the host epoch no longer follows
// the device's, so the next fiber_frame_begin restarts it; readbacks of the
// context wait for `s`, the stream the batch ran on.
void fiber_ctx_mark_replayed(fiber_ctx* c, cudaStream_t s);
// Predicted frame cost: segments x frusta + camera pixels + DOM texels.
uint64_t fiber_ctx_frame_cost(const fiber_ctx* c);
int fiber_ctx_device(const fiber_ctx* c);
// The stream the prepass's cell sort forks onto beside the frame's own stream
// (nullptr: the context's). The request server passes one of the frame's
// priority, so both branches of a frame run at the same stream priority.
void fiber_ctx_set_side_stream(fiber_ctx* c, cudaStream_t side);
