// fiber_server.cu — the served mode: continuous batching of render requests
// over scenes kept resident on the device.
//
// A server owns S slots. A slot is a fiber_ctx with its own streams and
// worker thread and buffers sized at start for the largest scene at the
// configured maximum frame, so that serving never allocates. The scenes'
// slabs are uploaded once and shared by every slot: a slot switches scenes by
// loading the shared scene's instance table (host side, no validation kernel,
// no device synchronisation). The slot count is what the HBM budget admits:
// (budget - slab bytes) / (bytes of one sized slot's frame buffers), at most
// kMaxSlots.
//
// Requests queue in arrival order; each worker takes the next request as soon
// as its previous frame has been read back, so requests that arrive while
// others are on the GPU are admitted as slots free up, and the frames of
// different slots overlap on the device. A request's frame runs at a stream
// priority set by its admission order: the oldest frame in flight at the
// highest, the frames admitted behind it at lower ones, so the device gives
// the oldest request its blocks first and the younger ones fill the SMs it
// leaves idle (first come, first served, with backfill).
//
// The temporal shadow history is off on every slot, so a request's image is
// the same whichever requests ran before it or next to it.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>

#include "fiber.h"
#include "fiber_internal.h"

namespace {

constexpr uint32_t kMaxSlots = 64;
constexpr uint32_t kDefaultSlots = 8;  // slots = 0 without an HBM budget
constexpr uint32_t kMaxLevels = 8;     // stream priority levels used

struct Slot {
    fiber_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;               // sizing frames
    std::vector<cudaStream_t> streams, sides;    // per priority level: the frame's stream and its side branch
    std::thread worker;
};

struct Pending {
    uint64_t ticket;
    fiber_server_request req;
};

// Inverse of a column-major 4x4 matrix (cofactor expansion in double).
void invert4(const float* m, float* out) {
    double a[16], inv[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] +
             a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] -
             a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] +
             a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] -
              a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] -
             a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] +
             a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] -
             a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] +
              a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] +
             a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] -
             a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] +
              a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] -
              a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] -
             a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] +
             a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] -
              a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] +
              a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    const double det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
    const double s = det != 0.0 ? 1.0 / det : 0.0;
    for (int i = 0; i < 16; ++i) out[i] = (float)(inv[i] * s);
}

}  // namespace

struct fiber_server {
    int device = 0;
    fiber_settings settings{};
    fiber_server_config cfg{};
    std::vector<Slot> slots;
    std::vector<fiber_scene_state*> scenes;  // instance tables over slot 0's slabs, shared by all slots
    std::vector<uint64_t> scene_segments;
    uint64_t slab_bytes = 0;                 // device bytes of the resident scenes
    std::vector<int> priorities;             // stream priority of each level, highest first
    uint32_t in_flight = 0;                  // frames rendering now (under mu)
    void* zero_scene = nullptr;  // pinned transparent background, max frame
    void* warm_out = nullptr;    // pinned scratch output of the sizing frames
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> queue;
    std::unordered_map<uint64_t, fiber_server_result> done;
    std::unordered_set<uint64_t> outstanding;  // submitted, not yet collected by fiber_server_wait
    uint64_t next_ticket = 1;
    bool started = false, stopping = false;
    std::atomic<uint32_t> rerenders{0};  // frames rendered again after a reference overflow
};

uint64_t fiber_server_now_ns(void) {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

namespace {

void release_slot(Slot& s) {
    if (s.ctx) fiber_ctx_destroy(s.ctx);
    if (s.stream) cudaStreamDestroy(s.stream);
    for (cudaStream_t x : s.streams) cudaStreamDestroy(x);
    for (cudaStream_t x : s.sides) cudaStreamDestroy(x);
    s = Slot{};
}

fiber_status make_slot(fiber_server* srv, Slot& s) {
    fiber_status st = fiber_ctx_create(srv->device, 0, &s.ctx);
    if (st == FIBER_OK) st = fiber_settings_set(s.ctx, &srv->settings);
    if (st == FIBER_OK && cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess) st = FIBER_ECUDA;
    for (size_t l = 0; l < srv->priorities.size() && st == FIBER_OK; ++l) {
        cudaStream_t a = nullptr, b = nullptr;
        if (cudaStreamCreateWithPriority(&a, cudaStreamNonBlocking, srv->priorities[l]) != cudaSuccess ||
            cudaStreamCreateWithPriority(&b, cudaStreamNonBlocking, srv->priorities[l]) != cudaSuccess) {
            cudaGetLastError();
            if (a) cudaStreamDestroy(a);
            st = FIBER_ECUDA;
            break;
        }
        s.streams.push_back(a);
        s.sides.push_back(b);
    }
    return st;
}

// One request on one slot at priority `level` (nullptr streams: the sizing
// stream); returns when its image is in host memory. A frame whose references
// overflowed the slot's capacity (sized from the segment count,
// src/plugin.rs:483-576) raises the slot's reference capacity to what the
// frame asked for and renders again, so no request returns a truncated
// image; the slot keeps the larger capacity for later requests.
fiber_status render(fiber_server* srv, Slot& slot, const fiber_server_request& r, uint32_t* renders,
                    int level = -1) {
    fiber_status st = fiber_ctx_load_scene(slot.ctx, srv->scenes[r.scene]);
    const cudaStream_t stream = level < 0 ? slot.stream : slot.streams[level];
    fiber_ctx_set_side_stream(slot.ctx, level < 0 ? nullptr : slot.sides[level]);
    const void* bg = r.scene_rgba16f ? r.scene_rgba16f : srv->zero_scene;
    for (int attempt = 0; st == FIBER_OK && attempt < 3; ++attempt) {
        if (renders) *renders = (uint32_t)attempt + 1u;
        st = fiber_frame_begin(slot.ctx, &r.camera_cfg, &r.camera, r.light_cfgs, r.lights, r.n_lights, stream);
        if (st == FIBER_OK) st = fiber_ctx_render_host_nodes(slot.ctx, bg, r.out_rgba16f, stream);
        if (cudaStreamSynchronize(stream) != cudaSuccess && st == FIBER_OK) st = FIBER_ECUDA;
        if (st == FIBER_OK) st = fiber_ctx_frame_status(slot.ctx, stream);
        if (st != FIBER_EOVERFLOW || !fiber_ctx_grow_refs(slot.ctx, stream)) break;
        st = FIBER_OK;
        srv->rerenders.fetch_add(1u);
    }
    return st;
}

// Predicted cost of a request: segments x frusta + camera pixels + shadow
// texels (as fiber_ctx_frame_cost), and its priority level under
// FIBER_PRIORITY_COST: 0 (highest) for the costliest request the server can
// get (the largest scene at the largest shape), one level lower per halving.
uint64_t request_cost(const fiber_server* srv, const fiber_server_request& r) {
    uint64_t c = srv->scene_segments[r.scene] * (1u + r.n_lights) +
                 (uint64_t)r.camera_cfg.screen_width * r.camera_cfg.screen_height;
    for (uint32_t l = 0; l < r.n_lights; ++l)
        c += (uint64_t)r.light_cfgs[l].screen_width * r.light_cfgs[l].screen_height;
    return std::max<uint64_t>(c, 1u);
}

uint32_t cost_level(const fiber_server* srv, const fiber_server_request& r) {
    uint64_t top = 1u;
    for (uint64_t segs : srv->scene_segments) top = std::max<uint64_t>(top, segs);
    top = top * (1u + srv->cfg.max_lights) + (uint64_t)srv->cfg.max_width * srv->cfg.max_height +
          (uint64_t)srv->cfg.max_lights * srv->cfg.max_dom * srv->cfg.max_dom;
    const uint64_t c = request_cost(srv, r);
    uint32_t level = 0;
    while (level + 1u < srv->priorities.size() && (c << (level + 1u)) <= top) ++level;
    return level;
}

void worker_main(fiber_server* srv, uint32_t si) {
    cudaSetDevice(srv->device);
    Slot& slot = srv->slots[si];
    for (;;) {
        Pending p;
        uint32_t level = 0;
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            srv->cv_work.wait(lk, [&] { return srv->stopping || !srv->queue.empty(); });
            if (srv->queue.empty()) return;
            p = srv->queue.front();
            srv->queue.pop_front();
            level = srv->cfg.priority_order == FIBER_PRIORITY_COST
                        ? cost_level(srv, p.req)
                        : std::min<uint32_t>(srv->in_flight, (uint32_t)srv->priorities.size() - 1u);
            ++srv->in_flight;
        }
        fiber_server_result res{};
        res.slot = si;
        res.priority = level;
        res.arrival_ns = p.req.arrival_ns;
        res.admit_ns = fiber_server_now_ns();
        res.status = render(srv, slot, p.req, &res.renders, (int)level);
        res.done_ns = fiber_server_now_ns();
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            --srv->in_flight;
            srv->done[p.ticket] = res;
        }
        srv->cv_done.notify_all();
    }
}

}  // namespace

fiber_status fiber_server_create(int device, const fiber_settings* settings, const fiber_server_config* cfg,
                                 fiber_server** out) {
    if (!cfg || !out) return FIBER_EINVAL;
    *out = nullptr;
    if (cfg->slots > kMaxSlots || cfg->max_width == 0 || cfg->max_height == 0 || cfg->priority_order > 1u ||
        cfg->max_lights > FIBER_SERVER_MAX_LIGHTS || (cfg->max_lights && cfg->max_dom == 0))
        return FIBER_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return FIBER_EINVAL;
    }
    fiber_server* srv = new fiber_server();
    srv->device = device;
    srv->cfg = *cfg;
    if (settings) srv->settings = *settings;
    else fiber_settings_default(&srv->settings);
    srv->settings.history_enabled = 0u;
    // Priority levels, highest first (CUDA: a lower number is a higher priority).
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) {
        cudaGetLastError();
        least = greatest = 0;
    }
    const uint32_t want = cfg->priority_levels ? std::min<uint32_t>(cfg->priority_levels, kMaxLevels) : kMaxLevels;
    for (int pr = greatest; pr <= least && srv->priorities.size() < want; ++pr) srv->priorities.push_back(pr);
    if (srv->priorities.empty()) srv->priorities.push_back(0);
    // Slot 0 holds the scenes' slabs; the other slots are made at start.
    srv->slots.resize(1);
    const fiber_status st = make_slot(srv, srv->slots[0]);
    if (st != FIBER_OK) {
        release_slot(srv->slots[0]);
        delete srv;
        return st;
    }
    *out = srv;
    return FIBER_OK;
}

fiber_status fiber_server_add_scene(fiber_server* srv, const fiber_server_scene* sc, uint32_t* scene_id) {
    if (!srv || !sc || !scene_id || srv->started) return FIBER_EINVAL;
    if (!sc->vertices || !sc->indices || !sc->meta || !sc->materials || !sc->n_vertices || !sc->n_indices ||
        !sc->n_meta || !sc->n_materials)
        return FIBER_EINVAL;
    cudaSetDevice(srv->device);
    const uint64_t bytes[5] = {(uint64_t)sc->n_vertices * 16u, (uint64_t)sc->n_indices * 4u,
                               (uint64_t)sc->n_meta * sizeof(fiber_strand_meta), sizeof(fiber_strand_geo),
                               (uint64_t)sc->n_materials * sizeof(fiber_strand_material)};
    const void* src[5] = {sc->vertices, sc->indices, sc->meta, &sc->geo, sc->materials};
    const uint32_t kinds[5] = {FIBER_SLAB_VERT, FIBER_SLAB_INDEX, FIBER_SLAB_META, FIBER_SLAB_GEO,
                               FIBER_SLAB_MATERIAL};
    Slot& s = srv->slots[0];
    uint32_t ids[5];
    for (int k = 0; k < 5; ++k) {
        fiber_devptr dp;
        fiber_status st = fiber_slab_alloc(s.ctx, kinds[k], bytes[k], &ids[k], &dp);
        if (st == FIBER_OK) st = fiber_slab_upload(s.ctx, kinds[k], ids[k], 0, src[k], bytes[k], nullptr);
        if (st != FIBER_OK) return st;
        srv->slab_bytes += bytes[k];
    }
    fiber_strand_instance row;
    std::memset(&row, 0, sizeof(row));
    row.vertex_id = ids[0];
    row.index_id = ids[1];
    row.meta_id = ids[2];
    row.geo_id = ids[3];
    row.material_id = ids[4];
    std::memcpy(row.world_from_local, sc->world_from_local, sizeof(row.world_from_local));
    invert4(sc->world_from_local, row.local_from_world);
    const fiber_status st = fiber_instance_set(s.ctx, &row, 1u);
    if (st != FIBER_OK) return st;
    srv->scenes.push_back(fiber_ctx_save_scene(s.ctx));
    srv->scene_segments.push_back(fiber_scene_segments(srv->scenes.back()));
    *scene_id = (uint32_t)(srv->scene_segments.size() - 1u);
    return FIBER_OK;
}

namespace {

// One frame of the largest scene at the configured maximum shape, so that the
// slot's buffers never grow while serving.
fiber_status size_slot(fiber_server* srv, Slot& s) {
    uint32_t big = 0;
    for (uint32_t i = 1; i < srv->scene_segments.size(); ++i)
        if (srv->scene_segments[i] > srv->scene_segments[big]) big = i;
    fiber_server_request r;
    std::memset(&r, 0, sizeof(r));
    r.scene = big;
    r.n_lights = srv->cfg.max_lights;
    r.camera_cfg = fiber_froxel_config{srv->cfg.max_width, srv->cfg.max_height, 8u, 8u, 64u};
    for (int i = 0; i < 16; i += 5) r.camera.clip_from_world[i] = 1.0f;
    for (uint32_t l = 0; l < r.n_lights; ++l) {
        r.light_cfgs[l] = fiber_froxel_config{srv->cfg.max_dom, srv->cfg.max_dom, 8u, 8u, 64u};
        for (int i = 0; i < 16; i += 5) r.lights[l].clip_from_world[i] = 1.0f;
        r.lights[l].direction_to_light[1] = 1.0f;
    }
    r.out_rgba16f = srv->warm_out;
    const fiber_status st = render(srv, s, r, nullptr);
    return st == FIBER_EOVERFLOW ? FIBER_OK : st;  // the sizing frame's image is not used
}

}  // namespace

fiber_status fiber_server_start(fiber_server* srv, uint32_t* slots_started) {
    if (!srv || srv->started || srv->scene_segments.empty()) return FIBER_EINVAL;
    cudaSetDevice(srv->device);
    const size_t frame_bytes = (size_t)srv->cfg.max_width * srv->cfg.max_height * 8u;
    if (cudaHostAlloc(&srv->zero_scene, frame_bytes, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc(&srv->warm_out, frame_bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return FIBER_ENOMEM;
    }
    std::memset(srv->zero_scene, 0, frame_bytes);
    fiber_status st = size_slot(srv, srv->slots[0]);
    if (st != FIBER_OK) return st;
    // Admission by HBM budget: the slabs once, then as many sized slots as the
    // rest of the budget holds.
    // A slot whose request outgrows its reference capacity grows it (render),
    // so each slot is counted at 1.5 times its sized bytes: the headroom that
    // lets half the slots double their reference buffers within the budget.
    const uint64_t held = fiber_ctx_allocated(srv->slots[0].ctx);
    const uint64_t sized = held > srv->slab_bytes ? held - srv->slab_bytes : held;
    const uint64_t per_slot = std::max<uint64_t>(1, sized + sized / 2u);
    uint32_t n = srv->cfg.slots ? srv->cfg.slots : (srv->cfg.hbm_budget ? kMaxSlots : kDefaultSlots);
    if (srv->cfg.hbm_budget) {
        const uint64_t room = srv->cfg.hbm_budget > srv->slab_bytes ? srv->cfg.hbm_budget - srv->slab_bytes : 0u;
        n = (uint32_t)std::min<uint64_t>(n, std::max<uint64_t>(1, room / per_slot));
    }
    srv->slots.resize(n);
    for (uint32_t i = 1; i < n && st == FIBER_OK; ++i) {
        st = make_slot(srv, srv->slots[i]);
        if (st == FIBER_OK) st = size_slot(srv, srv->slots[i]);
    }
    if (st != FIBER_OK) return st;
    srv->started = true;
    for (uint32_t i = 0; i < n; ++i) srv->slots[i].worker = std::thread(worker_main, srv, i);
    if (slots_started) *slots_started = n;
    return FIBER_OK;
}

fiber_status fiber_server_submit(fiber_server* srv, const fiber_server_request* req, uint64_t* ticket) {
    if (!srv || !req || !ticket || !srv->started) return FIBER_EINVAL;
    const fiber_server_config& c = srv->cfg;
    if (req->scene >= srv->scene_segments.size() || !req->out_rgba16f || req->n_lights > c.max_lights ||
        req->camera_cfg.screen_width == 0 || req->camera_cfg.screen_height == 0 ||
        req->camera_cfg.screen_width > c.max_width || req->camera_cfg.screen_height > c.max_height)
        return FIBER_EINVAL;
    for (uint32_t l = 0; l < req->n_lights; ++l)
        if (req->light_cfgs[l].screen_width > c.max_dom || req->light_cfgs[l].screen_height > c.max_dom)
            return FIBER_EINVAL;
    Pending p;
    p.req = *req;
    if (!p.req.arrival_ns) p.req.arrival_ns = fiber_server_now_ns();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        if (srv->stopping) return FIBER_EINVAL;
        p.ticket = srv->next_ticket++;
        srv->outstanding.insert(p.ticket);
        srv->queue.push_back(p);
    }
    srv->cv_work.notify_one();
    *ticket = p.ticket;
    return FIBER_OK;
}

fiber_status fiber_server_wait(fiber_server* srv, uint64_t ticket, fiber_server_result* out) {
    if (!srv || !out || ticket == 0) return FIBER_EINVAL;
    std::unique_lock<std::mutex> lk(srv->mu);
    if (!srv->outstanding.count(ticket)) return FIBER_EINVAL;  // unknown, or already collected
    srv->cv_done.wait(lk, [&] { return srv->done.count(ticket) != 0; });
    *out = srv->done[ticket];
    srv->done.erase(ticket);
    srv->outstanding.erase(ticket);
    return FIBER_OK;
}

fiber_status fiber_server_destroy(fiber_server* srv) {
    if (!srv) return FIBER_EINVAL;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stopping = true;
    }
    srv->cv_work.notify_all();
    for (Slot& s : srv->slots)
        if (s.worker.joinable()) s.worker.join();
    cudaSetDevice(srv->device);
    // Slot 0 owns the slabs every scene state points into: release it last.
    for (size_t i = srv->slots.size(); i-- > 0;) release_slot(srv->slots[i]);
    for (fiber_scene_state* st : srv->scenes) fiber_scene_state_free(st);
    if (srv->zero_scene) cudaFreeHost(srv->zero_scene);
    if (srv->warm_out) cudaFreeHost(srv->warm_out);
    delete srv;
    return FIBER_OK;
}
