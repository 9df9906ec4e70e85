// fiber_batch.cu — the batched mode: many independent views rendered by one
// CUDA graph launch.
//
// Each view is a caller-owned fiber_ctx holding its own strand set, settings
// and frame tables (fiber_frame_begin). The batch captures one replayable
// frame per view (fiber_ctx_enqueue_frame) into a single graph whose views are
// spread over B branches: the capture forks the launch stream into B
// non-blocking streams and joins them at the end, so views on different
// branches run concurrently on the device while each branch runs its views in
// turn. A replay is one cudaGraphLaunch for the whole batch, and every frame
// in it advances its look-back epoch and history on the device, so replays
// need no host work per view. The graph is recaptured when a view's frame
// shape changes (buffers, grid sizes, clear extents) or the tuning does.
//
// Tuning (fiber_batch_tune): every candidate (branch count x view order) is
// captured and timed over a few replays with events on the launch stream, and
// the fastest is kept. View order 1 hands views longest first to the least
// loaded branch (LPT) by their predicted frame cost.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "fiber.h"
#include "fiber_internal.h"

namespace {

constexpr uint32_t kMaxBranches = 32;
constexpr int kTuneReps = 3;

#define BATCH_CUDA(expr)                           \
    do {                                           \
        if ((expr) != cudaSuccess) {               \
            cudaGetLastError();                    \
            return FIBER_ECUDA;                    \
        }                                          \
    } while (0)

// Views in enqueue order and their branches.
void plan(const float* costs, uint32_t n, uint32_t branches, uint32_t order, uint32_t* assign, uint32_t* seq) {
    for (uint32_t v = 0; v < n; ++v) seq[v] = v;
    if (order == FIBER_BATCH_ORDER_LPT) {
        std::stable_sort(seq, seq + n, [&](uint32_t a, uint32_t b) { return costs[a] > costs[b]; });
        std::vector<double> load(branches, 0.0);
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t b = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
            assign[seq[i]] = b;
            load[b] += costs[seq[i]];
        }
    } else {
        for (uint32_t v = 0; v < n; ++v) assign[v] = v % branches;
    }
}

}  // namespace

struct fiber_batch {
    int device = 0;
    std::vector<fiber_ctx*> views;
    fiber_batch_tuning tuning{1u, FIBER_BATCH_ORDER_INDEX, 0.0f, 0u};
    cudaStream_t streams[kMaxBranches] = {};
    cudaEvent_t fork = nullptr, joins[kMaxBranches] = {}, t0 = nullptr, t1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    fiber_batch_tuning graph_tuning{};
    std::vector<uint64_t> graph_keys;
};

namespace {

void shape_keys(const fiber_batch* b, std::vector<uint64_t>& keys) {
    keys.assign(b->views.size() * kFrameShapeWords, 0u);
    for (size_t v = 0; v < b->views.size(); ++v) fiber_ctx_shape_key(b->views[v], keys.data() + v * kFrameShapeWords);
}

fiber_status capture(fiber_batch* b, cudaStream_t s0) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    const uint32_t n = (uint32_t)b->views.size();
    const uint32_t nb = std::max(1u, std::min(b->tuning.branches, std::min(n, kMaxBranches)));
    std::vector<float> costs(n);
    for (uint32_t v = 0; v < n; ++v) costs[v] = (float)fiber_ctx_frame_cost(b->views[v]);
    std::vector<uint32_t> assign(n), seq(n);
    plan(costs.data(), n, nb, b->tuning.order, assign.data(), seq.data());
    BATCH_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    fiber_status st = FIBER_OK;
    cudaError_t ce = cudaEventRecord(b->fork, s0);
    for (uint32_t i = 0; i < nb && ce == cudaSuccess; ++i) ce = cudaStreamWaitEvent(b->streams[i], b->fork, 0);
    if (ce != cudaSuccess) st = FIBER_ECUDA;
    for (uint32_t i = 0; i < n && st == FIBER_OK; ++i) st = fiber_ctx_enqueue_frame(b->views[seq[i]], b->streams[assign[seq[i]]]);
    // Join every branch that was forked, also after an error, so the capture ends cleanly.
    for (uint32_t i = 0; i < nb; ++i) {
        if (cudaEventRecord(b->joins[i], b->streams[i]) != cudaSuccess ||
            cudaStreamWaitEvent(s0, b->joins[i], 0) != cudaSuccess)
            st = st == FIBER_OK ? FIBER_ECUDA : st;
    }
    cudaGraph_t g = nullptr;
    ce = cudaStreamEndCapture(s0, &g);
    if (st == FIBER_OK && ce != cudaSuccess) st = FIBER_ECUDA;
    if (st == FIBER_OK && cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) st = FIBER_ECUDA;
    if (g) cudaGraphDestroy(g);
    if (st != FIBER_OK) {
        cudaGetLastError();
        b->graph = nullptr;
        return st;
    }
    b->graph_tuning = b->tuning;
    shape_keys(b, b->graph_keys);
    return FIBER_OK;
}

fiber_status launch(fiber_batch* b, cudaStream_t s0) {
    std::vector<uint64_t> keys;
    shape_keys(b, keys);
    const bool stale = !b->graph || keys != b->graph_keys || b->graph_tuning.branches != b->tuning.branches ||
                       b->graph_tuning.order != b->tuning.order;
    if (stale) {
        const fiber_status st = capture(b, s0);
        if (st != FIBER_OK) return st;
    }
    BATCH_CUDA(cudaGraphLaunch(b->graph, s0));
    for (fiber_ctx* c : b->views) fiber_ctx_mark_replayed(c, s0);
    return FIBER_OK;
}

}  // namespace

extern "C" {

fiber_status fiber_batch_plan(const float* costs, uint32_t n, uint32_t branches, uint32_t order, uint32_t* assign) {
    if ((n && (!costs || !assign)) || branches == 0u || order > FIBER_BATCH_ORDER_LPT) return FIBER_EINVAL;
    std::vector<uint32_t> seq(n);
    plan(costs, n, branches, order, assign, seq.data());
    return FIBER_OK;
}

fiber_status fiber_batch_create(fiber_ctx* const* views, uint32_t n, fiber_batch** out) {
    if (!out || !views || n == 0u) return FIBER_EINVAL;
    *out = nullptr;
    const int device = fiber_ctx_device(views[0]);
    for (uint32_t v = 0; v < n; ++v)
        if (!views[v] || fiber_ctx_device(views[v]) != device) return FIBER_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return FIBER_ECUDA;
    fiber_batch* b = new fiber_batch();
    b->device = device;
    b->views.assign(views, views + n);
    bool ok = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreate(&b->t0) == cudaSuccess && cudaEventCreate(&b->t1) == cudaSuccess;
    for (uint32_t i = 0; i < kMaxBranches && ok; ++i)
        ok = cudaStreamCreateWithFlags(&b->streams[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        fiber_batch_destroy(b);
        return FIBER_ECUDA;
    }
    *out = b;
    return FIBER_OK;
}

fiber_status fiber_batch_set_tuning(fiber_batch* b, const fiber_batch_tuning* t) {
    if (!b || !t || t->branches == 0u || t->branches > kMaxBranches || t->order > FIBER_BATCH_ORDER_LPT)
        return FIBER_EINVAL;
    b->tuning.branches = t->branches;
    b->tuning.order = t->order;
    return FIBER_OK;
}

fiber_status fiber_batch_get_tuning(const fiber_batch* b, fiber_batch_tuning* t) {
    if (!b || !t) return FIBER_EINVAL;
    *t = b->tuning;
    return FIBER_OK;
}

fiber_status fiber_batch_launch(fiber_batch* b, void* stream) {
    if (!b || !stream) return FIBER_EINVAL;  // the legacy stream cannot be captured
    if (cudaSetDevice(b->device) != cudaSuccess) return FIBER_ECUDA;
    return launch(b, (cudaStream_t)stream);
}

fiber_status fiber_batch_tune(fiber_batch* b, void* stream, fiber_batch_tuning* best_out) {
    if (!b || !stream) return FIBER_EINVAL;
    if (cudaSetDevice(b->device) != cudaSuccess) return FIBER_ECUDA;
    cudaStream_t s0 = (cudaStream_t)stream;
    const uint32_t n = (uint32_t)b->views.size();
    fiber_batch_tuning best{0u, 0u, 0.0f, 0u};
    for (uint32_t nb = 1; nb <= std::min(n, kMaxBranches); nb *= 2) {
        for (uint32_t order = FIBER_BATCH_ORDER_INDEX; order <= FIBER_BATCH_ORDER_LPT; ++order) {
            if (nb == 1u && order == FIBER_BATCH_ORDER_LPT) continue;  // one branch: order only permutes
            b->tuning.branches = nb;
            b->tuning.order = order;
            fiber_status st = launch(b, s0);  // captures, and warms the candidate up
            if (st != FIBER_OK) return st;
            BATCH_CUDA(cudaEventRecord(b->t0, s0));
            for (int r = 0; r < kTuneReps && st == FIBER_OK; ++r) st = launch(b, s0);
            if (st != FIBER_OK) return st;
            BATCH_CUDA(cudaEventRecord(b->t1, s0));
            BATCH_CUDA(cudaEventSynchronize(b->t1));
            float ms = 0.0f;
            BATCH_CUDA(cudaEventElapsedTime(&ms, b->t0, b->t1));
            ms /= (float)kTuneReps;
            if (best.branches == 0u || ms < best.ms) best = fiber_batch_tuning{nb, order, ms, 0u};
        }
    }
    b->tuning = best;
    if (best_out) *best_out = best;
    return FIBER_OK;
}

fiber_status fiber_batch_destroy(fiber_batch* b) {
    if (!b) return FIBER_EINVAL;
    cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (uint32_t i = 0; i < kMaxBranches; ++i) {
        if (b->streams[i]) {
            cudaStreamSynchronize(b->streams[i]);
            cudaStreamDestroy(b->streams[i]);
        }
        if (b->joins[i]) cudaEventDestroy(b->joins[i]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->t0) cudaEventDestroy(b->t0);
    if (b->t1) cudaEventDestroy(b->t1);
    delete b;
    return FIBER_OK;
}

}  // extern "C"
