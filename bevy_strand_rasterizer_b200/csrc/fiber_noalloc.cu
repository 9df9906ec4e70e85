// fiber_noalloc.cu — the froxel-page prefix with no device allocation.
//
// Some callers cannot allocate device memory at the point where they run the
// binning step: an engine that hands out every byte of GPU memory from its own
// pool (allocating around the pool would break its budget and can stall the
// device), or code running inside CUDA stream capture, where cudaMalloc is not
// allowed at all. fiber_prefix_pages_noalloc serves them: the caller passes
// its own input and output buffers, and the only scratch the kernel needs (the
// decoupled look-back status words) lives in one file-scope __device__ array
// of fixed size that every GPU loading this library holds until exit.
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "fiber_kernels.cuh"

namespace fiber {

// Largest page count one call accepts; the scratch is 8 B per page (512 KiB).
constexpr uint32_t kNoAllocMaxPages = 65536;
// Scratch words ahead of the look-back status words: [0] page claim counter,
// [1] error word, [2] finished-block counter, [3] reference total.
constexpr uint32_t kNoAllocHeadWords = 4;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocMaxPages + kNoAllocHeadWords];

// One block per page, in page order: exclusive scan of the page's 256 cell
// counts -> offsets; the page's reference base from a decoupled look-back over
// pages (prefix_fine_pages, strand_prepass.wgsl:2051-2143, with the ordered
// base the CUDA path uses instead of the reference's atomic tail). The block
// that finishes last writes totals: by then every block has set the error
// word if one of its waits gave up.
__global__ void __launch_bounds__(256) k_prefix_pages_noalloc(const uint32_t* __restrict__ counts, uint32_t pages,
                                                              uint32_t* __restrict__ offsets,
                                                              uint32_t* __restrict__ page_base,
                                                              uint32_t* __restrict__ totals,
                                                              unsigned long long* scratch) {
    __shared__ uint32_t s_page;
    __shared__ uint32_t s_warp[33];
    uint32_t* counter = reinterpret_cast<uint32_t*>(scratch);
    uint32_t* error = reinterpret_cast<uint32_t*>(scratch + 1);
    uint32_t* done = reinterpret_cast<uint32_t*>(scratch + 2);
    uint32_t* ref_total = reinterpret_cast<uint32_t*>(scratch + 3);
    unsigned long long* status = scratch + kNoAllocHeadWords;
    for (;;) {
        if (threadIdx.x == 0) s_page = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t page = s_page;
        if (page >= pages) break;
        const size_t g = (size_t)page * kPageSize + threadIdx.x;
        const uint32_t c = counts[g];
        uint32_t total;
        const uint32_t excl = block_exclusive_scan<256>(c, s_warp, total);
        offsets[g] = excl;
        if (threadIdx.x == 0) {
            const uint32_t base = lb_exclusive(status, page, 1u, total, error);
            page_base[page] = total > 0u ? base : 0u;
            if (page == pages - 1u) *((volatile uint32_t*)ref_total) = base + total;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(done, 1u) == gridDim.x - 1u) {
            __threadfence();
            totals[0] = *((volatile uint32_t*)ref_total);
            totals[1] = *((volatile uint32_t*)error);
        }
    }
}

namespace {
std::mutex g_setup_mutex;
unsigned long long* g_scratch_ptr[64] = {};
}  // namespace

}  // namespace fiber

using namespace fiber;

extern "C" fiber_status fiber_prefix_pages_noalloc(const uint32_t* counts, uint32_t pages, uint32_t* offsets,
                                                   uint32_t* page_base, uint32_t* totals, void* stream_) {
    if (pages > kNoAllocMaxPages) return FIBER_EINVAL;
    if (!totals || (pages && (!counts || !offsets || !page_base))) return FIBER_EINVAL;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return FIBER_ECUDA;
    }
    cudaStream_t s = (cudaStream_t)stream_;
    unsigned long long* scratch = nullptr;
    {
        // Set-up, once per device with that device current: the symbol's
        // host-side name is not a device address, so its address is fetched.
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return FIBER_ECUDA;
            }
            g_scratch_ptr[dev] = static_cast<unsigned long long*>(p);
        }
        scratch = g_scratch_ptr[dev];
    }
    // The counters, the error word and this call's status words must start at
    // zero; the array keeps the previous call's contents.
    if (cudaMemsetAsync(scratch, 0, ((size_t)pages + kNoAllocHeadWords) * sizeof(unsigned long long), s) !=
        cudaSuccess) {
        cudaGetLastError();
        return FIBER_ECUDA;
    }
    if (pages == 0) {
        if (cudaMemsetAsync(totals, 0, 2 * sizeof(uint32_t), s) != cudaSuccess) {
            cudaGetLastError();
            return FIBER_ECUDA;
        }
        return FIBER_OK;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    unsigned blocks = (unsigned)std::min<uint64_t>(pages, (uint64_t)sms * 6u);
    k_prefix_pages_noalloc<<<blocks, 256, 0, s>>>(counts, pages, offsets, page_base, totals, scratch);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FIBER_OK : FIBER_ECUDA;
}
