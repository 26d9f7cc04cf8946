// gb_nufft_convolve_nc2c_noalloc: the gridding (NC2C) convolution without
// any device allocation, for callers that cannot call cudaMalloc.
//
// Who needs it: code that runs where allocating is not allowed or not safe --
// inside a host callback or a real-time thread with a fixed memory budget, or
// in a process whose device memory is owned by another allocator (a framework
// caching allocator that must not be bypassed).  The regular entry point (gb_nufft_convolve with
// GB_CONV_NC2C) allocates the scratch of its split-tile reduction lazily with
// cudaMalloc; this one takes it from a fixed array in device memory instead.
//
// The scratch is a file-scope __device__ array of kScratchBytes (16 MiB) that
// every GPU which loads this library keeps until the process exits.  Host code
// cannot pass the array's name to a kernel (on the host it is only a stand-in
// symbol), so the first call on each device looks up its device address with
// cudaGetSymbolAddress while that device is current, and caches it.  That
// first call should therefore come before any stream capture.
//
// All calls share the one array and it keeps the last call's contents: the
// counters of the split-tile reduction are cleared (cudaMemsetAsync) before
// every launch, the partial tiles are always written before they are read.
// Calls that overlap on the GPU (other streams, other threads) race on the
// array and must be serialised by the caller.
#include <mutex>
#include <vector>

#include "gb_internal.cuh"
#include "gb_ops.hpp"

namespace gb {

namespace {

constexpr size_t kScratchBytes = 16u << 20;       // 16 MiB per device
constexpr size_t kCounterBytes = 64u << 10;       // first 64 KiB: counters
constexpr size_t kCounterElems = kCounterBytes / sizeof(unsigned int);
constexpr size_t kPartialElems = (kScratchBytes - kCounterBytes) / sizeof(float2);

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
std::vector<void *> g_scratch_ptr;   // per device, filled on first use

void *scratch_for_current_device() {
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(g_mu);
    if ((int)g_scratch_ptr.size() <= dev) g_scratch_ptr.resize(dev + 1, nullptr);
    if (!g_scratch_ptr[dev]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            cudaGetLastError();
            fail(GB_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") +
                                  cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = ptr;
    }
    return g_scratch_ptr[dev];
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" GB_API gb_status gb_nufft_convolve_nc2c_noalloc(gb_nufft_plan plan, const void *samples, void *grid,
                                                           int accumulate, uint32_t num_batches, void *stream) {
    try {
        NufftPlan *p = plan_from_handle(plan);
        if (!p) fail(GB_ERR_INVALID_ARGUMENT, "NULL plan");
        if (!samples || !grid) fail(GB_ERR_INVALID_ARGUMENT, "NULL input/output");
        const int nb = count_arg(num_batches, "number of batches");
        if (!p->prepped) fail(GB_ERR_NOT_PREPROCESSED, "preprocess has not been called");
        int old = -1;
        check_cuda(cudaGetDevice(&old), "cudaGetDevice");
        if (old != p->device) check_cuda(cudaSetDevice(p->device), "cudaSetDevice");
        struct Restore {
            int dev, cur;
            ~Restore() { if (dev != cur && dev >= 0) cudaSetDevice(dev); }
        } restore{old, p->device};
        size_t need_partials = 0, need_counters = 0;
        grid_scratch_need(*p, nb, &need_partials, &need_counters);
        if (need_partials > kPartialElems || need_counters > kCounterElems)
            fail(GB_ERR_INVALID_ARGUMENT,
                 "gb_nufft_convolve_nc2c_noalloc: this plan and batch count need " +
                     std::to_string(need_partials * sizeof(float2) + need_counters * sizeof(unsigned int)) +
                     " bytes of scratch, above the fixed " + std::to_string(kScratchBytes) + "-byte buffer");
        unsigned char *base = static_cast<unsigned char *>(scratch_for_current_device());
        unsigned int *counters = reinterpret_cast<unsigned int *>(base);
        float2 *partials = reinterpret_cast<float2 *>(base + kCounterBytes);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        if (need_counters) check_cuda(cudaMemsetAsync(counters, 0, need_counters * sizeof(unsigned int), st),
                                      "cudaMemsetAsync");
        launch_grid_external_scratch(*p, static_cast<const float2 *>(samples), static_cast<float2 *>(grid),
                                     nb, accumulate != 0, partials, counters, st);
        return GB_OK;
    } catch (...) {
        return current_exception_status();
    }
}
