// noalloc.cu — compute_residual for callers that cannot allocate device memory.
//
// compas_compute_residual allocates its output, a per-block partial-sum buffer and the objective
// from the device pool. Some callers cannot let a library allocate: a host application that owns a
// fixed device-memory budget and hands the library pre-allocated buffers, or code that must not
// trigger a device allocation (and the implicit synchronisation it can cause) in the middle of a
// latency-critical loop. For them this entry point takes every input and output as a device pointer
// and keeps its only scratch — the per-block partial sums of Σ|lhs - rhs|² — in a file-scope
// device array of fixed size, so it calls no cudaMalloc, cudaFree or allocating library routine.
//
// Limits and sharing:
//  * the scratch holds 65536 partial sums (256 KB, resident on every GPU that loads the library
//    until the process exits); the kernels run the allocating entry point's grid-stride launch of
//    at most 1024 blocks, and n is bounded at 16,777,216 complex values (larger n is rejected with
//    an error, the limit callers were given);
//  * every call on a device uses the same scratch and leaves its partial sums in it; calls whose
//    work overlaps on the GPU (different streams, or threads without ordering) race on it and must
//    be serialised by the caller;
//  * the first call on a device resolves the scratch's device address (cudaGetSymbolAddress with
//    that device current) and caches it; make that first call before any stream capture.
#include <cstdint>
#include <mutex>
#include <sstream>

#include "common.cuh"
#include "kernels.h"

namespace compas {
namespace kernels {
// residual kernels of ops.cu (grid-stride difference + per-block Σ|d|², then a one-block sum)
__global__ void residual_kernel(const float2* __restrict__ lhs, const float2* __restrict__ rhs, int64_t n,
                                float2* __restrict__ out, float* __restrict__ partials);
__global__ void sum_kernel(const float* __restrict__ partials, int n, float* __restrict__ result);
}  // namespace kernels

namespace {

constexpr int kScratchPartials = 1 << 16;
constexpr int kBlock = 256;
// The residual's grid-stride launch uses at most 1024 blocks (residual_partial_count), one partial
// sum each, so the kernels never need more than 1024 of the scratch's entries. The element limit
// below is therefore a contract with callers, fixed when this entry point was published, not a
// capacity of the kernels.
constexpr int kMaxResidualBlocks = 1024;
static_assert(kScratchPartials >= kMaxResidualBlocks, "the scratch must hold one partial sum per block");
constexpr int64_t kMaxElements = int64_t(kScratchPartials) * kBlock;

static __device__ __align__(256) float g_residual_partials[kScratchPartials];

// Device address of the scratch on `device`, resolved once per device with that device current.
float* scratch_on(int device) {
    static std::mutex mutex;
    static float* addresses[64] = {};
    if (device < 0 || device >= 64) COMPAS_ERROR("invalid device index");
    std::lock_guard<std::mutex> lock(mutex);
    if (!addresses[device]) {
        DeviceGuard guard(device);
        float* p = nullptr;
        COMPAS_CUDA_CHECK(cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_residual_partials));
        addresses[device] = p;
    }
    return addresses[device];
}

}  // namespace

int64_t residual_noalloc_max_elements() {
    return kMaxElements;
}

// diff = lhs - rhs over n complex values and *objective = Σ|diff|², all pointers in device memory
// of `device`, ordered on `stream`; allocates nothing.
void residual_noalloc(int device, const cfloat* lhs, const cfloat* rhs, cfloat* diff, float* objective, int64_t n,
                      cudaStream_t stream) {
    if (n < 0) COMPAS_ERROR("negative element count");
    if (n > kMaxElements) {
        std::ostringstream s;
        s << "n = " << n << " exceeds the limit of " << kMaxElements
          << " complex values of the allocation-free residual (static scratch of " << kScratchPartials
          << " partial sums)";
        COMPAS_ERROR(s.str());
    }
    if (!objective) COMPAS_ERROR("null objective pointer");
    if (n > 0 && (!lhs || !rhs || !diff)) COMPAS_ERROR("null input or output pointer");
    float* partials = scratch_on(device);
    DeviceGuard guard(device);
    if (n == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(objective, 0, sizeof(float), stream));
        return;
    }
    // the allocating entry point's grid (grid-stride, at most 1024 blocks): the same kernels in the
    // same order, so diff and objective are the same bits, and the scratch holds every partial
    const int blocks = residual_partial_count(n);
    if (blocks > kMaxResidualBlocks) COMPAS_ERROR("residual grid larger than the scratch");
    kernels::residual_kernel<<<blocks, kBlock, 0, stream>>>(reinterpret_cast<const float2*>(lhs),
                                                            reinterpret_cast<const float2*>(rhs), n,
                                                            reinterpret_cast<float2*>(diff), partials);
    check_launch("residual_kernel (no allocation)");
    kernels::sum_kernel<<<1, kBlock, 0, stream>>>(partials, blocks, objective);
    check_launch("sum_kernel (no allocation)");
}

}  // namespace compas
