// Host definitions of the CUDA built-ins that compas-toolkit's simulation kernels use, so that
// oracle/ref_sim.cpp can run those kernels (src/simulate/fisp_kernels.cuh,
// src/simulate/pssfp_kernels.cuh, src/operators/{epg,isochromat}.cuh) one thread at a time on the
// CPU. TEST INFRASTRUCTURE ONLY. The fast-math intrinsics map to the exact libm functions, so the
// golden values are the reference's formulas in FP32 with correctly rounded transcendentals.
#pragma once
#include <cmath>
#include <sys/types.h>

#include "kernel_float.h"

// Launch coordinates per host thread: each thread runs its own one-thread launches. Shared
// memory becomes a per-thread static, which is what one thread per block sees.
struct compas_ref_dim3 {
    unsigned x = 0, y = 0, z = 0;
};
inline thread_local compas_ref_dim3 threadIdx, blockIdx, blockDim {1, 1, 1}, gridDim {1, 1, 1};

#define __global__
#define __device__
#define __shared__ static thread_local
#define __launch_bounds__(...)
#define KMM_ASSUME(expr) ((void)0)
#define __builtin_assume(expr) ((void)0)

// CUDA's global min / max
#include <algorithm>
using std::max;
using std::min;

struct float2 {
    float x, y;
};

inline void __syncwarp() {}
inline void __syncthreads() {}

// Warp shuffles for a warp size of 1 (the only one these host launches use): the source lane
// is always outside the one-lane segment, so a shuffle returns the caller's own value. The
// reference's headers test COMPAS_IS_CUDA with #ifdef, which is true on the host too (it is
// defined as 0), so they reach these.
inline float __shfl_sync(unsigned, float v, int, int = 32) { return v; }
inline float __shfl_up_sync(unsigned, float v, unsigned, int = 32) { return v; }
inline float __shfl_down_sync(unsigned, float v, unsigned, int = 32) { return v; }
inline float __shfl_xor_sync(unsigned, float v, int, int = 32) { return v; }
inline float __expf(float x) { return std::exp(x); }
inline float __cosf(float x) { return std::cos(x); }
inline void __sincosf(float x, float* s, float* c) {
    *s = std::sin(x);
    *c = std::cos(x);
}
inline float rhypotf(float a, float b) { return 1.0f / std::hypot(a, b); }

// one-thread groups: the kernels run with a warp size of 1, so no shuffle is ever taken
namespace cooperative_groups {
struct thread_block {};
inline thread_block this_thread_block() { return {}; }
template<int N>
struct thread_block_tile {
    unsigned size() const { return N; }
    unsigned thread_rank() const { return threadIdx.x % N; }
    template<typename T>
    T shfl_down(T v, unsigned) const { return v; }
};
template<int N>
thread_block_tile<N> tiled_partition(thread_block) { return {}; }
}  // namespace cooperative_groups
