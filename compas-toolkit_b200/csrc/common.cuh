// common.cuh — shared host/device helpers of the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "compas/compas.h"

namespace compas {

// Device status word bits. Kernels never trap: they set a bit and return, and the host
// raises CompasException at the next synchronisation point.
enum : unsigned int {
    STATUS_WAIT_TIMEOUT = 1u << 0,
    STATUS_BAD_ARGUMENT = 1u << 1,
    STATUS_TMEM = 1u << 2,
};
const char* status_message(unsigned int value);

namespace detail {
unsigned int* device_status_word(int device);
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int device) {
        int cur = 0;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != device) {
            prev = cur;
            cudaSetDevice(device);
        }
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

void fill_float(float* ptr, int64_t n, float value, cudaStream_t stream);

// number of kernels this library has launched (process-wide), see compas_b200_launch_count
void note_launch();

inline void check_launch(const char* what) {
    note_launch();
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) throw_exception(__FILE__, __LINE__, std::string(what) + ": " + cudaGetErrorString(err));
}

inline int div_ceil(int a, int b) {
    return (a + b - 1) / b;
}

// ------------------------------------------------------------------------------------------
// device complex arithmetic on float2 {re, im}
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
    return make_float2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    return make_float2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ float2 cscale(float s, float2 a) {
    return make_float2(s * a.x, s * a.y);
}
__device__ __forceinline__ float2 cconj(float2 a) {
    return make_float2(a.x, -a.y);
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {  // c + a*b
    return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

// ------------------------------------------------------------------------------------------
// two-wide FP32 arithmetic of sm_100 (FADD2 / FMUL2 / FFMA2): one instruction performs the
// same round-to-nearest operation on .x and on .y, so two independent operands travel through
// one issue slot. Results equal the scalar operations bit for bit.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    return __fadd2_rn(a, b);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d)
        : "l"(*reinterpret_cast<const unsigned long long*>(&a)), "l"(*reinterpret_cast<const unsigned long long*>(&b)));
    return *reinterpret_cast<const float2*>(&d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    return __fmul2_rn(a, b);
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {  // a*b + c, one rounding
    return __ffma2_rn(a, b, c);
}
__device__ __forceinline__ float2 bcast2(float s) {
    return make_float2(s, s);
}

// L2 eviction policy "keep": lines written with it are evicted after other lines (PTX createpolicy)
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void st_l2_hint(float2* ptr, float2 v, uint64_t policy) {
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(ptr), "f"(v.x), "f"(v.y), "l"(policy)
                 : "memory");
}

// e^{i·2π·turns}: accurate for any magnitude of `turns` (sincospi reduces exactly)
__device__ __forceinline__ float2 cis_turns(double turns) {
    double frac = turns - rint(turns);  // exact in FP64 for |turns| < 2^52
    float s, c;
    sincospif(2.0f * float(frac), &s, &c);
    return make_float2(c, s);
}

// e^{iθ} with θ in radians, range-reduced modulo 2π in FP64 before the FP32 sincos
__device__ __forceinline__ float2 cis_rad(double theta) {
    constexpr double inv_2pi = 0.15915494309189533577;
    return cis_turns(theta * inv_2pi);
}

}  // namespace compas
