// ref_gpu_hermitian.cu — the reference's default Jᴴ·v path (GemmFast) on the B200 ("reference
// kernels, re-hosted").
//
// TEST INFRASTRUCTURE / BASELINE ONLY. Its own translation unit, as in the reference, because
// src/jacobian/hermitian_kernels.cuh and product_kernels.cuh both define compute_sample_decay.
// Restates src/jacobian/hermitian.cu:140-240 (compute_jacobian_hermitian_gemm<float>, one voxel
// chunk, TF32 as the C ABI's default: julia-bindings/src/bindings.cpp:335) around the reference's
// unmodified kernels (compute_sample_decay_hermitian, jacobian_hermitian_product_finalize,
// convert_complex_to_planar) and its cuBLAS calls (ref_gpu_gemm.cuh).
#include <cuda_runtime.h>

#include "kernel_float.h"  // the stand-in; some reference kernel headers use it without including it
#include "jacobian/hermitian_kernels.cuh"
#include "ref_gpu_gemm.cuh"
#include "utils/gemm_kernels.cuh"

using compas::cfloat;
using kmm::host_view;

extern "C" {

// Jᴴ·v [4][V] from echos, dT1, dT2 [R][V], coils [C][V], vector [C][R][S]
void ref_gpu_jacobian_hermitian(float* params, int V, float* echos, float* dT1, float* dT2, float* coils, int C,
                                int R, int S, float dt, float* k_start, float dk, float* vector, float* JHv,
                                void* stream_ptr) {
    auto stream = static_cast<cudaStream_t>(stream_ptr);
    const compas::TissueParametersView pv(host_view(params, 9, V));
    compas::CartesianTrajectoryView traj;
    traj.nreadouts = R;
    traj.samples_per_readout = S;
    traj.delta_t = dt;
    traj.k_start = host_view(reinterpret_cast<cfloat*>(k_start), R);
    traj.delta_k = cfloat(dk, 0.0f);
    float* E_H = ref_gpu::scratch("jhv.E_H", size_t(2) * V * S);
    float* dE_H = ref_gpu::scratch("jhv.dEdT2_H", size_t(2) * V * S);
    float* Ev = ref_gpu::scratch("jhv.Ev", size_t(2) * R * V);
    float* dEv = ref_gpu::scratch("jhv.dEdT2v", size_t(2) * R * V);
    float* vlo = ref_gpu::scratch("jhv.vector_lo", size_t(2) * R * S);
    auto* out = reinterpret_cast<cfloat*>(JHv);
    auto* vin = reinterpret_cast<cfloat*>(vector);
    cudaMemsetAsync(out, 0, sizeof(cfloat) * 4 * size_t(V), stream);
    const auto div_up = [](int64_t a, unsigned b) { return unsigned((a + b - 1) / b); };
    compas::kernels::compute_sample_decay_hermitian<float>
        <<<dim3(div_up(S, 64), div_up(V, 4)), dim3(64, 4), 0, stream>>>(
            kmm::Bounds<2, int> {{0, S}, {0, V}, {}}, host_view(E_H, 2, V, S), host_view(dE_H, 2, V, S), traj, pv);
    for (int c = 0; c < C; c++) {
        compas::kernels::convert_complex_to_planar<float><<<dim3(div_up(S, 32), div_up(R, 4)), dim3(32, 4), 0, stream>>>(
            R, S, host_view(vlo, 2, R, S), host_view(vin + int64_t(c) * R * S, R, S));
        ref_gpu::complex_gemm(stream, Ev, vlo, E_H, R, V, S, 1.0f, 0.0f, CUBLAS_COMPUTE_32F_FAST_TF32);
        ref_gpu::complex_gemm(stream, dEv, vlo, dE_H, R, V, S, 1.0f, 0.0f, CUBLAS_COMPUTE_32F_FAST_TF32);
        compas::kernels::jacobian_hermitian_product_finalize<<<div_up(V, 256), 256, 0, stream>>>(
            kmm::Range<int> {0, V}, R, c, host_view(out, 4, V), host_view(reinterpret_cast<cfloat*>(echos), R, V),
            host_view(reinterpret_cast<cfloat*>(dT1), R, V), host_view(reinterpret_cast<cfloat*>(dT2), R, V), pv,
            host_view(reinterpret_cast<cfloat*>(coils), C, V), host_view(Ev, 2, R, V), host_view(dEv, 2, R, V));
    }
}

int ref_gpu_hermitian_out_of_bounds(void) {
    unsigned int flag = 0;
    if (cudaMemcpyFromSymbol(&flag, kmm_ref_out_of_bounds, sizeof(flag)) != cudaSuccess) return -1;
    return flag ? 1 : 0;
}

}  // extern "C"
