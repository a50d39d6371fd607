// ref_gpu_products.cu — the reference's default Cartesian signal (MatmulFast) and J·v (GemmFast)
// paths on the B200 ("reference kernels, re-hosted").
//
// TEST INFRASTRUCTURE / BASELINE ONLY. The kernels are the reference's unmodified
// src/trajectories/signal_kernels.cuh, src/jacobian/product_kernels.cuh and
// src/utils/gemm_kernels.cuh; their launches restate the host code with the same shapes and the
// cuBLAS calls of src/utils/gemm.cu (ref_gpu_gemm.cuh), in TF32 as the C ABI's defaults select
// (julia-bindings/src/bindings.cpp:264, 307: low_precision = 0 → MatmulFast / GemmFast):
//  * signal: src/trajectories/signal.cu:103-156 (magnetization_to_signal_cartesian_gemm<float>);
//  * J·v: src/jacobian/product.cu:201-285 (compute_jacobian_gemm<float>), one voxel chunk;
//  * spiral signal: src/trajectories/signal.cu:170-240 (its only spiral method, no cuBLAS).
#include <cuda_runtime.h>

#include "kernel_float.h"  // the stand-in; some reference kernel headers use it without including it
#include "jacobian/product_kernels.cuh"
#include "ref_gpu_gemm.cuh"
#include "trajectories/signal_kernels.cuh"
#include "utils/gemm_kernels.cuh"

using compas::cfloat;
using kmm::host_view;

namespace {

unsigned div_up(int64_t a, unsigned b) {
    return unsigned((a + b - 1) / b);
}

compas::CartesianTrajectoryView cartesian(int R, int S, float dt, float* k_start, float dk) {
    compas::CartesianTrajectoryView t;
    t.nreadouts = R;
    t.samples_per_readout = S;
    t.delta_t = dt;
    t.k_start = host_view(reinterpret_cast<cfloat*>(k_start), R);
    t.delta_k = cfloat(dk, 0.0f);  // the C ABI passes a real Δk (julia-bindings/src/bindings.cpp:198-212)
    return t;
}

}  // namespace

extern "C" {

// signal [C][R][S] from echos [R][V], coils [C][V] (all device pointers, complex interleaved)
void ref_gpu_signal_cartesian(float* params, int V, float* echos, float* coils, int C, int R, int S, float dt,
                              float* k_start, float dk, float* signal, void* stream_ptr) {
    auto stream = static_cast<cudaStream_t>(stream_ptr);
    const compas::TissueParametersView pv(host_view(params, 9, V));
    const auto traj = cartesian(R, S, dt, k_start, dk);
    float* factors = ref_gpu::scratch("signal.factors", size_t(2) * R * V);
    float* exponents = ref_gpu::scratch("signal.exponents", size_t(2) * S * V);
    float* temp = ref_gpu::scratch("signal.temp", size_t(2) * R * S);
    auto* ec = reinterpret_cast<cfloat*>(echos);
    auto* cc = reinterpret_cast<cfloat*>(coils);
    auto* sc = reinterpret_cast<cfloat*>(signal);
    compas::kernels::prepare_readout_echos_planar<float><<<dim3(div_up(V, 32), div_up(R, 4)), dim3(32, 4), 0, stream>>>(
        kmm::Range<int> {0, V}, kmm::Range<int> {0, R}, host_view(factors, 2, R, V), host_view(ec, R, V), pv, traj);
    for (int c = 0; c < C; c++) {
        compas::kernels::prepare_sample_decay_cartesian_with_coil<float><<<div_up(V, 256), 256, 0, stream>>>(
            kmm::Range<int> {0, V}, S, host_view(exponents, 2, S, V), host_view(cc + int64_t(c) * V, V), pv, traj);
        ref_gpu::complex_gemm(stream, temp, factors, exponents, R, S, V, 1.0f, 0.0f, CUBLAS_COMPUTE_32F_FAST_TF32);
        compas::kernels::convert_planar_to_complex<float><<<dim3(div_up(S, 32), div_up(R, 4)), dim3(32, 4), 0, stream>>>(
            R, S, host_view(sc + int64_t(c) * R * S, R, S), host_view(temp, 2, R, S));
    }
}

// J·v [C][R][S] from echos, dT1, dT2 [R][V], coils [C][V], v [4][V]
void ref_gpu_jacobian(float* params, int V, float* echos, float* dT1, float* dT2, float* coils, int C, int R, int S,
                      float dt, float* k_start, float dk, float* vector, float* Jv, void* stream_ptr) {
    auto stream = static_cast<cudaStream_t>(stream_ptr);
    const compas::TissueParametersView pv(host_view(params, 9, V));
    const auto traj = cartesian(R, S, dt, k_start, dk);
    float* E = ref_gpu::scratch("jv.E", size_t(2) * S * V);
    float* dE = ref_gpu::scratch("jv.dEdT2", size_t(2) * S * V);
    float* adj_phase = ref_gpu::scratch("jv.adj_phase", size_t(2) * R * V);
    float* adj_decay = ref_gpu::scratch("jv.adj_decay", size_t(2) * R * V);
    float* jv_coil = ref_gpu::scratch("jv.coil", size_t(2) * R * S);
    auto ev = host_view(reinterpret_cast<cfloat*>(echos), R, V);
    auto d1 = host_view(reinterpret_cast<cfloat*>(dT1), R, V);
    auto d2 = host_view(reinterpret_cast<cfloat*>(dT2), R, V);
    auto cv = host_view(reinterpret_cast<cfloat*>(coils), C, V);
    auto vv = host_view(reinterpret_cast<cfloat*>(vector), 4, V);
    auto* out = reinterpret_cast<cfloat*>(Jv);
    compas::kernels::compute_sample_decay_planar<float><<<dim3(div_up(V, 32), div_up(S, 8)), dim3(32, 8), 0, stream>>>(
        kmm::Bounds<2, int> {{0, V}, {0, S}, {}}, host_view(E, 2, S, V), host_view(dE, 2, S, V), traj, pv);
    for (int c = 0; c < C; c++) {
        compas::kernels::compute_adjoint_sources_with_coil<float>
            <<<dim3(div_up(V, 32), div_up(R, 8)), dim3(32, 8), 0, stream>>>(
                kmm::Bounds<2, int> {{0, V}, {0, R}, {}}, host_view(adj_phase, 2, R, V), host_view(adj_decay, 2, R, V),
                c, cv, ev, d1, d2, vv, pv);
        ref_gpu::complex_gemm(stream, jv_coil, adj_phase, E, R, S, V, 1.0f, 0.0f, CUBLAS_COMPUTE_32F_FAST_TF32);
        ref_gpu::complex_gemm(stream, jv_coil, adj_decay, dE, R, S, V, 1.0f, 1.0f, CUBLAS_COMPUTE_32F_FAST_TF32);
        compas::kernels::convert_planar_to_complex<float><<<dim3(div_up(S, 32), div_up(R, 4)), dim3(32, 4), 0, stream>>>(
            R, S, host_view(out + int64_t(c) * R * S, R, S), host_view(jv_coil, 2, R, S));
    }
}

// spiral signal [C][R][S] from echos [R][V], coils [C][V], per-readout k_start and Δk [R] (complex):
// src/trajectories/signal.cu:170-240 (magnetization_to_signal_spiral) with its launch shapes
void ref_gpu_signal_spiral(float* params, int V, float* echos, float* coils, int C, int R, int S, float dt,
                           float* k_start, float* delta_k, float* signal, void* stream_ptr) {
    auto stream = static_cast<cudaStream_t>(stream_ptr);
    const compas::TissueParametersView pv(host_view(params, 9, V));
    compas::SpiralTrajectoryView traj;
    traj.nreadouts = R;
    traj.samples_per_readout = S;
    traj.delta_t = dt;
    traj.k_start = host_view(reinterpret_cast<cfloat*>(k_start), R);
    traj.delta_k = host_view(reinterpret_cast<cfloat*>(delta_k), R);
    auto* readout_echos = reinterpret_cast<cfloat*>(ref_gpu::scratch("spiral.readout_echos", size_t(2) * R * V));
    auto* decay = reinterpret_cast<cfloat*>(ref_gpu::scratch("spiral.sample_decay", size_t(2) * R * V));
    const dim3 block(32, 4), grid(div_up(V, 32), div_up(R, 4));
    compas::kernels::prepare_readout_echos<<<grid, block, 0, stream>>>(
        kmm::Range<int> {0, V}, kmm::Range<int> {0, R}, host_view(readout_echos, R, V),
        host_view(reinterpret_cast<cfloat*>(echos), R, V), pv, traj);
    compas::kernels::prepare_sample_decay_spiral<<<grid, block, 0, stream>>>(host_view(decay, R, V), pv, traj);
    constexpr unsigned threads_per_block = 64, threads_cooperative = 32, samples_per_thread = 8,
                       coils_per_thread = 1;
    const dim3 sgrid(div_up(int64_t(div_up(S, samples_per_thread)) * threads_cooperative, threads_per_block),
                     unsigned(R), div_up(C, coils_per_thread));
    compas::kernels::sum_signal_spiral<threads_per_block, threads_cooperative, samples_per_thread, coils_per_thread>
        <<<sgrid, threads_per_block, 0, stream>>>(host_view(reinterpret_cast<cfloat*>(signal), C, R, S),
                                                  host_view(decay, R, V), host_view(readout_echos, R, V),
                                                  host_view(reinterpret_cast<cfloat*>(coils), C, V));
}

int ref_gpu_products_out_of_bounds(void) {
    unsigned int flag = 0;
    if (cudaMemcpyFromSymbol(&flag, kmm_ref_out_of_bounds, sizeof(flag)) != cudaSuccess) return -1;
    return flag ? 1 : 0;
}

}  // extern "C"
