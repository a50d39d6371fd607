// ref_gpu.cu — the reference's FISP and pSSFP kernels built for the B200 ("reference kernels,
// re-hosted").
//
// TEST INFRASTRUCTURE / BASELINE ONLY. Built by oracle/Makefile (target `ref`) into
// oracle/_ref/libref_gpu.so from the reference's unmodified kernel headers (include and src trees
// on the include path, nothing copied) with the reference's own CUDA flags (COMPAS_USE_CUDA=1,
// --use_fast_math) and the kmm / kernel_float stand-ins of oracle/refshim. The reference cannot be
// built as shipped (its kmm runtime submodule is empty), so the host side here restates its launch
// code with the same shapes:
//  * FISP: src/simulate/fisp.cu:13-100 — per max_state class a (max_N, warp_size) instantiation,
//    256 threads per block as (warp_size, 256/warp_size), one launch of kernels::simulate_fisp per
//    slice position accumulating into zeroed transposed echoes [nv][nTR], then
//    kernels::expand_undersampled_echos with 32x32 blocks (fisp.cu:125-137);
//  * pSSFP: src/simulate/pssfp.cu:8-66 — zeroed echoes, then kernels::simulate_pssfp<batch> for
//    batches of 32, 16, 8, 4, 2, 1 z positions, 256 threads per block.
// Every view index in device code is bounds-checked by the stand-in (refshim/kmm/core/view.hpp);
// ref_gpu_out_of_bounds() reports whether any check fired.
#include <cuda_runtime.h>

#include "simulate/fisp_kernels.cuh"
#include "simulate/pssfp_kernels.cuh"

using compas::cfloat;
using kmm::host_view;

namespace {

unsigned div_up(unsigned a, unsigned b) {
    return (a + b - 1) / b;
}

template<int max_N, int warp_size>
void fisp_for_size(int nv, cfloat* transposed, const compas::TissueParametersView& pv,
                   const compas::FISPSequenceView& seq, int nTR, int P, cudaStream_t stream) {
    constexpr int threads_per_block = 256;
    constexpr int warps_per_block = threads_per_block / warp_size;
    cudaMemsetAsync(transposed, 0, sizeof(cfloat) * size_t(nv) * nTR, stream);
    const dim3 block(warp_size, warps_per_block);
    const dim3 grid(1, div_up(unsigned(nv), warps_per_block));
    const auto tview = host_view(transposed, nv, nTR);
    for (int i = 0; i < P; i++)
        compas::kernels::simulate_fisp<max_N, warp_size, warps_per_block><<<grid, block, 0, stream>>>(
            kmm::Range<int> {0, nv}, tview, seq.sliceprofiles.drop_axis(i), pv, seq);
}

template<int batch>
int pssfp_batch(int nv, int iz, int nz, float* z, cfloat* echos, int nTR, const compas::TissueParametersView& pv,
                const compas::pSSFPSequenceView& seq, cudaStream_t stream) {
    const unsigned threads = 256;
    const unsigned grid = div_up(unsigned(nv * batch), threads);
    while (iz + batch <= nz) {
        compas::kernels::simulate_pssfp<batch><<<grid, threads, 0, stream>>>(nv, host_view(echos, nTR, nv),
                                                                              host_view(z + iz, batch), pv, seq);
        iz += batch;
    }
    return iz;
}

}  // namespace

extern "C" {

// FISP echoes [nTR*uf][nv] into `echos`, with `transposed` [nv][nTR] as scratch; all pointers are
// device memory, params [9][nv] float, rf [nTR] and slices [P][nTR] complex. Returns 0, or -1
// for max_state > 128.
int ref_gpu_fisp(float* params, int nv, float* rf, float* slices, int nTR, int P, float TR, float TE, float TW,
                 float TI, int max_state, int uf, int reps, float* transposed, float* echos, void* stream_ptr) {
    auto stream = static_cast<cudaStream_t>(stream_ptr);
    compas::TissueParametersView pv(host_view(params, 9, nv));
    compas::FISPSequenceView seq;
    seq.RF_train = host_view(reinterpret_cast<cfloat*>(rf), nTR);
    seq.sliceprofiles = host_view(reinterpret_cast<cfloat*>(slices), P, nTR);
    seq.TR = TR;
    seq.TE = TE;
    seq.TW = TW;
    seq.max_state = max_state;
    seq.TI = TI;
    seq.undersampling_factor = uf;
    seq.repetitions = reps;
    seq.inversion_prepulse = true;  // the C ABI's FISP sequence (julia-bindings/src/bindings.cpp:151-174)
    seq.wait_spoiling = true;
    auto* t = reinterpret_cast<cfloat*>(transposed);
    if (max_state <= 4) fisp_for_size<4, 2>(nv, t, pv, seq, nTR, P, stream);
    else if (max_state <= 8) fisp_for_size<8, 4>(nv, t, pv, seq, nTR, P, stream);
    else if (max_state <= 16) fisp_for_size<16, 8>(nv, t, pv, seq, nTR, P, stream);
    else if (max_state <= 32) fisp_for_size<32, 16>(nv, t, pv, seq, nTR, P, stream);
    else if (max_state <= 64) fisp_for_size<64, 32>(nv, t, pv, seq, nTR, P, stream);
    else if (max_state <= 96) fisp_for_size<96, 32>(nv, t, pv, seq, nTR, P, stream);
    else if (max_state <= 128) fisp_for_size<128, 32>(nv, t, pv, seq, nTR, P, stream);
    else return -1;
    const int R = nTR * uf;
    const dim3 block(32, 32), grid(div_up(unsigned(nv), 32), div_up(unsigned(R), 32));
    compas::kernels::expand_undersampled_echos<<<grid, block, 0, stream>>>(
        kmm::Range<int> {0, nv}, kmm::Range<int> {0, R}, uf, host_view(reinterpret_cast<cfloat*>(echos), R, nv),
        host_view(t, nv, nTR));
    return 0;
}

// pSSFP echoes [nTR][nv]; device pointers: params [9][nv], rf [nTR] and gamma_dt_RF [nRF] complex,
// z [nz]; dt / gz = {ex, inv, pr}.
int ref_gpu_pssfp(float* params, int nv, float* rf, int nTR, float TR, float* gamma_dt_RF, int nRF, const float* dt,
                  const float* gz, float* z, int nz, float* echos, void* stream_ptr) {
    auto stream = static_cast<cudaStream_t>(stream_ptr);
    compas::TissueParametersView pv(host_view(params, 9, nv));
    compas::pSSFPSequenceView seq;
    seq.nTR = nTR;
    seq.RF_train = host_view(reinterpret_cast<cfloat*>(rf), nTR);
    seq.TR = TR;
    seq.gamma_dt_RF = host_view(reinterpret_cast<cfloat*>(gamma_dt_RF), nRF);
    seq.dt = {dt[0], dt[1], dt[2]};
    seq.gamma_dt_GRz = {gz[0], gz[1], gz[2]};
    seq.z = host_view(z, nz);
    auto* e = reinterpret_cast<cfloat*>(echos);
    cudaMemsetAsync(e, 0, sizeof(cfloat) * size_t(nTR) * nv, stream);
    int iz = 0;
    iz = pssfp_batch<32>(nv, iz, nz, z, e, nTR, pv, seq, stream);
    iz = pssfp_batch<16>(nv, iz, nz, z, e, nTR, pv, seq, stream);
    iz = pssfp_batch<8>(nv, iz, nz, z, e, nTR, pv, seq, stream);
    iz = pssfp_batch<4>(nv, iz, nz, z, e, nTR, pv, seq, stream);
    iz = pssfp_batch<2>(nv, iz, nz, z, e, nTR, pv, seq, stream);
    iz = pssfp_batch<1>(nv, iz, nz, z, e, nTR, pv, seq, stream);
    return iz == nz ? 0 : -1;
}

// 1 when a device view index of any launch so far was out of range (and clamped), else 0;
// -1 when the flag could not be read
int ref_gpu_out_of_bounds(void) {
    unsigned int flag = 0;
    if (cudaMemcpyFromSymbol(&flag, kmm_ref_out_of_bounds, sizeof(flag)) != cudaSuccess) return -1;
    return flag ? 1 : 0;
}

}  // extern "C"
