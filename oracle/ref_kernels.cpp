// ref_kernels.cpp — the reference's FISP and Cartesian-signal kernels as a host library.
//
// TEST INFRASTRUCTURE / CPU BASELINE ONLY. Built by oracle/Makefile (target `ref`) into
// oracle/_ref/libref_kernels.so from the reference's own sources (include and src trees on the
// include path, nothing copied) with the host stand-ins of oracle/refshim. It lets the CPU baseline
// and the reference arm of bench.py time the reference's own code on the host cores, and the tests
// compare the oracle with it:
//  * ref_fisp: kernels::simulate_fisp<max_N, 1, 1> (src/simulate/fisp_kernels.cuh:225-241) as a
//    one-thread launch per (slice position, voxel), positions accumulated as src/simulate/fisp.cu:35-48
//    does, then the undersampling expansion of kernels::expand_undersampled_echos (:243-257);
//    voxels are spread over OpenMP threads;
//  * ref_signal_cartesian_entries: kernels::sum_signal_cartesian_naive
//    (src/trajectories/signal_kernels.cuh:137-167) for selected (coil, readout, sample) entries, each
//    a sum over all voxels, entries spread over OpenMP threads.
#include <omp.h>

#include <cstdint>
#include <vector>

#include "simulate/fisp_kernels.cuh"
#include "trajectories/signal_kernels.cuh"

using compas::cfloat;
using kmm::host_view;

namespace {

template<int max_N>
void fisp_voxels(float* params, int64_t nv, const int* vidx, int64_t nidx, cfloat* rf, cfloat* slices, int nTR,
                 int P, const compas::FISPSequenceView& base, cfloat* out, int nthreads) {
    const int uf = base.undersampling_factor, R = nTR * uf;
    compas::TissueParametersView pv;
    pv.parameters = host_view(params, 9, nv);
#pragma omp parallel num_threads(nthreads)
    {
        compas::FISPSequenceView seq = base;
        seq.RF_train = host_view(rf, nTR);
        seq.sliceprofiles = host_view(slices, P, nTR);
        std::vector<cfloat> row(nTR);
#pragma omp for schedule(dynamic, 1)
        for (int64_t q = 0; q < nidx; q++) {
            const int v = vidx ? vidx[q] : int(q);
            std::fill(row.begin(), row.end(), cfloat(0));
            // the voxel's transposed echo row [nTR]; the kernel addresses it as row `voxel` of a
            // [nv][nTR] view, so give it a view with a zero voxel stride, every row of which is
            // this buffer
            kmm::View<cfloat, 2> tview;
            tview.ptr = row.data();
            tview.ext[0] = nv;
            tview.ext[1] = nTR;
            tview.str[0] = 0;
            tview.str[1] = 1;
            for (int i = 0; i < P; i++) {
                blockDim = {1, 1, 1};
                blockIdx = {0, unsigned(v), 0};
                threadIdx = {0, 0, 0};
                compas::kernels::simulate_fisp<max_N, 1, 1>(kmm::Range<int> {0, int(nv)}, tview,
                                                            seq.sliceprofiles.drop_axis(i), pv, seq);
            }
            for (int r = 0; r < R; r++) out[int64_t(r) * nidx + q] = row[r / uf];
        }
    }
}

}  // namespace

extern "C" {

// echoes [nTR*uf][nidx] of the voxels vidx (all voxels when vidx is NULL); returns 0, or -1 for
// max_state > 128
int ref_fisp(float* params, int64_t nv, const int* vidx, int64_t nidx, float* rf, float* slices, int nTR, int P,
             float TR, float TE, float TW, float TI, int max_state, int uf, int reps, int inversion, int wait_spoil,
             float* out, int nthreads) {
    compas::FISPSequenceView seq;
    seq.TR = TR;
    seq.TE = TE;
    seq.TW = TW;
    seq.max_state = max_state;
    seq.TI = TI;
    seq.undersampling_factor = uf;
    seq.repetitions = reps;
    seq.inversion_prepulse = inversion != 0;
    seq.wait_spoiling = wait_spoil != 0;
    auto* c_rf = reinterpret_cast<cfloat*>(rf);
    auto* c_sl = reinterpret_cast<cfloat*>(slices);
    auto* c_out = reinterpret_cast<cfloat*>(out);
    if (max_state <= 32)
        fisp_voxels<32>(params, nv, vidx, nidx, c_rf, c_sl, nTR, P, seq, c_out, nthreads);
    else if (max_state <= 128)
        fisp_voxels<128>(params, nv, vidx, nidx, c_rf, c_sl, nTR, P, seq, c_out, nthreads);
    else
        return -1;
    return 0;
}

// signal entries (coil, readout, sample) = entries[3e..3e+2], each summed over all nv voxels
void ref_signal_cartesian_entries(float* echos, float* params, int64_t nv, int R, int S, float dt, float* k_start,
                                  float dk, float* coils, int C, const int* entries, int64_t nent, float* out,
                                  int nthreads) {
    compas::CartesianTrajectoryView traj;
    traj.nreadouts = R;
    traj.samples_per_readout = S;
    traj.delta_t = dt;
    traj.k_start = host_view(reinterpret_cast<cfloat*>(k_start), R);
    traj.delta_k = cfloat(dk, 0.0f);
    compas::TissueParametersView pv;
    pv.parameters = host_view(params, 9, nv);
    auto ev = host_view(reinterpret_cast<cfloat*>(echos), R, int(nv));
    auto cv = host_view(reinterpret_cast<cfloat*>(coils), C, int(nv));
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int64_t e = 0; e < nent; e++) {
        cfloat value;
        kmm::View<cfloat, 3> sview;  // every (c, r, s) of this [C][R][S] view is `value` (zero strides)
        const int c = entries[3 * e], r = entries[3 * e + 1], s = entries[3 * e + 2];
        sview.ptr = &value;
        sview.ext[0] = C;
        sview.ext[1] = R;
        sview.ext[2] = S;
        blockDim = {1, 1, 1};
        blockIdx = {unsigned(s), unsigned(r), unsigned(c)};
        threadIdx = {0, 0, 0};
        compas::kernels::sum_signal_cartesian_naive(kmm::Range<int> {0, int(nv)}, sview, ev, pv, traj, cv);
        out[2 * e] = value.re;
        out[2 * e + 1] = value.im;
    }
}

}  // extern "C"
