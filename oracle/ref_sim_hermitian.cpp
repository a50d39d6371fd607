// ref_sim_hermitian.cpp — the reference's naive Jᴴ·v kernel run on the CPU for oracle/ref_sim.cpp.
//
// TEST INFRASTRUCTURE ONLY. A translation unit of its own, as in the reference, because
// src/jacobian/hermitian_kernels.cuh and src/jacobian/product_kernels.cuh both define
// kernels::compute_sample_decay. jacobian_hermitian_product_naive
// (src/jacobian/hermitian_kernels.cuh:30-92) runs as one one-thread launch per voxel.
#include "jacobian/hermitian_kernels.cuh"

using compas::cfloat;
using kmm::host_view;

void run_jacobian_hermitian_naive(int nv, int R, int S, int C, cfloat* jhv, cfloat* echos, cfloat* d1, cfloat* d2,
                                  float* params, const compas::CartesianTrajectoryView& traj, cfloat* coils,
                                  cfloat* u) {
    compas::TissueParametersView pv;
    pv.parameters = host_view(params, 9, nv);
    for (int v = 0; v < nv; v++) {
        blockDim = {1, 1, 1};
        gridDim = {unsigned(nv), 1, 1};
        blockIdx = {unsigned(v), 0, 0};
        threadIdx = {0, 0, 0};
        compas::kernels::jacobian_hermitian_product_naive(
            kmm::Range<int> {0, nv}, R, S, C, host_view(jhv, 4, nv), host_view(echos, R, nv), host_view(d1, R, nv),
            host_view(d2, R, nv), pv, traj, host_view(coils, C, nv), host_view(u, C, R, S));
    }
}
