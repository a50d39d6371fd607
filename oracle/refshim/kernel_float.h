// Host stand-in for the kernel_float submodule (empty in the reference tree): the compas-toolkit
// kernels compiled by oracle/ref_sim.cpp, ref_kernels.cpp and the ref_gpu*.cu files name only its
// scalar cast. TEST INFRASTRUCTURE ONLY.
#pragma once

namespace kernel_float {
template<typename T, typename U>
#if defined(__CUDACC__)
__host__ __device__
#endif
T cast(U value) {
    return T(value);
}
}  // namespace kernel_float
