// Host stand-in for the kernel_float submodule (empty in the reference tree): the compas-toolkit
// kernels compiled by oracle/ref_sim.cpp name only its scalar cast. TEST INFRASTRUCTURE ONLY.
#pragma once

namespace kernel_float {
template<typename T, typename U>
T cast(U value) {
    return T(value);
}
}  // namespace kernel_float
