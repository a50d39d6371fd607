// Stand-in for the kmm geometry types the compas-toolkit kernel headers name.
// TEST INFRASTRUCTURE ONLY (oracle/ref_sim.cpp); kmm itself is an empty submodule in the
// reference tree and is not reproduced here.
#pragma once
#include <cstddef>

#if defined(__CUDACC__)
#define KMM_REF_HD __host__ __device__
#else
#define KMM_REF_HD
#endif

namespace kmm {
template<typename T>
struct Range {
    T begin = 0, end = 0;
    KMM_REF_HD T size() const { return end - begin; }
    KMM_REF_HD bool contains(T i) const { return i >= begin && i < end; }
};

// index box; the kernels read its axes as .x, .y, .z
template<size_t N, typename T = int>
struct Bounds {
    Range<T> x, y, z;
    KMM_REF_HD bool contains(T i) const { return x.contains(i); }
    KMM_REF_HD bool contains(T i, T j) const { return x.contains(i) && y.contains(j); }
    KMM_REF_HD bool contains(T i, T j, T k) const { return x.contains(i) && y.contains(j) && z.contains(k); }
};
}  // namespace kmm
