// Host stand-in for the one kmm geometry type the compas-toolkit kernel headers name.
// TEST INFRASTRUCTURE ONLY (oracle/ref_sim.cpp); kmm itself is an empty submodule in the
// reference tree and is not reproduced here.
#pragma once
#include <cstddef>

namespace kmm {
template<typename T>
struct Range {
    T begin = 0, end = 0;
    T size() const { return end - begin; }
    bool contains(T i) const { return i >= begin && i < end; }
};

// index box; the kernels read its axes as .x, .y, .z
template<size_t N, typename T = int>
struct Bounds {
    Range<T> x, y, z;
    bool contains(T i) const { return x.contains(i); }
    bool contains(T i, T j) const { return x.contains(i) && y.contains(j); }
    bool contains(T i, T j, T k) const { return x.contains(i) && y.contains(j) && z.contains(k); }
};
}  // namespace kmm
