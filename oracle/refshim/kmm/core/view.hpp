// Stand-in for the kmm view types that compas-toolkit's include/compas/core/view.h aliases.
// TEST INFRASTRUCTURE ONLY: enough to compile the reference's kernels for the host
// (oracle/ref_sim.cpp, oracle/ref_kernels.cpp) and, with nvcc, for the GPU (oracle/ref_gpu.cu):
// element access, row access, size, drop_axis, in_bounds. Not the kmm library. In device code
// every element or row index is checked against the view's extent; an index outside it sets
// kmm_ref_out_of_bounds and is replaced by 0, so no access leaves the buffer. Built with
// KMM_REF_UNCHECKED the check is left out (kmm's own views do not check either), for timing the
// reference's kernels only on launches that the checked build ran without a flagged index.
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <type_traits>

#include "kmm/utils/geometry.hpp"

#if defined(__CUDACC__)
#define KMM_REF_HD __host__ __device__
#else
#define KMM_REF_HD
#endif

#if defined(__CUDACC__)
static __device__ unsigned int kmm_ref_out_of_bounds = 0;
#endif

// kmm's optimisation hint; a no-op here
#ifndef KMM_ASSUME
#define KMM_ASSUME(expr) ((void)0)
#endif

namespace kmm {

KMM_REF_HD inline int64_t checked_index(int64_t i, int64_t extent) {
#if defined(__CUDA_ARCH__) && !defined(KMM_REF_UNCHECKED)
    if (i < 0 || i >= extent) {
        kmm_ref_out_of_bounds = 1;
        return 0;
    }
#endif
    (void)extent;
    return i;
}

// rank-N view over strided memory (strides in elements)
template<typename T, size_t N = 1>
struct View {
    T* ptr = nullptr;
    int64_t ext[N] = {};
    int64_t str[N] = {};

    KMM_REF_HD T* data() const { return ptr; }

    KMM_REF_HD int64_t size(size_t axis) const { return ext[axis]; }
    KMM_REF_HD int64_t size() const {
        int64_t n = 1;
        for (size_t i = 0; i < N; i++) n *= ext[i];
        return n;
    }

    // view without axis A at index i
    template<size_t A = 0, size_t M = N, std::enable_if_t<(M >= 2), int> = 0>
    KMM_REF_HD View<T, N - 1> drop_axis(int64_t i) const {
        View<T, N - 1> v;
        v.ptr = ptr + checked_index(i, ext[A]) * str[A];
        for (size_t a = 0, b = 0; a < N; a++) {
            if (a == A) continue;
            v.ext[b] = ext[a];
            v.str[b] = str[a];
            b++;
        }
        return v;
    }

    template<typename... I>
    KMM_REF_HD bool in_bounds(I... index) const {
        static_assert(sizeof...(I) == N);
        const int64_t i[] = {int64_t(index)...};
        for (size_t a = 0; a < N; a++)
            if (i[a] < 0 || i[a] >= ext[a]) return false;
        return true;
    }
    KMM_REF_HD bool in_bounds(const std::array<int64_t, N>& i) const {
        for (size_t a = 0; a < N; a++)
            if (i[a] < 0 || i[a] >= ext[a]) return false;
        return true;
    }

    KMM_REF_HD decltype(auto) operator[](int64_t i) const {
        if constexpr (N == 1) {
            return static_cast<T&>(ptr[checked_index(i, ext[0]) * str[0]]);
        } else {
            return drop_axis<0>(i);
        }
    }
};

template<typename T, size_t N = 1> using ViewMut = View<T, N>;
template<typename T, size_t N = 1> using ViewStrided = View<T, N>;
template<typename T, size_t N = 1> using ViewStridedMut = View<T, N>;
template<typename T, size_t N = 1> using Subview = View<T, N>;
template<typename T, size_t N = 1> using SubviewMut = View<T, N>;
template<typename T, size_t N = 1> using SubviewStrided = View<T, N>;
template<typename T, size_t N = 1> using SubviewStridedMut = View<T, N>;
template<typename T, size_t N = 1> using GPUView = View<T, N>;
template<typename T, size_t N = 1> using GPUViewMut = View<T, N>;
template<typename T, size_t N = 1> using GPUViewStrided = View<T, N>;
template<typename T, size_t N = 1> using GPUViewStridedMut = View<T, N>;
template<typename T, size_t N = 1> using GPUSubview = View<T, N>;
template<typename T, size_t N = 1> using GPUSubviewMut = View<T, N>;
template<typename T, size_t N = 1> using GPUSubviewStrided = View<T, N>;
template<typename T, size_t N = 1> using GPUSubviewStridedMut = View<T, N>;

// contiguous row-major view of a host buffer
template<typename T, typename... I>
View<T, sizeof...(I)> host_view(T* data, I... extents) {
    View<T, sizeof...(I)> v;
    v.ptr = data;
    const int64_t e[] = {int64_t(extents)...};
    int64_t s = 1;
    for (size_t a = sizeof...(I); a-- > 0;) {
        v.ext[a] = e[a];
        v.str[a] = s;
        s *= e[a];
    }
    return v;
}

}  // namespace kmm
