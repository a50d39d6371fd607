// vector.h — the fixed-size vector value type of the C++ API: compas::vector<T, N> and its aliases
// (vec2 / vfloat2 / vdouble2, vec3 / vfloat3 / vdouble3, vec4 / vfloat4 / vdouble4, ndint<N>),
// usable in host and device code.
//
// Source-level counterpart of the reference's include/compas/core/vector.h:141-227 (the type and its
// members: value / element-list / storage construction, at, operator[], size, begin/end, cbegin/cend,
// map) and :298-386 (norm, dot, cross, the elementwise + - * / with vectors and scalars and their
// assignment forms, == and !=, the aliases). Vectors of 1 to 4 elements name their elements x, y, z,
// w; 2- and 4-element vectors are aligned to their whole size (a vfloat2 is 8 bytes, 8-aligned, a
// vfloat4 16), a vfloat3 is three packed floats.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define COMPAS_VECTOR_HD __host__ __device__
#else
#define COMPAS_VECTOR_HD
#endif

namespace compas {

namespace detail {

COMPAS_VECTOR_HD inline float vector_sqrt(float x) {
    return sqrtf(x);
}
COMPAS_VECTOR_HD inline double vector_sqrt(double x) {
    return sqrt(x);
}

template<typename T, int N>
struct vector_elements {
    T values[N];
    COMPAS_VECTOR_HD T* data() { return values; }
    COMPAS_VECTOR_HD const T* data() const { return values; }
};

template<typename T>
struct vector_elements<T, 0> {
    COMPAS_VECTOR_HD T* data() { return nullptr; }
    COMPAS_VECTOR_HD const T* data() const { return nullptr; }
};

template<typename T>
struct vector_elements<T, 1> {
    T x;
    COMPAS_VECTOR_HD T* data() { return &x; }
    COMPAS_VECTOR_HD const T* data() const { return &x; }
};

template<typename T>
struct alignas(2 * alignof(T)) vector_elements<T, 2> {
    T x, y;
    COMPAS_VECTOR_HD T* data() { return &x; }
    COMPAS_VECTOR_HD const T* data() const { return &x; }
};

template<typename T>
struct vector_elements<T, 3> {
    T x, y, z;
    COMPAS_VECTOR_HD T* data() { return &x; }
    COMPAS_VECTOR_HD const T* data() const { return &x; }
};

template<typename T>
struct alignas(4 * alignof(T)) vector_elements<T, 4> {
    T x, y, z, w;
    COMPAS_VECTOR_HD T* data() { return &x; }
    COMPAS_VECTOR_HD const T* data() const { return &x; }
};

}  // namespace detail

template<typename T, int N>
struct vector: detail::vector_elements<T, N> {
    using storage_type = detail::vector_elements<T, N>;

    // every element set to `value`
    COMPAS_VECTOR_HD vector(const T& value = {}) {
        for (int i = 0; i < N; i++) this->data()[i] = value;
    }

    COMPAS_VECTOR_HD vector(const storage_type& storage) : storage_type(storage) {}

    // exactly N elements, in order
    template<typename... Ts>
    COMPAS_VECTOR_HD vector(const T& first, const T& second, const Ts&... rest) {
        static_assert(2 + sizeof...(Ts) == N, "a vector<T, N> is built from exactly N elements");
        const T list[] = {first, second, T(rest)...};
        for (int i = 0; i < N; i++) this->data()[i] = list[i];
    }

    COMPAS_VECTOR_HD T& at(int i) { return this->data()[i]; }
    COMPAS_VECTOR_HD const T& at(int i) const { return this->data()[i]; }
    COMPAS_VECTOR_HD T& operator[](int i) { return at(i); }
    COMPAS_VECTOR_HD const T& operator[](int i) const { return at(i); }
    COMPAS_VECTOR_HD int size() const { return N; }

    COMPAS_VECTOR_HD T* begin() { return this->data(); }
    COMPAS_VECTOR_HD T* end() { return this->data() + N; }
    COMPAS_VECTOR_HD const T* begin() const { return this->data(); }
    COMPAS_VECTOR_HD const T* end() const { return this->data() + N; }
    COMPAS_VECTOR_HD const T* cbegin() const { return this->data(); }
    COMPAS_VECTOR_HD const T* cend() const { return this->data() + N; }

    // elementwise fun(x) as a vector of fun's result type
    template<typename F>
    COMPAS_VECTOR_HD auto map(F fun) const -> vector<decltype(fun(T {})), N> {
        vector<decltype(fun(T {})), N> out;
        for (int i = 0; i < N; i++) out[i] = fun(at(i));
        return out;
    }
};

template<typename T, int N>
COMPAS_VECTOR_HD T dot(const vector<T, N>& a, const vector<T, N>& b) {
    T s = T {};
    for (int i = 0; i < N; i++) s += a[i] * b[i];
    return s;
}

// Euclidean length. Scaled by the largest magnitude, so that squares neither overflow nor underflow.
template<typename T, int N>
COMPAS_VECTOR_HD T norm(const vector<T, N>& a) {
    T m = T {};
    for (int i = 0; i < N; i++) {
        const T v = a[i] < T {} ? -a[i] : a[i];
        if (!(v == v)) return v;  // NaN in, NaN out
        m = v > m ? v : m;
    }
    if (!(m > T {})) return m;
    T s = T {};
    for (int i = 0; i < N; i++) {
        const T q = a[i] / m;
        s += q * q;
    }
    return m * detail::vector_sqrt(s);
}

template<typename T>
COMPAS_VECTOR_HD vector<T, 3> cross(const vector<T, 3>& a, const vector<T, 3>& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

#define COMPAS_VECTOR_ELEMENTWISE(OP, OP_ASSIGN)                                                   \
    template<typename T, int N>                                                                    \
    COMPAS_VECTOR_HD vector<T, N> operator OP(const vector<T, N>& a, const vector<T, N>& b) {      \
        vector<T, N> r;                                                                            \
        for (int i = 0; i < N; i++) r[i] = a[i] OP b[i];                                           \
        return r;                                                                                  \
    }                                                                                              \
    template<typename T, int N>                                                                    \
    COMPAS_VECTOR_HD vector<T, N> operator OP(const vector<T, N>& a, const T& b) {                 \
        return a OP vector<T, N>(b);                                                               \
    }                                                                                              \
    template<typename T, int N>                                                                    \
    COMPAS_VECTOR_HD vector<T, N> operator OP(const T& a, const vector<T, N>& b) {                 \
        return vector<T, N>(a) OP b;                                                               \
    }                                                                                              \
    template<typename T, int N>                                                                    \
    COMPAS_VECTOR_HD vector<T, N>& operator OP_ASSIGN(vector<T, N>& a, const vector<T, N>& b) {    \
        a = a OP b;                                                                                \
        return a;                                                                                  \
    }                                                                                              \
    template<typename T, int N>                                                                    \
    COMPAS_VECTOR_HD vector<T, N>& operator OP_ASSIGN(vector<T, N>& a, const T& b) {               \
        a = a OP b;                                                                                \
        return a;                                                                                  \
    }

COMPAS_VECTOR_ELEMENTWISE(+, +=)
COMPAS_VECTOR_ELEMENTWISE(-, -=)
COMPAS_VECTOR_ELEMENTWISE(*, *=)
COMPAS_VECTOR_ELEMENTWISE(/, /=)
#undef COMPAS_VECTOR_ELEMENTWISE

// equal when the sizes match and every element compares equal
template<typename T, int N, typename R, int M>
COMPAS_VECTOR_HD bool operator==(const vector<T, N>& a, const vector<R, M>& b) {
    if (N != M) return false;
    for (int i = 0; i < N && i < M; i++)
        if (!(a[i] == b[i])) return false;
    return true;
}

template<typename T, int N, typename R, int M>
COMPAS_VECTOR_HD bool operator!=(const vector<T, N>& a, const vector<R, M>& b) {
    return !(a == b);
}

template<typename T, int N>
using vec = vector<T, N>;
template<typename T>
using vec2 = vector<T, 2>;
template<typename T>
using vec3 = vector<T, 3>;
template<typename T>
using vec4 = vector<T, 4>;
using vfloat2 = vec2<float>;
using vdouble2 = vec2<double>;
using vfloat3 = vec3<float>;
using vdouble3 = vec3<double>;
using vfloat4 = vec4<float>;
using vdouble4 = vec4<double>;
template<int N>
using ndint = vector<int, N>;

}  // namespace compas
