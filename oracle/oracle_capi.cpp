// oracle_capi.cpp — plain C entry points over compas_oracle.hpp.
//
// TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline). Built into
// oracle/liboracle.so; loaded by tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py. Never linked into the product.
//
// Suffix _f64 computes in double (truth); _f32 computes in float (the
// reference-arithmetic twin). Complex arrays are interleaved {re, im}; layouts
// follow the reference: echos [R][V], coils [C][V], signal [C][R][S],
// J·v input [4][V], Jᴴ·v input [C][R][S], Jᴴ·v output [4][V].
#include <omp.h>

#include <cstdint>

#include "compas_oracle.hpp"

using namespace oracle;

namespace {

template<typename T, typename Out>
void store(Out* out, int64_t i, cx<T> v) {
    out[2 * i] = Out(v.re);
    out[2 * i + 1] = Out(v.im);
}

template<typename T, typename Out>
int fisp_impl(const float* params, int64_t nv, const int* vidx, int64_t nidx, const float* rf,
              const float* slices, int nTR, int P, float TR, float TE, float TW, float TI, int max_state,
              int uf, int reps, int inversion, int wait_spoil, Out* echo, int nthreads) {
    if (max_state < 1 || uf < 1 || reps < 1 || nTR < 1 || P < 1) return -1;
    FispSequence s {rf, slices, nTR, P, TR, TE, TW, TI, max_state, uf, reps, inversion, wait_spoil};
    int64_t n = vidx ? nidx : nv;
    int64_t R = int64_t(nTR) * uf;
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<cx<T>> buf(R);
#pragma omp for schedule(dynamic, 4)
        for (int64_t i = 0; i < n; i++) {
            int64_t v = vidx ? vidx[i] : i;
            fisp_voxel<T>(load_voxel<T>(params, nv, v), s, buf.data(), 1);
            for (int64_t r = 0; r < R; r++) store<T>(echo, r * n + i, buf[r]);
        }
    }
    return 0;
}

template<typename T, typename Out>
int pssfp_impl(const float* params, int64_t nv, const int* vidx, int64_t nidx, const float* rf, int nTR,
               const float* gdtrf, int nRF, float dt_ex, float dt_inv, float dt_pr, float gz_ex, float gz_inv,
               float gz_pr, const float* z, int nz, Out* echo, int nthreads) {
    if (nTR < 1 || nRF < 0 || nz < 1) return -1;
    PssfpSequence s {rf, nTR, gdtrf, nRF, dt_ex, dt_inv, dt_pr, gz_ex, gz_inv, gz_pr, z, nz};
    int64_t n = vidx ? nidx : nv;
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<cx<T>> buf(nTR);
#pragma omp for schedule(dynamic, 4)
        for (int64_t i = 0; i < n; i++) {
            int64_t v = vidx ? vidx[i] : i;
            pssfp_voxel<T>(load_voxel<T>(params, nv, v), s, buf.data(), 1);
            for (int64_t r = 0; r < nTR; r++) store<T>(echo, r * n + i, buf[r]);
        }
    }
    return 0;
}

// entries: (c, r, k) int triples; when null all C*R*S entries in [C][R][S] order.
template<typename T, typename Out, typename F>
void for_entries(int nc, int nr, int ns, const int* entries, int64_t nent, Out* out, int nthreads, F fn) {
    int64_t n = entries ? nent : int64_t(nc) * nr * ns;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 8)
    for (int64_t i = 0; i < n; i++) {
        int c, r, k;
        if (entries) {
            c = entries[3 * i];
            r = entries[3 * i + 1];
            k = entries[3 * i + 2];
        } else {
            c = int(i / (int64_t(nr) * ns));
            r = int((i / ns) % nr);
            k = int(i % ns);
        }
        store<T>(out, i, fn(c, r, k));
    }
}

}  // namespace

extern "C" {

int oracle_fisp_f64(const float* params, int64_t nv, const int* vidx, int64_t nidx, const float* rf,
                    const float* slices, int nTR, int P, float TR, float TE, float TW, float TI, int max_state,
                    int uf, int reps, int inversion, int wait_spoil, double* echo, int nthreads) {
    return fisp_impl<double>(params, nv, vidx, nidx, rf, slices, nTR, P, TR, TE, TW, TI, max_state, uf, reps,
                             inversion, wait_spoil, echo, nthreads);
}

int oracle_fisp_f32(const float* params, int64_t nv, const int* vidx, int64_t nidx, const float* rf,
                    const float* slices, int nTR, int P, float TR, float TE, float TW, float TI, int max_state,
                    int uf, int reps, int inversion, int wait_spoil, float* echo, int nthreads) {
    return fisp_impl<float>(params, nv, vidx, nidx, rf, slices, nTR, P, TR, TE, TW, TI, max_state, uf, reps,
                            inversion, wait_spoil, echo, nthreads);
}

int oracle_pssfp_f64(const float* params, int64_t nv, const int* vidx, int64_t nidx, const float* rf, int nTR,
                     const float* gdtrf, int nRF, float dt_ex, float dt_inv, float dt_pr, float gz_ex,
                     float gz_inv, float gz_pr, const float* z, int nz, double* echo, int nthreads) {
    return pssfp_impl<double>(params, nv, vidx, nidx, rf, nTR, gdtrf, nRF, dt_ex, dt_inv, dt_pr, gz_ex, gz_inv,
                              gz_pr, z, nz, echo, nthreads);
}

int oracle_pssfp_f32(const float* params, int64_t nv, const int* vidx, int64_t nidx, const float* rf, int nTR,
                     const float* gdtrf, int nRF, float dt_ex, float dt_inv, float dt_pr, float gz_ex,
                     float gz_inv, float gz_pr, const float* z, int nz, float* echo, int nthreads) {
    return pssfp_impl<float>(params, nv, vidx, nidx, rf, nTR, gdtrf, nRF, dt_ex, dt_inv, dt_pr, gz_ex, gz_inv,
                             gz_pr, z, nz, echo, nthreads);
}

int oracle_phase_encoding_f64(const float* echo, const float* params, int64_t nv, int nr, const float* k_start,
                              double* out) {
    for (int r = 0; r < nr; r++)
        for (int64_t v = 0; v < nv; v++) {
            Voxel<double> p = load_voxel<double>(params, nv, v);
            cx<double> m = {echo[2 * (r * nv + v)], echo[2 * (r * nv + v) + 1]};
            store<double>(out, r * nv + v, phase_encode(m, p, cx<double>{k_start[2 * r], k_start[2 * r + 1]}));
        }
    return 0;
}

int oracle_signal_cartesian_f64(const float* echo, const float* params, int64_t nv, int nr, int ns, float dt,
                                const float* k_start, float dk_re, float dk_im, const float* coils, int nc,
                                const int* entries, int64_t nent, double* out, int nthreads) {
    Cartesian t {nr, ns, dt, k_start, dk_re, dk_im};
    for_entries<double>(nc, nr, ns, entries, nent, out, nthreads, [&](int c, int r, int k) {
        return signal_cartesian_entry<double>(echo, params, nv, t, coils, c, r, k);
    });
    return 0;
}

int oracle_signal_cartesian_f32(const float* echo, const float* params, int64_t nv, int nr, int ns, float dt,
                                const float* k_start, float dk_re, float dk_im, const float* coils, int nc,
                                const int* entries, int64_t nent, float* out, int nthreads) {
    Cartesian t {nr, ns, dt, k_start, dk_re, dk_im};
    for_entries<float>(nc, nr, ns, entries, nent, out, nthreads, [&](int c, int r, int k) {
        return signal_cartesian_entry<float>(echo, params, nv, t, coils, c, r, k);
    });
    return 0;
}

int oracle_signal_spiral_f64(const float* echo, const float* params, int64_t nv, int nr, int ns, float dt,
                             const float* k_start, const float* dk, const float* coils, int nc,
                             const int* entries, int64_t nent, double* out, int nthreads) {
    Spiral t {nr, ns, dt, k_start, dk};
    for_entries<double>(nc, nr, ns, entries, nent, out, nthreads, [&](int c, int r, int k) {
        return signal_spiral_entry<double>(echo, params, nv, t, coils, c, r, k);
    });
    return 0;
}

int oracle_jacobian_f64(const float* echo, const float* dT1, const float* dT2, const float* params, int64_t nv,
                        int nr, int ns, float dt, float dk_re, float dk_im, const float* coils, int nc,
                        const float* vec, const int* entries, int64_t nent, double* out, int nthreads) {
    Cartesian t {nr, ns, dt, nullptr, dk_re, dk_im};
    for_entries<double>(nc, nr, ns, entries, nent, out, nthreads, [&](int c, int r, int k) {
        return jacobian_entry<double>(echo, dT1, dT2, params, nv, t, coils, vec, c, r, k);
    });
    return 0;
}

// out: [4][n] where n = nidx (voxel list) or nv.
int oracle_jacobian_hermitian_f64(const float* echo, const float* dT1, const float* dT2, const float* params,
                                  int64_t nv, int nr, int ns, float dt, float dk_re, float dk_im,
                                  const float* coils, int nc, const float* vec, const int* vidx, int64_t nidx,
                                  double* out, int nthreads) {
    Cartesian t {nr, ns, dt, nullptr, dk_re, dk_im};
    int64_t n = vidx ? nidx : nv;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
    for (int64_t i = 0; i < n; i++) {
        int64_t v = vidx ? vidx[i] : i;
        cx<double> res[4];
        jacobian_hermitian_voxel<double>(echo, dT1, dT2, params, nv, t, coils, nc, vec, v, res);
        for (int f = 0; f < 4; f++) store<double>(out, f * n + i, res[f]);
    }
    return 0;
}

int oracle_spiral_jacobian_f64(const float* echo, const float* dT1, const float* dT2, const float* params,
                               int64_t nv, int nr, int ns, float dt, const float* k_start, const float* dk,
                               const float* coils, int nc, const float* vec, const int* entries, int64_t nent,
                               double* out, int nthreads) {
    Spiral t {nr, ns, dt, k_start, dk};
    for_entries<double>(nc, nr, ns, entries, nent, out, nthreads, [&](int c, int r, int k) {
        return spiral_jacobian_entry<double>(echo, dT1, dT2, params, nv, t, coils, vec, c, r, k);
    });
    return 0;
}

int oracle_spiral_jacobian_hermitian_f64(const float* echo, const float* dT1, const float* dT2, const float* params,
                                         int64_t nv, int nr, int ns, float dt, const float* k_start,
                                         const float* dk, const float* coils, int nc, const float* vec,
                                         const int* vidx, int64_t nidx, double* out, int nthreads) {
    Spiral t {nr, ns, dt, k_start, dk};
    int64_t n = vidx ? nidx : nv;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
    for (int64_t i = 0; i < n; i++) {
        int64_t v = vidx ? vidx[i] : i;
        cx<double> res[4];
        spiral_jacobian_hermitian_voxel<double>(echo, dT1, dT2, params, nv, t, coils, nc, vec, v, res);
        for (int f = 0; f < 4; f++) store<double>(out, f * n + i, res[f]);
    }
    return 0;
}

// residual d = lhs - rhs, returns Σ|d|²   (src/utils/residual_kernels.cuh:26-64)
double oracle_residual_f64(const float* lhs, const float* rhs, int64_t n, double* out) {
    double acc = 0;
    for (int64_t i = 0; i < n; i++) {
        double dr = double(lhs[2 * i]) - rhs[2 * i], di = double(lhs[2 * i + 1]) - rhs[2 * i + 1];
        if (out) {
            out[2 * i] = dr;
            out[2 * i + 1] = di;
        }
        acc += dr * dr + di * di;
    }
    return acc;
}

int oracle_max_threads() {
    return omp_get_max_threads();
}

// Evaluate the FP32 twin's complex primitives on packed inputs (used to pin them
// against the reference's own complex_type.h, see ref_golden.cpp).
//   op 0: exp(z)          in: re, im                 out: re, im
//   op 1: pow(a, b)       in: a.re, a.im, b          out: re, im
//   op 2: c + a*b (fma)   in: a, b, c (6 floats)     out: re, im
//   op 3: a * b           in: a, b (4 floats)        out: re, im
int oracle_cx_eval_f32(int op, const float* in, int64_t n, float* out) {
    for (int64_t i = 0; i < n; i++) {
        cx<float> r;
        if (op == 0) {
            r = cexp(cx<float>{in[2 * i], in[2 * i + 1]});
        } else if (op == 1) {
            r = cpow(cx<float>{in[3 * i], in[3 * i + 1]}, in[3 * i + 2]);
        } else if (op == 2) {
            const float* q = in + 6 * i;
            r = add_mul(cx<float>{q[4], q[5]}, cx<float>{q[0], q[1]}, cx<float>{q[2], q[3]});
        } else if (op == 3) {
            const float* q = in + 4 * i;
            r = cx<float>{q[0], q[1]} * cx<float>{q[2], q[3]};
        } else {
            return -1;
        }
        out[2 * i] = r.re;
        out[2 * i + 1] = r.im;
    }
    return 0;
}

}  // extern "C"
