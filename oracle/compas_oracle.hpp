// compas_oracle.hpp — CPU oracle for the compas-toolkit simulation hot path.
//
// TEST INFRASTRUCTURE ONLY. This header is the checker: the parity tests, the
// smoke check and the CPU-baseline leg of the benchmark may use it. The product
// library (libcompas_b200.so) never includes, links or calls anything here.
//
// It restates, in plain C++ templated on the scalar type T, the arithmetic of
// the reference implementation (NLeSC-COMPAS/compas-toolkit). T = double is the
// "truth" used for every error figure; T = float is the "reference-arithmetic
// twin" that follows the reference's formulas and operation order in FP32.
//
// Each function cites the reference file:line it restates. Parity status: the
// reference ships no golden vectors and cannot be built as shipped (its `kmm`
// runtime submodule is absent, there is no Julia). The oracle is pinned by
// (a) golden vectors from the reference's own code built for the host: the
// complex primitives of `compas/core/complex_type.h` (oracle/ref_golden.cpp)
// and its FISP / pSSFP simulation, phase-encoding, signal (Cartesian naive,
// spiral), Jacobian (naive J·v, Jᴴ·v) and residual kernels run one thread at a
// time (oracle/ref_sim.cpp), which the FP64 functions here match to FP32
// rounding; (b) analytic known-answer tests and (c) structural identities
// (adjointness of J and Jᴴ, finite differences, undersampling replication).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle {

template<typename T>
struct cx {
    T re = 0, im = 0;
    cx() = default;
    cx(T r, T i = T(0)) : re(r), im(i) {}
};

template<typename T> inline cx<T> operator+(cx<T> a, cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template<typename T> inline cx<T> operator-(cx<T> a, cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template<typename T> inline cx<T> operator*(cx<T> a, cx<T> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template<typename T> inline cx<T> operator*(T s, cx<T> a) { return {s * a.re, s * a.im}; }
template<typename T> inline cx<T> operator*(cx<T> a, T s) { return {s * a.re, s * a.im}; }
template<typename T> inline cx<T>& operator+=(cx<T>& a, cx<T> b) { a = a + b; return a; }
template<typename T> inline cx<T> conj(cx<T> a) { return {a.re, -a.im}; }
template<typename T> inline T norm2(cx<T> a) { return a.re * a.re + a.im * a.im; }

// `c + a*b` with the two-level fused form used by the reference's complex fma
// (compas/core/complex_type.h:174-178).
template<typename T> inline cx<T> add_mul(cx<T> c, cx<T> a, cx<T> b) {
    return {std::fma(a.re, b.re, std::fma(-a.im, b.im, c.re)),
            std::fma(a.re, b.im, std::fma(a.im, b.re, c.im))};
}

template<typename T> inline cx<T> polar1(T angle) { return {std::cos(angle), std::sin(angle)}; }

// exp(z) = e^{re} (cos im, sin im)   (complex_type.h:106-119)
template<typename T> inline cx<T> cexp(cx<T> z) {
    T e = std::exp(z.re);
    return {e * std::cos(z.im), e * std::sin(z.im)};
}

// pow(a, b) = exp(b * log(a)), log(a) = (log|a|, arg a)   (complex_type.h:141-161)
template<typename T> inline cx<T> cpow(cx<T> a, T b) {
    cx<T> l = {std::log(std::hypot(a.re, a.im)), std::atan2(a.im, a.re)};
    return cexp(cx<T>{b * l.re, b * l.im});
}

template<typename T> inline T two_pi() { return T(2.0 * M_PI); }

// Tissue parameters: SoA float[9][nv] in the device order T1,T2,B1,B0,rho_x,rho_y,x,y,z
// (compas/parameters/tissue_view.cuh:53-71).
enum { F_T1 = 0, F_T2, F_B1, F_B0, F_RHOX, F_RHOY, F_X, F_Y, F_Z, F_NUM };

template<typename T>
struct Voxel {
    T T1, T2, B1, B0, x, y, z;
    cx<T> rho;
};

template<typename T>
inline Voxel<T> load_voxel(const float* params, int64_t nv, int64_t v) {
    Voxel<T> p;
    p.T1 = T(params[F_T1 * nv + v]);
    p.T2 = T(params[F_T2 * nv + v]);
    p.B1 = T(params[F_B1 * nv + v]);
    p.B0 = T(params[F_B0 * nv + v]);
    p.rho = {T(params[F_RHOX * nv + v]), T(params[F_RHOY * nv + v])};
    p.x = T(params[F_X * nv + v]);
    p.y = T(params[F_Y * nv + v]);
    p.z = T(params[F_Z * nv + v]);
    return p;
}

// --------------------------------------------------------------------------------------------
// FISP / EPG   (src/operators/epg.cuh:13-322, src/simulate/fisp_kernels.cuh:99-223,
//               src/simulate/fisp.cu:7-43,386-399)
// --------------------------------------------------------------------------------------------

template<typename T>
struct ExciteMatrix {
    T R11;
    cx<T> R12, R13;
    T R33;

    // EPGExciteMatrix(RF, B1)   (epg.cuh:37-90)
    ExciteMatrix(cx<T> RF, T B1) {
        const T deg2rad = T(M_PI) / T(180);
        T abs_rf = std::hypot(RF.re, RF.im);
        T alpha = deg2rad * abs_rf * B1;
        T x = alpha * T(0.5);
        T sinx = std::sin(x), cosx = std::cos(x);
        T sinx_sq = sinx * sinx, cosx_sq = cosx * cosx;
        T sinalpha = T(2) * sinx * cosx;
        T cosalpha = T(2) * cosx_sq - T(1);
        T cosphi = 1, sinphi = 0;
        if (abs_rf > T(1.17549435e-38)) {
            cosphi = RF.re / abs_rf;
            sinphi = RF.im / abs_rf;
        }
        T sin2phi = (T(2) * cosphi) * sinphi;
        T cos2phi = (T(2) * cosphi) * cosphi - T(1);
        R11 = cosx_sq;
        R12 = {cos2phi * sinx_sq, sin2phi * sinx_sq};
        R13 = {sinphi * sinalpha, -cosphi * sinalpha};
        R33 = cosalpha;
    }

    // apply()   (epg.cuh:92-111)
    void apply(cx<T>& Fp, cx<T>& Fm, cx<T>& Z) const {
        cx<T> R21 = conj(R12), R23 = conj(R13);
        T R22 = R11;
        cx<T> R31 = {T(-0.5) * R13.re, T(0.5) * R13.im};
        cx<T> R32 = conj(R31);
        cx<T> fp = add_mul(add_mul(R11 * Fp, R12, Fm), R13, Z);
        cx<T> fm = add_mul(add_mul(R22 * Fm, R21, Fp), R23, Z);
        cx<T> z = add_mul(add_mul(R31 * Fp, R32, Fm), cx<T>(R33), Z);
        Fp = fp;
        Fm = fm;
        Z = z;
    }
};

template<typename T>
struct EPGState {
    int N;
    std::vector<cx<T>> Fp, Fm, Z;

    explicit EPGState(int n) : N(n), Fp(n), Fm(n), Z(n) { Z[0] = {T(1), T(0)}; }

    void invert() { for (auto& z : Z) z = T(-1) * z; }                         // epg.cuh:146-152
    void spoil() { for (int i = 0; i < N; i++) Fp[i] = Fm[i] = cx<T>(); }       // epg.cuh:154-161
    void decay(T E1, T E2) {                                                    // epg.cuh:163-171
        for (int i = 0; i < N; i++) { Fp[i] = E2 * Fp[i]; Fm[i] = E2 * Fm[i]; Z[i] = E1 * Z[i]; }
    }
    void rotate_decay(T E1, T E2, cx<T> r) {                                    // epg.cuh:182-190
        cx<T> a = E2 * r;
        for (int i = 0; i < N; i++) { Fp[i] = Fp[i] * a; Fm[i] = Fm[i] * conj(a); Z[i] = E1 * Z[i]; }
    }
    void regrowth(T E1) { Z[0].re += T(1) - E1; }                               // epg.cuh:192-200
    void excite(const ExciteMatrix<T>& m) { for (int i = 0; i < N; i++) m.apply(Fp[i], Fm[i], Z[i]); }
    // dephasing = shift_down then shift_up   (epg.cuh:229-298)
    void dephasing() {
        for (int i = 0; i + 1 < N; i++) Fm[i] = Fm[i + 1];
        Fm[N - 1] = cx<T>();
        for (int i = N - 1; i > 0; i--) Fp[i] = Fp[i - 1];
        Fp[0] = conj(Fm[0]);
    }
};

struct FispSequence {
    const float* rf;       // complex [nTR]
    const float* slices;   // complex [P][nTR]
    int nTR, P;
    float TR, TE, TW, TI;
    int max_state, uf, reps;
    int inversion, wait_spoil;
};

// One voxel of `simulate_magnetization(ctx, params, FISPSequence)`; writes the
// undersampling-expanded echo (nTR*uf complex values) with stride `stride`.
template<typename T>
void fisp_voxel(const Voxel<T>& p, const FispSequence& s, cx<T>* echo, int64_t stride) {
    auto E = [](T dt, T TT) { return std::exp(-dt * (T(1) / TT)); };         // fisp_kernels.cuh:119-121
    auto rot = [](T dt, T B0) -> cx<T> {                                        // fisp_kernels.cuh:110-117
        if (B0 == T(0)) return {T(1), T(0)};
        return polar1(two_pi<T>() * dt * B0);
    };
    T TR = s.TR, TE = s.TE, TI = s.TI, TW = s.TW;
    T E1_TE = E(TE, p.T1), E2_TE = E(TE, p.T2);
    T E1_TI = E(TI, p.T1), E2_TI = E(TI, p.T2);
    T E1_TRTE = E(TR - TE, p.T1), E2_TRTE = E(TR - TE, p.T2);
    T E1_W = E(TW, p.T1), E2_W = E(TW, p.T2);
    cx<T> r_TE = rot(TE, p.B0), r_TRTE = rot(TR - TE, p.B0), r_TW = rot(TW, p.B0);

    std::vector<cx<T>> acc(s.nTR);
    for (int pos = 0; pos < s.P; pos++) {
        EPGState<T> st(s.max_state);
        for (int rep = s.reps; rep >= 1; rep--) {
            bool sampled = (rep == 1);
            if (s.inversion) {                                                 // fisp_kernels.cuh:146-152
                st.invert();
                st.spoil();
                st.decay(E1_TI, E2_TI);
                st.regrowth(E1_TI);
            }
            for (int t = 0; t < s.nTR; t++) {                                  // fisp_kernels.cuh:53-82
                cx<T> sp = {T(s.slices[2 * (int64_t(pos) * s.nTR + t)]), T(s.slices[2 * (int64_t(pos) * s.nTR + t) + 1])};
                cx<T> rf = {T(s.rf[2 * t]), T(s.rf[2 * t + 1])};
                st.excite(ExciteMatrix<T>(sp * rf, p.B1));
                st.rotate_decay(E1_TE, E2_TE, r_TE);
                st.regrowth(E1_TE);
                if (sampled) acc[t] += st.Fp[0];
                st.rotate_decay(E1_TRTE, E2_TRTE, r_TRTE);
                st.regrowth(E1_TRTE);
                st.dephasing();
            }
            if (s.wait_spoil) st.spoil();                                      // fisp_kernels.cuh:195-200
            st.rotate_decay(E1_W, E2_W, r_TW);
            st.regrowth(E1_W);
        }
    }
    // expand_undersampled_echos (fisp_kernels.cuh:246-259): echo[r] = sample[r / uf]
    for (int r = 0; r < s.nTR * s.uf; r++) echo[int64_t(r) * stride] = acc[r / s.uf];
}

// --------------------------------------------------------------------------------------------
// pSSFP / isochromat   (src/operators/isochromat.cuh:9-128, src/simulate/pssfp_kernels.cuh:14-108)
// --------------------------------------------------------------------------------------------

template<typename T>
struct Iso {
    T x = 0, y = 0, z = 1;

    // rotate(γΔtRF, γΔtGR, r, dt, p)   (isochromat.cuh:14-73)
    Iso rotate(cx<T> gdtrf, T gdtgr, T r, T dt, const Voxel<T>& p) const {
        T ax = gdtrf.re * p.B1, ay = -gdtrf.im * p.B1;
        T az = -(gdtgr * r) - dt * two_pi<T>() * p.B0;
        T th2 = ax * ax + ay * ay + az * az;
        T th = std::sqrt(th2);
        Iso m = *this;
        if (std::fabs(th) > T(1e-9)) {
            T kx = ax / th, ky = ay / th, kz = az / th;
            T s = std::sin(th), c = std::cos(th);
            T cxp = ky * z - kz * y, cyp = kz * x - kx * z, czp = kx * y - ky * x;
            T d = kx * x + ky * y + kz * z;
            m.x = c * x + s * cxp + d * (T(1) - c) * kx;
            m.y = c * y + s * cyp + d * (T(1) - c) * ky;
            m.z = c * z + s * czp + d * (T(1) - c) * kz;
        }
        return m;
    }
    // rotate(γΔtGR, r, dt, p): precession about z   (isochromat.cuh:75-97)
    Iso precess(T gdtgr, T r, T dt, const Voxel<T>& p) const {
        T th = -(gdtgr * r) - dt * two_pi<T>() * p.B0;
        T s = std::sin(th), c = std::cos(th);
        Iso m;
        m.x = c * x - s * y;
        m.y = c * y + s * x;
        m.z = z;
        return m;
    }
    Iso decay(T E1, T E2) const { Iso m = *this; m.x *= E2; m.y *= E2; m.z *= E1; return m; }
    Iso regrowth(T E1) const { Iso m = *this; m.z += T(1) - E1; return m; }
    Iso invert(const Voxel<T>& p) const { Iso m = *this; m.z *= std::cos(T(M_PI) * p.B1); return m; }
};

struct PssfpSequence {
    const float* rf;       // complex [nTR]
    int nTR;
    const float* gdtrf;    // complex [nRF]
    int nRF;
    float dt_ex, dt_inv, dt_pr;
    float gz_ex, gz_inv, gz_pr;
    const float* z;        // [nz]
    int nz;
};

template<typename T>
void pssfp_voxel(const Voxel<T>& p, const PssfpSequence& s, cx<T>* echo, int64_t stride) {
    auto E = [](T dt, T TT) { return std::exp(-dt * (T(1) / TT)); };
    T E1_ex = E(s.dt_ex, p.T1), E2_ex = E(s.dt_ex, p.T2);
    T E1_pr = E(s.dt_pr, p.T1), E2_pr = E(s.dt_pr, p.T2);
    T E1_inv = E(s.dt_inv, p.T1), E2_inv = E(s.dt_inv, p.T2);
    std::vector<cx<T>> acc(s.nTR);
    for (int iz = 0; iz < s.nz; iz++) {
        T zz = T(s.z[iz]);
        auto excite = [&](Iso<T> m, cx<T> theta) {                             // pssfp_kernels.cuh:46-55
            for (int i = 0; i < s.nRF; i++) {
                cx<T> zap = theta * cx<T>{T(s.gdtrf[2 * i]), T(s.gdtrf[2 * i + 1])};
                m = m.rotate(zap, T(s.gz_ex), zz, T(s.dt_ex), p).decay(E1_ex, E2_ex).regrowth(E1_ex);
            }
            return m;
        };
        auto precess = [&](Iso<T> m) {                                         // pssfp_kernels.cuh:58-63
            return m.precess(T(s.gz_pr), zz, T(s.dt_pr), p).decay(E1_pr, E2_pr).regrowth(E1_pr);
        };
        Iso<T> m;
        m = m.invert(p).decay(E1_inv, E2_inv).regrowth(E1_inv);                // pssfp_kernels.cuh:68-71
        cx<T> theta0 = {-T(s.rf[0]) / T(2), -T(s.rf[1]) / T(2)};
        m = excite(m, theta0);                                                 // pssfp_kernels.cuh:73-75
        m = m.precess(T(2) * T(s.gz_pr), zz, T(s.dt_pr), p).decay(E1_pr, E2_pr).regrowth(E1_pr);
        for (int t = 0; t < s.nTR; t++) {                                      // pssfp_kernels.cuh:83-107
            m = excite(m, cx<T>{T(s.rf[2 * t]), T(s.rf[2 * t + 1])});
            m = precess(m);
            acc[t] += cx<T>{m.x, m.y};
            m = precess(m);
        }
    }
    for (int t = 0; t < s.nTR; t++) echo[int64_t(t) * stride] = acc[t];
}

// --------------------------------------------------------------------------------------------
// Trajectories, signal, Jacobian products
// --------------------------------------------------------------------------------------------

struct Cartesian {
    int nr, ns;
    float dt;
    const float* k_start;  // complex [nr]
    float dk_re, dk_im;
};

// Cartesian readout factor: rewind to readout start + x-prephaser
// (compas/trajectories/cartesian_view.cuh:28-44)
template<typename T>
cx<T> cart_readout_factor(const Cartesian& t, const Voxel<T>& p) {
    T R2 = T(1) / p.T2;
    cx<T> arg = {-R2, two_pi<T>() * p.B0};
    cx<T> res = (T(-0.5) * T(t.ns) * T(t.dt)) * arg;
    T k0re = T(-0.5) * T(t.ns) * T(t.dk_re);
    res.im += k0re * p.x;
    return cexp(res);
}

// sample phase/decay from readout start   (cartesian_view.cuh:52-63)
template<typename T>
cx<T> cart_sample(const Cartesian& t, const Voxel<T>& p, int k) {
    T R2 = T(1) / p.T2;
    T Theta = T(t.dk_re) * p.x + T(t.dk_im) * p.y + T(t.dt) * two_pi<T>() * p.B0;
    return cexp(cx<T>{T(k) * (-T(t.dt) * R2), T(k) * Theta});
}

// echo-centred sample decay and its T2 derivative   (cartesian_view.cuh:65-92)
template<typename T>
void cart_sample_abs(const Cartesian& t, const Voxel<T>& p, int k, cx<T>& E, cx<T>& dE) {
    T R2 = T(1) / p.T2;
    T s = T(k) - T(0.5) * T(t.ns);
    T Theta = T(t.dk_re) * p.x + T(t.dk_im) * p.y + T(t.dt) * two_pi<T>() * p.B0;
    E = cexp(cx<T>{s * (-T(t.dt) * R2), s * Theta});
    dE = (s * T(t.dt) * R2 * R2) * E;
}

// phase_encoding: echo * exp(i y Im k_start[r])   (phase_encoding_kernels.cuh:10-25)
template<typename T>
cx<T> phase_encode(cx<T> m, const Voxel<T>& p, cx<T> kstart) {
    return m * cexp(cx<T>{T(0), p.y * kstart.im});
}

// Cartesian signal entry s[c][r][k] = Σ_v (ms ρ) s_k c   (signal_kernels.cuh:137-167)
template<typename T>
cx<T> signal_cartesian_entry(const float* echo, const float* params, int64_t nv, const Cartesian& t,
                             const float* coils, int c, int r, int k) {
    cx<T> sum;
    for (int64_t v = 0; v < nv; v++) {
        Voxel<T> p = load_voxel<T>(params, nv, v);
        cx<T> m = {T(echo[2 * (int64_t(r) * nv + v)]), T(echo[2 * (int64_t(r) * nv + v) + 1])};
        cx<T> ms = m * cart_readout_factor(t, p);
        cx<T> sk = cart_sample(t, p, k);
        cx<T> cc = {T(coils[2 * (int64_t(c) * nv + v)]), T(coils[2 * (int64_t(c) * nv + v) + 1])};
        sum += ((ms * p.rho) * sk) * cc;
    }
    return sum;
}

struct Spiral {
    int nr, ns;
    float dt;
    const float* k_start;  // complex [nr]
    const float* dk;       // complex [nr]
};

// spiral readout factor: rewind + prephaser with Re k0 · x only   (spiral_view.cuh:13-59)
template<typename T>
cx<T> spiral_readout(const Spiral& t, const Voxel<T>& p, int r, cx<T> m) {
    T R2 = T(1) / p.T2;
    T dtr = T(0.5 * t.ns) * T(t.dt);
    m = m * cexp(cx<T>{dtr * R2, dtr * (-two_pi<T>() * p.B0)});
    T k0re = T(t.k_start[2 * r]);
    return m * cexp(cx<T>{T(0), k0re * p.x});
}

// spiral per-sample step z = exp(-Δt R2 + iΘ_r)   (spiral_view.cuh:61-73)
template<typename T>
cx<T> spiral_step(const Spiral& t, const Voxel<T>& p, int r) {
    T R2 = T(1) / p.T2;
    T Theta = T(t.dk[2 * r]) * p.x + T(t.dk[2 * r + 1]) * p.y + T(t.dt) * two_pi<T>() * p.B0;
    return cexp(cx<T>{-T(t.dt) * R2, Theta});
}

// Spiral signal entry s[c][r][k] = Σ_v c · A[r][v] · z^k   (signal_kernels.cuh:274-345)
// The k-th power is evaluated exactly as exp(k(-Δt R2 + iΘ)) in the oracle.
template<typename T>
cx<T> signal_spiral_entry(const float* echo, const float* params, int64_t nv, const Spiral& t,
                          const float* coils, int c, int r, int k) {
    cx<T> sum;
    for (int64_t v = 0; v < nv; v++) {
        Voxel<T> p = load_voxel<T>(params, nv, v);
        cx<T> m = {T(echo[2 * (int64_t(r) * nv + v)]), T(echo[2 * (int64_t(r) * nv + v) + 1])};
        cx<T> A = spiral_readout(t, p, r, m) * p.rho;
        T R2 = T(1) / p.T2;
        T Theta = T(t.dk[2 * r]) * p.x + T(t.dk[2 * r + 1]) * p.y + T(t.dt) * two_pi<T>() * p.B0;
        cx<T> zk = cexp(cx<T>{T(k) * (-T(t.dt) * R2), T(k) * Theta});
        cx<T> cc = {T(coils[2 * (int64_t(c) * nv + v)]), T(coils[2 * (int64_t(c) * nv + v) + 1])};
        sum += cc * (A * zk);
    }
    return sum;
}

// J·v entry   (product_kernels.cuh:7-67)
template<typename T>
cx<T> jacobian_entry(const float* echo, const float* dT1, const float* dT2, const float* params, int64_t nv,
                     const Cartesian& t, const float* coils, const float* vec, int c, int r, int k) {
    cx<T> res;
    auto ld = [&](const float* a, int64_t i) { return cx<T>{T(a[2 * i]), T(a[2 * i + 1])}; };
    for (int64_t v = 0; v < nv; v++) {
        Voxel<T> p = load_voxel<T>(params, nv, v);
        cx<T> E, dE;
        cart_sample_abs(t, p, k, E, dE);
        cx<T> me = ld(echo, int64_t(r) * nv + v);
        cx<T> d1 = ld(dT1, int64_t(r) * nv + v), d2 = ld(dT2, int64_t(r) * nv + v);
        cx<T> prod = ld(vec, 0 * nv + v) * E * p.T1 * p.rho * d1
                   + ld(vec, 1 * nv + v) * (E * d2 + dE * me) * p.T2 * p.rho
                   + ld(vec, 2 * nv + v) * E * me
                   + ld(vec, 3 * nv + v) * E * cx<T>{T(0), T(1)} * me;
        res += prod * ld(coils, int64_t(c) * nv + v);
    }
    return res;
}

// Jᴴ·v for one voxel, all 4 fields   (hermitian_kernels.cuh:30-92)
template<typename T>
void jacobian_hermitian_voxel(const float* echo, const float* dT1, const float* dT2, const float* params,
                              int64_t nv, const Cartesian& t, const float* coils, int nc, const float* vec,
                              int64_t v, cx<T> out[4]) {
    auto ld = [&](const float* a, int64_t i) { return cx<T>{T(a[2 * i]), T(a[2 * i + 1])}; };
    Voxel<T> p = load_voxel<T>(params, nv, v);
    std::vector<cx<T>> E(t.ns), dE(t.ns);
    for (int k = 0; k < t.ns; k++) cart_sample_abs(t, p, k, E[k], dE[k]);
    for (int i = 0; i < 4; i++) out[i] = cx<T>();
    for (int c = 0; c < nc; c++) {
        cx<T> mHv, d0, d1;
        for (int r = 0; r < t.nr; r++) {
            cx<T> me = ld(echo, int64_t(r) * nv + v);
            cx<T> a1 = ld(dT1, int64_t(r) * nv + v), a2 = ld(dT2, int64_t(r) * nv + v);
            for (int k = 0; k < t.ns; k++) {
                cx<T> f = ld(vec, (int64_t(c) * t.nr + r) * t.ns + k);
                mHv += f * conj(E[k] * me);
                d0 += f * conj(a1 * E[k]);
                d1 += f * conj(a2 * E[k] + me * dE[k]);
            }
        }
        cx<T> cc = ld(coils, int64_t(c) * nv + v);
        out[0] += conj(p.T1 * p.rho) * conj(cc) * d0;
        out[1] += conj(p.T2 * p.rho) * conj(cc) * d1;
        out[2] += conj(cc) * mHv;
        out[3] += conj(cc) * mHv * cx<T>{T(0), T(-1)};
    }
}

// ---- spiral J·v and Jᴴ·v ----------------------------------------------------------------
// The reference's Jacobians accept only CartesianTrajectory (compas/jacobian/product.h:30,
// hermitian.h:30). These differentiate the spiral signal model of signal_spiral_entry
// (spiral_view.cuh:13-73, signal_kernels.cuh:274-345) with the column scaling of the Cartesian
// products (product_kernels.cuh:44-63): the per-readout factor F_rvk = readout_rv · z_rv^k depends
// on T2 through R2 = 1/T2 in the rewind exp((S/2)Δt R2) and in z^k = exp(k(-Δt R2 + iΘ)), so
// dF/dT2 = (k - S/2)·Δt·R2²·F, the same form as the Cartesian dE/dT2.
template<typename T>
cx<T> spiral_factor(const Spiral& t, const Voxel<T>& p, int r, int k) {
    const T R2 = T(1) / p.T2;
    const T Theta = T(t.dk[2 * r]) * p.x + T(t.dk[2 * r + 1]) * p.y + T(t.dt) * two_pi<T>() * p.B0;
    const cx<T> zk = cexp(cx<T>{T(k) * (-T(t.dt) * R2), T(k) * Theta});
    return spiral_readout(t, p, r, cx<T>{T(1), T(0)}) * zk;
}

template<typename T>
cx<T> spiral_jacobian_entry(const float* echo, const float* dT1, const float* dT2, const float* params, int64_t nv,
                            const Spiral& t, const float* coils, const float* vec, int c, int r, int k) {
    cx<T> res;
    auto ld = [&](const float* a, int64_t i) { return cx<T>{T(a[2 * i]), T(a[2 * i + 1])}; };
    for (int64_t v = 0; v < nv; v++) {
        Voxel<T> p = load_voxel<T>(params, nv, v);
        const cx<T> F = spiral_factor(t, p, r, k);
        const T R2 = T(1) / p.T2;
        const cx<T> dF = F * ((T(k) - T(0.5) * T(t.ns)) * T(t.dt) * R2 * R2);
        cx<T> me = ld(echo, int64_t(r) * nv + v);
        cx<T> d1 = ld(dT1, int64_t(r) * nv + v), d2 = ld(dT2, int64_t(r) * nv + v);
        cx<T> prod = ld(vec, 0 * nv + v) * F * p.T1 * p.rho * d1
                   + ld(vec, 1 * nv + v) * (F * d2 + dF * me) * p.T2 * p.rho
                   + ld(vec, 2 * nv + v) * F * me
                   + ld(vec, 3 * nv + v) * F * cx<T>{T(0), T(1)} * me;
        res += prod * ld(coils, int64_t(c) * nv + v);
    }
    return res;
}

template<typename T>
void spiral_jacobian_hermitian_voxel(const float* echo, const float* dT1, const float* dT2, const float* params,
                                     int64_t nv, const Spiral& t, const float* coils, int nc, const float* vec,
                                     int64_t v, cx<T> out[4]) {
    auto ld = [&](const float* a, int64_t i) { return cx<T>{T(a[2 * i]), T(a[2 * i + 1])}; };
    Voxel<T> p = load_voxel<T>(params, nv, v);
    const T R2 = T(1) / p.T2;
    for (int i = 0; i < 4; i++) out[i] = cx<T>();
    for (int r = 0; r < t.nr; r++) {
        cx<T> me = ld(echo, int64_t(r) * nv + v);
        cx<T> a1 = ld(dT1, int64_t(r) * nv + v), a2 = ld(dT2, int64_t(r) * nv + v);
        for (int k = 0; k < t.ns; k++) {
            const cx<T> F = spiral_factor(t, p, r, k);
            const cx<T> dF = F * ((T(k) - T(0.5) * T(t.ns)) * T(t.dt) * R2 * R2);
            for (int c = 0; c < nc; c++) {
                const cx<T> f = ld(vec, (int64_t(c) * t.nr + r) * t.ns + k) * conj(ld(coils, int64_t(c) * nv + v));
                out[0] += conj(p.T1 * p.rho) * f * conj(a1 * F);
                out[1] += conj(p.T2 * p.rho) * f * conj(a2 * F + me * dF);
                out[2] += f * conj(F * me);
            }
        }
    }
    out[3] = out[2] * cx<T>{T(0), T(-1)};
}

}  // namespace oracle
