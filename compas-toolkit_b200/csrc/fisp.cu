// fisp.cu — FISP extended-phase-graph simulation on sm_100a.
//
// Restates the reference's FISP EPG recurrence (src/operators/epg.cuh:13-322,
// src/simulate/fisp_kernels.cuh:99-223, src/simulate/fisp.cu:7-140) with a layout
// chosen for B200:
//
// * Work unit: one (voxel, slice position) pair per group of G lanes; each lane keeps
//   K consecutive EPG states (F+, F-, Z) in registers (G = 1: the whole state vector of
//   a voxel/position lives in one thread — no shuffles at all). A CTA holds VB = 32/G
//   voxels; its W warps sweep the slice positions round-robin and the per-TR samples of
//   all positions are summed in shared memory in a fixed order (deterministic result).
// * Algebra (exact rearrangement of the reference's per-TR sequence excite → decay(TE) →
//   sample → decay(TR-TE) → dephase): decay and rotation commute with the dephasing shift,
//   so the two relaxation steps of TR t are folded into the excitation matrix of TR t+1
//   (M' = M·diag(c, c̄, E1), c = E2(TR)·e^{2πi·B0·TR}); the regrowth becomes one additive
//   term on state 0. F+ and g = conj(F-) are stored; the update is done on
//   P = F+ + conj(F-), Q = F+ - conj(F-), in which M' is 2×2-block structured. Per state
//   and TR this is 26 FP32 operations against 48 for the reference's order.
// * The per-(position, TR) RF angle and phase table is built once per sequence and kept
//   resident with it.
#include <cfloat>
#include <optional>
#include <type_traits>

#include "common.cuh"
#include "compas/compas.h"
#include "job_args.cuh"
#include "kernels.h"

namespace compas {
namespace kernels {

// table[p][t] = {½·(π/180)·|sliceprofile[p][t]·RF[t]|, cos φ, sin φ, 0} for p < P, and in the extra
// row P: table[P][0].x = 1 when some entry has sin φ ≠ 0, else 0 (the row is zeroed before the launch)
__global__ void fisp_table_kernel(const float2* __restrict__ rf, const float2* __restrict__ slices, int nTR,
                                  int P, float4* __restrict__ table) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nTR * P) return;
    int t = i % nTR;
    float2 s = slices[i], r = rf[t];
    double re = double(s.x) * r.x - double(s.y) * r.y;
    double im = double(s.x) * r.y + double(s.y) * r.x;
    double a = sqrt(re * re + im * im);
    double cp = 1.0, sp = 0.0;
    if (a > double(FLT_MIN)) {  // epg.cuh:64-67
        cp = re / a;
        sp = im / a;
    }
    table[i] = make_float4(float(0.5 * (M_PI / 180.0) * a), float(cp), float(sp), 0.0f);
    if (float(sp) != 0.0f) table[int64_t(P) * nTR].x = 1.0f;  // every writer stores the same value
}

// True when every phase of the sequence's table is real (sin φ = 0 exactly: a real RF train and real
// slice profiles, as in the usual MR-STAT FISP sequences). The excitation coefficient d_re = sin φ·sin α·E1
// and β·R13_re are then ±0, and the packed update leaves out their products (EPGPacked::excite<true>).
__device__ __forceinline__ bool fisp_real_phases(const FispArgs& a) {
    return __ldg(&a.table[int64_t(a.P) * a.nTR].x) == 0.0f;
}


// Excitation coefficients of one TR, already multiplied by the preceding relaxation
// D = diag(c, c̄, E1) (see file header). Halved where the P/Q update needs it.
struct ExciteCoefs {
    float A1, A2, A3, A4;   // ½(a ± b) combinations
    float dre, dim;         // d = R13·E1
    float ere, eim;         // e = R31·c
    float f;                // R33·E1
    float bre, bim, bz;     // β·R13 (added to F+0 and conj(F-0)), β·R33 (added to Z0)
};

// Every operation is written with an explicit rounding (no multiply-add left to the compiler to
// fuse), so that the real-phase form below gives the same bits.
__device__ __forceinline__ ExciteCoefs make_coefs(float4 tab, float B1, float2 c, float E1, float beta) {
    float s, co;
    __sincosf(tab.x * B1, &s, &co);  // x = α/2   (epg.cuh:41-51)
    const float s2 = __fmul_rn(s, s), c2 = __fmul_rn(co, co);
    const float sa = __fmul_rn(2.0f * s, co);      // sin α
    const float ca = __fmaf_rn(2.0f, c2, -1.0f);   // cos α
    const float cp = tab.y, sp = tab.z;
    const float cos2p = __fmaf_rn(2.0f * cp, cp, -1.0f), sin2p = __fmul_rn(2.0f * cp, sp);
    // R11 = cos²(α/2), R12 = e^{2iφ} sin²(α/2), R13 = -i e^{iφ} sin α, R31 = -½ conj(R13), R33 = cos α
    const float r12re = __fmul_rn(cos2p, s2), r12im = __fmul_rn(sin2p, s2);
    const float r13re = __fmul_rn(sp, sa), r13im = -__fmul_rn(cp, sa);
    const float r31re = -0.5f * r13re, r31im = 0.5f * r13im;
    // a = R11·c, b = R12·c̄, d = R13·E1, e = R31·c, f = R33·E1
    const float are = __fmul_rn(c2, c.x), aim = __fmul_rn(c2, c.y);
    const float bre = __fmaf_rn(r12re, c.x, __fmul_rn(r12im, c.y));
    const float bim = __fmaf_rn(r12im, c.x, -__fmul_rn(r12re, c.y));
    ExciteCoefs k;
    k.A1 = 0.5f * __fadd_rn(are, bre);
    k.A2 = 0.5f * __fsub_rn(bim, aim);
    k.A3 = 0.5f * __fadd_rn(aim, bim);
    k.A4 = 0.5f * __fsub_rn(are, bre);
    k.dre = __fmul_rn(r13re, E1);
    k.dim = __fmul_rn(r13im, E1);
    k.ere = __fmaf_rn(r31re, c.x, -__fmul_rn(r31im, c.y));
    k.eim = __fmaf_rn(r31re, c.y, __fmul_rn(r31im, c.x));
    k.f = __fmul_rn(ca, E1);
    k.bre = __fmul_rn(beta, r13re);
    k.bim = __fmul_rn(beta, r13im);
    k.bz = __fmul_rn(beta, ca);
    return k;
}

// make_coefs for a real phase (sin φ = 0 and cos φ = ±1 exactly, as the table holds them when the
// RF sample times the slice profile is real): cos 2φ = 1 and sin 2φ = ±0, so R12 = sin²(α/2) and
// R13, R31 are imaginary. The products with those exact ones and zeros are left out; every other
// operation is the general form's, so the coefficients it returns are the same bits (up to the sign
// of an exact zero). d_re and β·R13_re, zero here, are not computed (the real-phase update does not
// read them).
__device__ __forceinline__ ExciteCoefs make_coefs_real(float4 tab, float B1, float2 c, float E1, float beta) {
    float s, co;
    __sincosf(tab.x * B1, &s, &co);
    const float s2 = __fmul_rn(s, s), c2 = __fmul_rn(co, co);
    const float sa = __fmul_rn(2.0f * s, co);
    const float ca = __fmaf_rn(2.0f, c2, -1.0f);
    const float cp = tab.y;
    const float r13im = -__fmul_rn(cp, sa);
    const float r31im = 0.5f * r13im;
    const float are = __fmul_rn(c2, c.x), aim = __fmul_rn(c2, c.y);
    const float bre = __fmul_rn(s2, c.x);
    const float bim = -__fmul_rn(s2, c.y);
    ExciteCoefs k;
    k.A1 = 0.5f * __fadd_rn(are, bre);
    k.A2 = 0.5f * __fsub_rn(bim, aim);
    k.A3 = 0.5f * __fadd_rn(aim, bim);
    k.A4 = 0.5f * __fsub_rn(are, bre);
    k.dre = 0.0f;
    k.dim = __fmul_rn(r13im, E1);
    k.ere = -__fmul_rn(r31im, c.y);
    k.eim = __fmul_rn(r31im, c.x);
    k.f = __fmul_rn(ca, E1);
    k.bre = 0.0f;
    k.bim = __fmul_rn(beta, r13im);
    k.bz = __fmul_rn(beta, ca);
    return k;
}

// y ← M'·x for one state (F+ = u, conj(F-) = g, Z = z)
__device__ __forceinline__ void excite_state(float2& u, float2& g, float2& z, const ExciteCoefs& k) {
    float Pr = u.x + g.x, Pi = u.y + g.y;
    float Qr = u.x - g.x, Qi = u.y - g.y;
    float Phr = fmaf(k.A1, Pr, fmaf(k.A2, Pi, k.dre * z.x));
    float Phi = fmaf(k.A3, Pr, fmaf(k.A4, Pi, k.dim * z.x));
    float Qhr = fmaf(k.A4, Qr, fmaf(-k.A3, Qi, -k.dim * z.y));
    float Qhi = fmaf(-k.A2, Qr, fmaf(k.A1, Qi, k.dre * z.y));
    float zr = fmaf(k.ere, Pr, fmaf(-k.eim, Pi, k.f * z.x));
    float zi = fmaf(k.ere, Qi, fmaf(k.eim, Qr, k.f * z.y));
    u = make_float2(Phr + Qhr, Phi + Qhi);
    g = make_float2(Phr - Qhr, Phi - Qhi);
    z = make_float2(zr, zi);
}

template<int K, int G>
struct EPG {
    float2 u[K], g[K], z[K];

    __device__ __forceinline__ void init(int sub) {
#pragma unroll
        for (int i = 0; i < K; i++) {
            u[i] = g[i] = z[i] = make_float2(0.f, 0.f);
        }
        if (sub == 0) z[0].x = 1.0f;
    }

    // dephasing gradient (epg.cuh:229-298): F- one state down with zero at ≥ N-1,
    // F+ one state up, F+0 = conj(F-0).
    // When the layout holds more than N states, F-[N-1] is zeroed by a one-hot bit test per slot.
    // Written as a compare of each slot index against N-1, the compiler may fold the unrolled
    // chain into one store at a run-time index, which moves the whole state to local memory.
    __device__ __forceinline__ void shift(int sub, int N) {
        if constexpr (G == 1) {
#pragma unroll
            for (int i = 0; i < K - 1; i++) g[i] = g[i + 1];
            g[K - 1] = make_float2(0.f, 0.f);
            if (N < K) {
                const unsigned cut = 1u << (N - 1);
#pragma unroll
                for (int i = 0; i < K - 1; i++)
                    if (cut & (1u << i)) g[i] = make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int i = K - 1; i > 0; i--) u[i] = u[i - 1];
            u[0] = g[0];
        } else {
            const unsigned mask = 0xffffffffu;
            float gx, gy, ux, uy;
            if constexpr ((G & (G - 1)) == 0) {
                gx = __shfl_down_sync(mask, g[0].x, 1, G);
                gy = __shfl_down_sync(mask, g[0].y, 1, G);
                ux = __shfl_up_sync(mask, u[K - 1].x, 1, G);
                uy = __shfl_up_sync(mask, u[K - 1].y, 1, G);
            } else {
                // groups that do not divide the warp (32 / G groups, the last 32 % G lanes idle):
                // explicit neighbour lanes; the values that cross a group boundary are replaced
                // below, as in the power-of-two case
                const int lane = threadIdx.x & 31;
                const int next = min(lane + 1, 31), prev = max(lane - 1, 0);
                gx = __shfl_sync(mask, g[0].x, next);
                gy = __shfl_sync(mask, g[0].y, next);
                ux = __shfl_sync(mask, u[K - 1].x, prev);
                uy = __shfl_sync(mask, u[K - 1].y, prev);
            }
#pragma unroll
            for (int i = 0; i < K - 1; i++) g[i] = g[i + 1];
            g[K - 1] = (sub == G - 1) ? make_float2(0.f, 0.f) : make_float2(gx, gy);
            const int lane_n = (N - 1) / K, slot_n = (N - 1) % K;
            if (sub == lane_n) {
                const unsigned cut = 1u << slot_n;
#pragma unroll
                for (int i = 0; i < K; i++)
                    if (cut & (1u << i)) g[i] = make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int i = K - 1; i > 0; i--) u[i] = u[i - 1];
            u[0] = (sub == 0) ? g[0] : make_float2(ux, uy);
        }
    }

    __device__ __forceinline__ void excite(const ExciteCoefs& k, int sub) {
#pragma unroll
        for (int i = 0; i < K; i++) excite_state(u[i], g[i], z[i], k);
        if (sub == 0) {
            u[0].x += k.bre;
            u[0].y += k.bim;
            g[0].x += k.bre;
            g[0].y += k.bim;
            z[0].x += k.bz;
        }
    }

    // F *= c (F+ by c, F- by c̄ ⇒ conj(F-) by c), Z *= E1, Z0 += 1 - E1
    __device__ __forceinline__ void relax(float2 c, float E1, int sub) {
#pragma unroll
        for (int i = 0; i < K; i++) {
            u[i] = cmul(u[i], c);
            g[i] = cmul(g[i], c);
            z[i] = cscale(E1, z[i]);
        }
        if (sub == 0) z[0].x += 1.0f - E1;
    }

    __device__ __forceinline__ void invert_spoil() {
#pragma unroll
        for (int i = 0; i < K; i++) {
            u[i] = g[i] = make_float2(0.f, 0.f);
            z[i] = make_float2(-z[i].x, -z[i].y);
        }
    }

    __device__ __forceinline__ void spoil() {
#pragma unroll
        for (int i = 0; i < K; i++) u[i] = g[i] = make_float2(0.f, 0.f);
    }

    // inversion, spoiling, then longitudinal relaxation and regrowth over TI
    __device__ __forceinline__ void invert_decay(float E1, int sub) {
        invert_spoil();
#pragma unroll
        for (int i = 0; i < K; i++) z[i] = cscale(E1, z[i]);
        if (sub == 0) z[0].x += 1.0f - E1;
    }

    __device__ __forceinline__ float2 f0() const { return u[0]; }  // F+ of state 0 (lane sub == 0)
};

// The excitation coefficients of make_coefs broadcast to both halves of a pair. The packed state
// keeps -Im Z and forms -Im Q, which turns every negated coefficient of excite_state into a
// positive one except -e_im (the two-wide FMA has no operand negation, so each negated copy would
// cost a register pair).
struct ExciteCoefs2 {
    float2 A1, A2, A3, A4, dre, dim, ere, neim, f;
    float bre, bim, bz;
};

template<bool REAL = false>
__device__ __forceinline__ ExciteCoefs2 make_coefs2(float4 tab, float B1, float2 c, float E1, float beta) {
    const ExciteCoefs k = REAL ? make_coefs_real(tab, B1, c, E1, beta) : make_coefs(tab, B1, c, E1, beta);
    ExciteCoefs2 q;
    q.A1 = bcast2(k.A1);
    q.A2 = bcast2(k.A2);
    q.A3 = bcast2(k.A3);
    q.A4 = bcast2(k.A4);
    q.dre = bcast2(k.dre);
    q.dim = bcast2(k.dim);
    q.ere = bcast2(k.ere);
    q.neim = bcast2(-k.eim);
    q.f = bcast2(k.f);
    q.bre = k.bre;
    q.bim = k.bim;
    q.bz = k.bz;
    return q;
}

// Packed-pair EPG state (one lane per voxel/position, 2·KP + EXTRA state slots): pair j holds state
// j in .x and state j + KP in .y, one register pair per real component (Re/Im of F+, of conj(F-), and
// Re Z and -Im Z). All states of a TR share the excitation coefficients, so every operation of
// excite_state becomes one two-wide instruction (add2/mul2/fma2) on a pair: 26 issue slots per
// two states instead of 52, with the same roundings as the scalar update (negating an operand or
// a result is exact). Only the two states that cross the pair boundary in the dephasing shift
// (KP-1 → KP for F+, KP → KP-1 for conj(F-)) move between halves. EXTRA = 1 adds an unpaired slot
// 2·KP (scalar registers, the same operations one-wide): an odd state count then needs no padding
// slot (25 states: 12 pairs and one slot, where 13 pairs spend a twenty-sixth slot's update on a
// state that is zeroed every TR).
template<int KP, int EXTRA = 0>
struct EPGPacked {
    static_assert(KP >= 2, "at least two pairs");
    static_assert(EXTRA == 0 || EXTRA == 1, "at most one unpaired slot");
    static constexpr int K = 2 * KP + EXTRA;
    float2 ur[KP], ui[KP], gr[KP], gi[KP], zr[KP], zn[KP];  // zn = -Im Z
    float eur, eui, egr, egi, ezr, ezn;                      // the unpaired slot 2·KP (EXTRA)

    __device__ __forceinline__ void init(int) {
#pragma unroll
        for (int j = 0; j < KP; j++) ur[j] = ui[j] = gr[j] = gi[j] = zr[j] = zn[j] = make_float2(0.f, 0.f);
        zr[0].x = 1.0f;
        eur = eui = egr = egi = ezr = ezn = 0.f;
    }

    // dephasing (epg.cuh:229-298): conj(F-) one state down (state s ← s+1, zero at ≥ N-1), F+ one
    // state up (s ← s-1), F+0 = conj(F-0). The zeroing of state N-1 uses a one-hot bit test per
    // slot, which keeps the state in registers.
    __device__ __forceinline__ void shift(int, int N) {
        const float cr = gr[0].y, ci = gi[0].y;  // conj(F-) of state KP → state KP-1
#pragma unroll
        for (int j = 0; j < KP - 1; j++) {
            gr[j] = gr[j + 1];
            gi[j] = gi[j + 1];
        }
        // state 2KP-1 takes the unpaired slot's conj(F-), or the zero beyond the layout; the unpaired
        // slot takes the zero beyond the layout
        gr[KP - 1] = make_float2(cr, EXTRA ? egr : 0.f);
        gi[KP - 1] = make_float2(ci, EXTRA ? egi : 0.f);
        egr = egi = 0.f;
        if constexpr (EXTRA == 0) {
            if (N == K - 1) {  // one padding slot (25 states in 26): state K-2 is pair KP-2, high half
                gr[KP - 2].y = gi[KP - 2].y = 0.f;
            } else if (N < K - 1) {
                const unsigned cut = 1u << (N - 1);
#pragma unroll
                for (int j = 0; j < KP; j++) {
                    if (cut & (1u << j)) gr[j].x = gi[j].x = 0.f;
                    if (cut & (1u << (j + KP))) gr[j].y = gi[j].y = 0.f;
                }
            }
        } else if (N < K) {  // state N-1 is a paired slot (N = K: the unpaired slot, zero already)
            const unsigned cut = 1u << (N - 1);
#pragma unroll
            for (int j = 0; j < KP; j++) {
                if (cut & (1u << j)) gr[j].x = gi[j].x = 0.f;
                if (cut & (1u << (j + KP))) gr[j].y = gi[j].y = 0.f;
            }
        }
        const float ar = ur[KP - 1].x, ai = ui[KP - 1].x;  // F+ of state KP-1 → state KP
        if constexpr (EXTRA) {  // F+ of state 2KP-1 → the unpaired slot (its old F+ leaves the layout)
            eur = ur[KP - 1].y;
            eui = ui[KP - 1].y;
        }
#pragma unroll
        for (int j = KP - 1; j > 0; j--) {
            ur[j] = ur[j - 1];
            ui[j] = ui[j - 1];
        }
        ur[0] = make_float2(gr[0].x, ar);
        ui[0] = make_float2(gi[0].x, ai);
    }

    // excite_state on a pair with Qn = -Im Q, zn = -Im Z and nQhi = -Im Qh:
    //   Qh_r = A4·Qr + A3·Qn + d_im·zn,   -Qh_i = A2·Qr + A1·Qn + d_re·zn,
    //   Z_r' = e_re·Pr - e_im·Pi + f·Z_r,   -Z_i' = e_re·Qn - e_im·Qr + f·zn
    // REAL (every RF phase real, fisp_real_phases): d_re and β·R13_re are ±0, so d_re·Z_r, d_re·zn and
    // the β·R13_re additions are left out: 24 instructions per pair instead of 26. An FMA that adds ±0
    // to a product returns the rounded product, so the results are the same bits up to the sign of an
    // exact zero.
    template<bool REAL = false>
    __device__ __forceinline__ void excite(const ExciteCoefs2& k, int) {
        // the unpaired slot first: the same operations one-wide (placed before the pairs, the
        // 25-slot kernel ran 44.1 ms at the MR-STAT slice; after them 45.9 ms)
        if constexpr (EXTRA) {
            const float Pr = eur + egr, Pi = eui + egi;
            const float Qr = eur - egr, Qn = egi - eui;
            const float Phr = REAL ? fmaf(k.A1.x, Pr, k.A2.x * Pi) : fmaf(k.A1.x, Pr, fmaf(k.A2.x, Pi, k.dre.x * ezr));
            const float Phi = fmaf(k.A3.x, Pr, fmaf(k.A4.x, Pi, k.dim.x * ezr));
            const float Qhr = fmaf(k.A4.x, Qr, fmaf(k.A3.x, Qn, k.dim.x * ezn));
            const float nQhi = REAL ? fmaf(k.A2.x, Qr, k.A1.x * Qn) : fmaf(k.A2.x, Qr, fmaf(k.A1.x, Qn, k.dre.x * ezn));
            const float nzr = fmaf(k.ere.x, Pr, fmaf(k.neim.x, Pi, k.f.x * ezr));
            const float nzn = fmaf(k.ere.x, Qn, fmaf(k.neim.x, Qr, k.f.x * ezn));
            eur = Phr + Qhr;
            eui = Phi - nQhi;
            egr = Phr - Qhr;
            egi = Phi + nQhi;
            ezr = nzr;
            ezn = nzn;
        }
#pragma unroll
        for (int j = 0; j < KP; j++) {
            const float2 Pr = add2(ur[j], gr[j]), Pi = add2(ui[j], gi[j]);
            const float2 Qr = sub2(ur[j], gr[j]), Qn = sub2(gi[j], ui[j]);
            const float2 Phr = REAL ? fma2(k.A1, Pr, mul2(k.A2, Pi)) : fma2(k.A1, Pr, fma2(k.A2, Pi, mul2(k.dre, zr[j])));
            const float2 Phi = fma2(k.A3, Pr, fma2(k.A4, Pi, mul2(k.dim, zr[j])));
            const float2 Qhr = fma2(k.A4, Qr, fma2(k.A3, Qn, mul2(k.dim, zn[j])));
            const float2 nQhi = REAL ? fma2(k.A2, Qr, mul2(k.A1, Qn)) : fma2(k.A2, Qr, fma2(k.A1, Qn, mul2(k.dre, zn[j])));
            const float2 nzr = fma2(k.ere, Pr, fma2(k.neim, Pi, mul2(k.f, zr[j])));
            const float2 nzn = fma2(k.ere, Qn, fma2(k.neim, Qr, mul2(k.f, zn[j])));
            ur[j] = add2(Phr, Qhr);
            ui[j] = sub2(Phi, nQhi);
            gr[j] = sub2(Phr, Qhr);
            gi[j] = add2(Phi, nQhi);
            zr[j] = nzr;
            zn[j] = nzn;
        }
        if constexpr (!REAL) {
            ur[0].x += k.bre;
            gr[0].x += k.bre;
        }
        ui[0].x += k.bim;
        gi[0].x += k.bim;
        zr[0].x += k.bz;
    }

    // F *= c (F+ by c, conj(F-) by c), Z *= E1, Z0 += 1 - E1
    __device__ __forceinline__ void relax(float2 c, float E1, int) {
        const float2 cx = bcast2(c.x), cy = bcast2(c.y), ncy = bcast2(-c.y), e1 = bcast2(E1);
#pragma unroll
        for (int j = 0; j < KP; j++) {
            const float2 a = fma2(ur[j], cx, mul2(ui[j], ncy)), b = fma2(ur[j], cy, mul2(ui[j], cx));
            const float2 d = fma2(gr[j], cx, mul2(gi[j], ncy)), e = fma2(gr[j], cy, mul2(gi[j], cx));
            ur[j] = a;
            ui[j] = b;
            gr[j] = d;
            gi[j] = e;
            zr[j] = mul2(e1, zr[j]);
            zn[j] = mul2(e1, zn[j]);
        }
        if constexpr (EXTRA) {
            const float a = fmaf(eur, cx.x, eui * ncy.x), b = fmaf(eur, cy.x, eui * cx.x);
            const float d = fmaf(egr, cx.x, egi * ncy.x), e = fmaf(egr, cy.x, egi * cx.x);
            eur = a;
            eui = b;
            egr = d;
            egi = e;
            ezr = E1 * ezr;
            ezn = E1 * ezn;
        }
        zr[0].x += 1.0f - E1;
    }

    __device__ __forceinline__ void invert_spoil() {
#pragma unroll
        for (int j = 0; j < KP; j++) {
            ur[j] = ui[j] = gr[j] = gi[j] = make_float2(0.f, 0.f);
            zr[j] = make_float2(-zr[j].x, -zr[j].y);
            zn[j] = make_float2(-zn[j].x, -zn[j].y);
        }
        eur = eui = egr = egi = 0.f;
        ezr = -ezr;
        ezn = -ezn;
    }

    __device__ __forceinline__ void spoil() {
#pragma unroll
        for (int j = 0; j < KP; j++) ur[j] = ui[j] = gr[j] = gi[j] = make_float2(0.f, 0.f);
        eur = eui = egr = egi = 0.f;
    }

    __device__ __forceinline__ void invert_decay(float E1, int) {
        invert_spoil();
        const float2 e1 = bcast2(E1);
#pragma unroll
        for (int j = 0; j < KP; j++) {
            zr[j] = mul2(e1, zr[j]);
            zn[j] = mul2(e1, zn[j]);
        }
        ezr = E1 * ezr;
        ezn = E1 * ezn;
        zr[0].x += 1.0f - E1;
    }

    __device__ __forceinline__ float2 f0() const { return make_float2(ur[0].x, ui[0].x); }
};

// Forward-mode tangents ∂/∂T1 and ∂/∂T2 carried with the state.
//
// The reference differentiates by forward differences, one more simulation per field at
// p + Δ·e_field (src/simulate/derivative.cu:11-62, derivative_kernels.cuh:6-35). Every step of
// the recurrence is affine in the state, x' = M(θ)·x + b(θ), so its tangent is
// x'_θ = M·x_θ + M_θ·x + b_θ. With the relaxation folded into the excitation (file header) the
// extra terms are the same excitation applied to a shifted input:
//  * T1 enters through E1 = e^{-t/T1} on Z and the regrowth (1 - E1) on Z0, and
//    ∂E1/∂T1 = s1·E1 with s1 = t/T1², so M_θ·x + b_θ = M·(0, 0, s1·(z - δ_{n0})): the T1 tangent
//    is the excitation of (u₁, g₁, z₁ + s1·(z - δ_{n0}));
//  * T2 enters through c = E2·e^{2πi·B0·t} on F+ and conj(F-), ∂c/∂T2 = s2·c with s2 = t/T2²:
//    the T2 tangent is the excitation of (u₂ + s2·u, g₂ + s2·g, z₂).
// Per state and TR that is 26 + 28 + 30 FP32 operations, about what the value and two
// forward-difference simulations cost, without the differences' cancellation error.
template<int K, int G>
struct EPGTangent {
    EPG<K, G> x, d1, d2;  // value, ∂/∂T1, ∂/∂T2

    __device__ __forceinline__ void init(int sub) {
        x.init(sub);
#pragma unroll
        for (int i = 0; i < K; i++) {
            d1.u[i] = d1.g[i] = d1.z[i] = make_float2(0.f, 0.f);
            d2.u[i] = d2.g[i] = d2.z[i] = make_float2(0.f, 0.f);
        }
    }

    __device__ __forceinline__ void shift(int sub, int N) {
        x.shift(sub, N);
        d1.shift(sub, N);
        d2.shift(sub, N);
    }

    // z - δ_{n0}: the regrowth's share of ∂Z/∂E1 (state 0 lives in slot 0 of lane 0)
    __device__ __forceinline__ float2 zshift(int i, int sub) const {
        return make_float2(i == 0 && sub == 0 ? x.z[0].x - 1.0f : x.z[i].x, x.z[i].y);
    }

    // excitation k, which holds the relaxation over t before it; s1 = t/T1², s2 = t/T2²
    __device__ __forceinline__ void excite(const ExciteCoefs& k, float s1, float s2, int sub) {
#pragma unroll
        for (int i = 0; i < K; i++) {
            const float2 zs = zshift(i, sub);
            float2 z1 = make_float2(fmaf(s1, zs.x, d1.z[i].x), fmaf(s1, zs.y, d1.z[i].y));
            float2 u2 = make_float2(fmaf(s2, x.u[i].x, d2.u[i].x), fmaf(s2, x.u[i].y, d2.u[i].y));
            float2 g2 = make_float2(fmaf(s2, x.g[i].x, d2.g[i].x), fmaf(s2, x.g[i].y, d2.g[i].y));
            excite_state(d1.u[i], d1.g[i], z1, k);
            d1.z[i] = z1;
            excite_state(u2, g2, d2.z[i], k);
            d2.u[i] = u2;
            d2.g[i] = g2;
        }
        x.excite(k, sub);
    }

    // relaxation over t: F·c, Z·E1, Z0 += 1 - E1
    __device__ __forceinline__ void relax(float2 c, float E1, float s1, float s2, int sub) {
#pragma unroll
        for (int i = 0; i < K; i++) {
            const float2 zs = zshift(i, sub);
            d1.u[i] = cmul(d1.u[i], c);
            d1.g[i] = cmul(d1.g[i], c);
            d1.z[i] = cscale(E1, make_float2(fmaf(s1, zs.x, d1.z[i].x), fmaf(s1, zs.y, d1.z[i].y)));
            d2.u[i] = cmul(make_float2(fmaf(s2, x.u[i].x, d2.u[i].x), fmaf(s2, x.u[i].y, d2.u[i].y)), c);
            d2.g[i] = cmul(make_float2(fmaf(s2, x.g[i].x, d2.g[i].x), fmaf(s2, x.g[i].y, d2.g[i].y)), c);
            d2.z[i] = cscale(E1, d2.z[i]);
        }
        x.relax(c, E1, sub);
    }

    // inversion, spoiling, then longitudinal relaxation over TI (s1 = TI/T1²)
    __device__ __forceinline__ void invert_decay(float E1, float s1, int sub) {
        x.invert_spoil();
        d1.invert_spoil();
        d2.invert_spoil();
#pragma unroll
        for (int i = 0; i < K; i++) {
            const float2 zs = zshift(i, sub);
            d1.z[i] = cscale(E1, make_float2(fmaf(s1, zs.x, d1.z[i].x), fmaf(s1, zs.y, d1.z[i].y)));
            d2.z[i] = cscale(E1, d2.z[i]);
            x.z[i] = cscale(E1, x.z[i]);
        }
        if (sub == 0) x.z[0].x += 1.0f - E1;
    }

    __device__ __forceinline__ void spoil() {
        x.spoil();
        d1.spoil();
        d2.spoil();
    }

    // F+ of state 0 (lane sub == 0) of the value (v = 0), ∂/∂T1 (1) or ∂/∂T2 (2)
    __device__ __forceinline__ float2 f0(int v) const { return v == 0 ? x.u[0] : v == 1 ? d1.u[0] : d2.u[0]; }
};

// The excitation of one pair of states in the packed representation (EPGPacked::excite's update,
// without the regrowth terms of state 0): every operation two-wide, in excite_state's order.
template<bool REAL>
__device__ __forceinline__ void excite_pair(const ExciteCoefs2& k, float2& ur, float2& ui, float2& gr, float2& gi,
                                            float2& zr, float2& zn) {
    const float2 Pr = add2(ur, gr), Pi = add2(ui, gi);
    const float2 Qr = sub2(ur, gr), Qn = sub2(gi, ui);
    const float2 Phr = REAL ? fma2(k.A1, Pr, mul2(k.A2, Pi)) : fma2(k.A1, Pr, fma2(k.A2, Pi, mul2(k.dre, zr)));
    const float2 Phi = fma2(k.A3, Pr, fma2(k.A4, Pi, mul2(k.dim, zr)));
    const float2 Qhr = fma2(k.A4, Qr, fma2(k.A3, Qn, mul2(k.dim, zn)));
    const float2 nQhi = REAL ? fma2(k.A2, Qr, mul2(k.A1, Qn)) : fma2(k.A2, Qr, fma2(k.A1, Qn, mul2(k.dre, zn)));
    const float2 nzr = fma2(k.ere, Pr, fma2(k.neim, Pi, mul2(k.f, zr)));
    const float2 nzn = fma2(k.ere, Qn, fma2(k.neim, Qr, mul2(k.f, zn)));
    ur = add2(Phr, Qhr);
    ui = sub2(Phi, nQhi);
    gr = sub2(Phr, Qhr);
    gi = add2(Phi, nQhi);
    zr = nzr;
    zn = nzn;
}

// Two-wide form of EPGTangent: the value and its T1 and T2 tangents (vectors v = 0, 1, 2), each in
// the packed representation of EPGPacked (pair j of a lane holds the lane's states j in .x and j + KP
// in .y; Re Z and -Im Z), on G lanes of K = 2·KP states each (states sub·K .. sub·K + K-1 on lane sub).
// The operations are EPGTangent's in the same order, so layout (K, G) gives the bits of the scalar
// tangent layout (K, G). The dephasing shift exchanges the boundary states with the neighbour lanes
// as EPG<K, G> does.
// CUT0: state N-1 is the first state of its lane ((N-1) % K == 0, as for 25 states on 4 lanes of 8),
// so the truncation zeroes one known slot; otherwise a one-hot bit test per slot finds it. The
// bit tests and their selects sat between every shifted state and its next excitation (the ALU pipe
// 22 % busy at 25 states on 4 x 8). Zeroing is exact either way: the same bits.
template<int KP, int G, bool CUT0 = false>
struct EPGPackedTangent {
    static_assert(KP >= 2 && G >= 1 && G <= 32 && (G & (G - 1)) == 0, "pairs per lane, power-of-two lane groups");
    static constexpr int K = 2 * KP;
    float2 ur[3][KP], ui[3][KP], gr[3][KP], gi[3][KP], zr[3][KP], zn[3][KP];  // zn = -Im Z

    __device__ __forceinline__ void init(int sub) {
#pragma unroll
        for (int v = 0; v < 3; v++)
#pragma unroll
            for (int j = 0; j < KP; j++) ur[v][j] = ui[v][j] = gr[v][j] = gi[v][j] = zr[v][j] = zn[v][j] = make_float2(0.f, 0.f);
        if (sub == 0) zr[0][0].x = 1.0f;
    }

    __device__ __forceinline__ void shift_vector(int v, int sub, int N) {
        const unsigned mask = 0xffffffffu;
        // the neighbour lanes' boundary states, read before this lane shifts: conj(F-) of the next
        // lane's first state, F+ of the previous lane's last state
        float ngr = 0.f, ngi = 0.f, pur = 0.f, pui = 0.f;
        if constexpr (G > 1) {
            ngr = __shfl_down_sync(mask, gr[v][0].x, 1, G);
            ngi = __shfl_down_sync(mask, gi[v][0].x, 1, G);
            pur = __shfl_up_sync(mask, ur[v][KP - 1].y, 1, G);
            pui = __shfl_up_sync(mask, ui[v][KP - 1].y, 1, G);
        }
        const float cr = gr[v][0].y, ci = gi[v][0].y;  // conj(F-) of state KP → state KP-1
#pragma unroll
        for (int j = 0; j < KP - 1; j++) {
            gr[v][j] = gr[v][j + 1];
            gi[v][j] = gi[v][j + 1];
        }
        const bool last = sub == G - 1;  // the last lane's top state takes the zero beyond the layout
        gr[v][KP - 1] = make_float2(cr, last ? 0.f : ngr);
        gi[v][KP - 1] = make_float2(ci, last ? 0.f : ngi);
        if constexpr (CUT0) {
            if (sub == (N - 1) / K) gr[v][0].x = gi[v][0].x = 0.f;  // state N-1 = this lane's slot 0
        } else if (sub == (N - 1) / K) {  // zero state N-1 (one-hot bit test per slot)
            const unsigned cut = 1u << ((N - 1) % K);
#pragma unroll
            for (int j = 0; j < KP; j++) {
                if (cut & (1u << j)) gr[v][j].x = gi[v][j].x = 0.f;
                if (cut & (1u << (j + KP))) gr[v][j].y = gi[v][j].y = 0.f;
            }
        }
        const float ar = ur[v][KP - 1].x, ai = ui[v][KP - 1].x;  // F+ of state KP-1 → state KP
#pragma unroll
        for (int j = KP - 1; j > 0; j--) {
            ur[v][j] = ur[v][j - 1];
            ui[v][j] = ui[v][j - 1];
        }
        ur[v][0] = make_float2(sub == 0 ? gr[v][0].x : pur, ar);  // F+0 = conj(F-0)
        ui[v][0] = make_float2(sub == 0 ? gi[v][0].x : pui, ai);
    }

    __device__ __forceinline__ void shift(int sub, int N) {
#pragma unroll
        for (int v = 0; v < 3; v++) shift_vector(v, sub, N);
    }

    // EPGTangent::excite: the T1 tangent excites (F1, Z1 + s1·(Z - δ_{n0})), the T2 tangent
    // (F2 + s2·F, Z2), both from the value before its own excitation
    template<bool REAL = false>
    __device__ __forceinline__ void excite(const ExciteCoefs2& k, float s1, float s2, int sub) {
        const float2 S1 = bcast2(s1), S2 = bcast2(s2);
#pragma unroll
        for (int j = 0; j < KP; j++) {
            float2 zs = zr[0][j];
            if (j == 0 && sub == 0) zs.x = zr[0][0].x - 1.0f;
            zr[1][j] = fma2(S1, zs, zr[1][j]);
            zn[1][j] = fma2(S1, zn[0][j], zn[1][j]);
            excite_pair<REAL>(k, ur[1][j], ui[1][j], gr[1][j], gi[1][j], zr[1][j], zn[1][j]);
            ur[2][j] = fma2(S2, ur[0][j], ur[2][j]);
            ui[2][j] = fma2(S2, ui[0][j], ui[2][j]);
            gr[2][j] = fma2(S2, gr[0][j], gr[2][j]);
            gi[2][j] = fma2(S2, gi[0][j], gi[2][j]);
            excite_pair<REAL>(k, ur[2][j], ui[2][j], gr[2][j], gi[2][j], zr[2][j], zn[2][j]);
        }
#pragma unroll
        for (int j = 0; j < KP; j++) excite_pair<REAL>(k, ur[0][j], ui[0][j], gr[0][j], gi[0][j], zr[0][j], zn[0][j]);
        if (sub == 0) {  // the regrowth terms of state 0 (EPG::excite)
            if constexpr (!REAL) {
                ur[0][0].x += k.bre;
                gr[0][0].x += k.bre;
            }
            ui[0][0].x += k.bim;
            gi[0][0].x += k.bim;
            zr[0][0].x += k.bz;
        }
    }

    // EPGTangent::relax: F·c, Z·E1 on the value; the tangents as there
    __device__ __forceinline__ void relax(float2 c, float E1, float s1, float s2, int sub) {
        const float2 cx = bcast2(c.x), cy = bcast2(c.y), ncy = bcast2(-c.y), e1 = bcast2(E1);
        const float2 S1 = bcast2(s1), S2 = bcast2(s2);
        auto rot = [&](float2& re, float2& im) {
            const float2 a = fma2(re, cx, mul2(im, ncy)), b = fma2(re, cy, mul2(im, cx));
            re = a;
            im = b;
        };
#pragma unroll
        for (int j = 0; j < KP; j++) {
            float2 zs = zr[0][j];
            if (j == 0 && sub == 0) zs.x = zr[0][0].x - 1.0f;
            rot(ur[1][j], ui[1][j]);
            rot(gr[1][j], gi[1][j]);
            zr[1][j] = mul2(e1, fma2(S1, zs, zr[1][j]));
            zn[1][j] = mul2(e1, fma2(S1, zn[0][j], zn[1][j]));
            ur[2][j] = fma2(S2, ur[0][j], ur[2][j]);
            ui[2][j] = fma2(S2, ui[0][j], ui[2][j]);
            gr[2][j] = fma2(S2, gr[0][j], gr[2][j]);
            gi[2][j] = fma2(S2, gi[0][j], gi[2][j]);
            rot(ur[2][j], ui[2][j]);
            rot(gr[2][j], gi[2][j]);
            zr[2][j] = mul2(e1, zr[2][j]);
            zn[2][j] = mul2(e1, zn[2][j]);
        }
#pragma unroll
        for (int j = 0; j < KP; j++) {
            rot(ur[0][j], ui[0][j]);
            rot(gr[0][j], gi[0][j]);
            zr[0][j] = mul2(e1, zr[0][j]);
            zn[0][j] = mul2(e1, zn[0][j]);
        }
        if (sub == 0) zr[0][0].x += 1.0f - E1;
    }

    __device__ __forceinline__ void spoil() {
#pragma unroll
        for (int v = 0; v < 3; v++)
#pragma unroll
            for (int j = 0; j < KP; j++) ur[v][j] = ui[v][j] = gr[v][j] = gi[v][j] = make_float2(0.f, 0.f);
    }

    // EPGTangent::invert_decay: inversion and spoiling of all three, then relaxation over TI
    __device__ __forceinline__ void invert_decay(float E1, float s1, int sub) {
        spoil();
        const float2 e1 = bcast2(E1), S1 = bcast2(s1);
#pragma unroll
        for (int v = 0; v < 3; v++)
#pragma unroll
            for (int j = 0; j < KP; j++) {
                zr[v][j] = make_float2(-zr[v][j].x, -zr[v][j].y);
                zn[v][j] = make_float2(-zn[v][j].x, -zn[v][j].y);
            }
#pragma unroll
        for (int j = 0; j < KP; j++) {
            float2 zs = zr[0][j];
            if (j == 0 && sub == 0) zs.x = zr[0][0].x - 1.0f;
            zr[1][j] = mul2(e1, fma2(S1, zs, zr[1][j]));
            zn[1][j] = mul2(e1, fma2(S1, zn[0][j], zn[1][j]));
            zr[2][j] = mul2(e1, zr[2][j]);
            zn[2][j] = mul2(e1, zn[2][j]);
            zr[0][j] = mul2(e1, zr[0][j]);
            zn[0][j] = mul2(e1, zn[0][j]);
        }
        if (sub == 0) zr[0][0].x += 1.0f - E1;
    }

    __device__ __forceinline__ float2 f0(int v) const { return make_float2(ur[v][0].x, ui[v][0].x); }
};

// The work of a FISP simulation is a list of items (voxel tile, slice position), tile-major:
// item = tile·P + p, a tile being VB = 32/G voxels. A CTA runs a contiguous range of items in
// rounds of W: in each round warp w runs item base + w (its whole TR sequence), so a round may
// hold the last positions of one tile and the first of the next and no warp idles at a tile's
// end (35 positions on 8 warps no longer leave a round of 3). The one-simulation kernel gives each
// CTA a contiguous range of whole tiles; the batched work-queue kernel runs one tile per queue
// item. Both call this function.
// Summation: the echo of a voxel is the sum over positions in increasing p, accumulated one
// position at a time, ((s_0 + s_1) + s_2) + … . A round adds its positions of a tile to the
// partial sum the previous round wrote to the echo array, so the result does not depend on how
// the items fall into rounds: the work-queue kernel gives the same bits as the one-simulation
// kernel.
// TRs per sample chunk: the CTA's warps meet at a barrier once per chunk to sum their positions'
// samples in shared memory ([W][chunk][VB] per sample plane). The split-lane tangent layouts use
// 64 TRs, halving their barriers (271 -> 266 ms on the 224² MR-STAT slice), and so do the one-lane
// value layouts (with four TRs per loop iteration: 42.7 -> 41.8 ms; with two, 64 had measured 0.5 %
// slower); the value layouts split over lanes and the one-lane tangent layouts keep 32 (three planes
// of 32 voxels per warp would not fit in 227 KB at 64).
template<int G, bool TAN>
constexpr int kFispChunk = ((TAN && G > 1) || (!TAN && G == 1)) ? 64 : 32;

// state type of a layout: value PACKED (G = 1) → EPGPacked<K/2, K%2>; TAN → EPGTangent, or
// EPGPackedTangent<K/2, G, CUT0> when PACKED; else EPG
template<int K, int G, bool TAN, bool PACKED, bool CUT0 = false>
using FispState =
    std::conditional_t<TAN, std::conditional_t<PACKED, EPGPackedTangent<K / 2, G, CUT0>, EPGTangent<K, G>>,
                       std::conditional_t<PACKED, EPGPacked<K / 2, K % 2>, EPG<K, G>>>;

// Balanced item split of the one-simulation kernel: the order of a CTA's items (at most
// kFispBalancedItems) and its hand-off points, in shared memory
constexpr int kFispBalancedItems = 2048;
struct FispOrder {
    int item[kFispBalancedItems];  // item of the u-th position in the CTA's order
    int wait_u;                    // first u of the head part (positions of the shared first tile)
    int publish_u;                 // u after the tail part (first positions of the shared last tile)
    int cta;
    int* handoff;                  // per-CTA flags, zero at launch
    unsigned int* status;          // device status word
};

// Hand-off flags of the balanced item split: a CTA publishes the partial sums of its last, shared
// tile, and the next CTA waits for them before it adds its positions of that tile. The wait is
// bounded: one that gives up records STATUS_WAIT_TIMEOUT in the status word and returns.
__device__ __forceinline__ void handoff_publish(int* flag) {
    __threadfence();  // the CTA's partial-sum stores (ordered before by the barrier) are visible first
    atomicExch(flag, 1);
}
__device__ __forceinline__ void handoff_wait(const int* flag, unsigned int* status) {
    const long long t0 = clock64();
    for (;;) {
        int v;
        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v != 0) return;
        if (clock64() - t0 > 4000000000LL) {
            if (status) atomicOr(status, STATUS_WAIT_TIMEOUT);
            return;
        }
        __nanosleep(256);
    }
}

// TAN: also propagate ∂/∂T1 and ∂/∂T2 (EPGTangent) and write them to a.dT1, a.dT2; the
// value goes through the same operations either way.
// BAL: items u = item_begin .. item_end-1 of the order `ord` (one-simulation kernel, balanced split):
// the tail of the CTA's share (the first positions of its last tile, shared with CTA cta + 1), its
// whole tiles, then the head (the last positions of its first tile, shared with CTA cta - 1); the
// tail's partial sums are published as soon as they are written and the head waits for the
// predecessor's. Every tile's positions are still added one at a time in increasing order, so the
// echoes are the same bits as with whole tiles per CTA.
// REAL (packed layouts only): every RF phase is real, the excitation without the d_re products.
// CUT0 (packed tangent layouts only): state N-1 is the first state of its lane (EPGPackedTangent).
template<int K, int G, bool TAN = false, bool PACKED = false, bool BAL = false, bool REAL = false,
         bool CUT0 = false>
__device__ __forceinline__ void fisp_items(const FispArgs& a, const int item_begin, const int item_end,
                                           float2* samples, const FispOrder* ord = nullptr) {
    static_assert(!PACKED || TAN || G == 1, "packed value layouts hold one voxel per lane");
    static_assert(!PACKED || !TAN || K % 2 == 0, "packed tangent layouts hold pairs of states");
    static_assert(!REAL || PACKED, "the real-phase update is a packed-layout form");
    static_assert(!CUT0 || (PACKED && TAN), "the slot-0 truncation is a packed tangent form");
    constexpr int VB = 32 / G;
    const int W = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, sub = lane % G;
    const int P = a.P;
    // a group size that does not divide 32 leaves the last 32 % G lanes without a voxel: they run
    // alongside (on a clamped voxel) and write nothing
    constexpr bool kSpareLanes = (32 % G) != 0;
    const bool writer = sub == 0 && (!kSpareLanes || grp < VB);
    constexpr int CH = kFispChunk<G, TAN>;
    const int plane = W * CH * VB;  // sample planes: value, ∂/∂T1, ∂/∂T2
    constexpr int NQ = TAN ? 3 : 1;

    // item of position u of the order: the identity unless BAL
    auto item_at = [&](int u) { return BAL ? ord->item[u] : u; };
    for (int base = item_begin; base < item_end; base += W) {
        const int nact = min(W, item_end - base);  // warps with an item this round
        if (BAL && base <= ord->wait_u && ord->wait_u < base + nact) {
            // this round reaches the head: its tile's first positions come from CTA cta - 1
            if (threadIdx.x == 0) handoff_wait(ord->handoff + ord->cta - 1, ord->status);
            __syncthreads();
        }
        const int item = item_at(base + min(warp, nact - 1));
        const bool pok = warp < nact;  // warp-uniform
        const int tile = item / P, p = item % P;
        const int vloc = tile * VB + (kSpareLanes ? min(grp, VB - 1) : grp);
        const bool vok = vloc < a.nvoxels;
        const int64_t vcol = a.voxel_begin + (vok ? vloc : a.nvoxels - 1);

        const float T1 = a.params[0 * a.param_stride + vcol];
        const float T2 = a.params[1 * a.param_stride + vcol];
        const float B1 = a.params[2 * a.param_stride + vcol];
        const float B0 = a.params[3 * a.param_stride + vcol];

        // per-voxel relaxation factors (fisp_kernels.cuh:110-144)
        const float R1 = 1.0f / T1, R2 = 1.0f / T2;
        auto rot = [&](float dt) -> float2 {
            if (B0 == 0.0f) return make_float2(1.f, 0.f);
            float s, c;
            sincospif(2.0f * dt * B0, &s, &c);
            return make_float2(c, s);
        };
        const float E1_TR = expf(-a.TR * R1), E2_TR = expf(-a.TR * R2);
        const float2 c_TR = cscale(E2_TR, rot(a.TR));
        const float2 c_TE = cscale(expf(-a.TE * R2), rot(a.TE));
        const float E1_TI = expf(-a.TI * R1);
        const float E1_W = expf(-a.TW * R1);
        const float2 c_W = cscale(expf(-a.TW * R2), rot(a.TW));
        const float beta = 1.0f - E1_TR;
        // tangent factors t/T1², t/T2² of each relaxation interval
        const float s1_TR = a.TR * R1 * R1, s2_TR = a.TR * R2 * R2, s2_TE = a.TE * R2 * R2;
        const float s1_TI = a.TI * R1 * R1, s1_W = a.TW * R1 * R1, s2_W = a.TW * R2 * R2;

        // segments of this round: runs of consecutive warps on the same tile (bit w set where
        // warp w starts one); every thread derives the same mask
        unsigned starts = 0;
        for (int w = 0; w < nact; w++)
            if (w == 0 || item_at(base + w) / P != item_at(base + w - 1) / P) starts |= 1u << w;

        const float4* tab = a.table + int64_t(p) * a.nTR;
        FispState<K, G, TAN, PACKED, CUT0> st;
        st.init(sub);
        for (int rep = a.reps; rep >= 1; rep--) {
            const bool sampled = (rep == 1);
            if (a.inversion) {  // invert, spoil, decay(TI), regrowth (fisp_kernels.cuh:146-152)
                if constexpr (TAN) st.invert_decay(E1_TI, s1_TI, sub);
                else st.invert_decay(E1_TI, sub);
            }
            // the RF table entry of the next TR is loaded one TR ahead, so its latency hides behind
            // a whole TR of state updates (the last load repeats entry nTR-1: in bounds)
            float4 tv_next = __ldg(tab);
            for (int t0 = 0; t0 < a.nTR; t0 += CH) {
                const int nt = min(CH, a.nTR - t0);
                if (pok) {
                    // several TRs per iteration, so the compiler can absorb dephasing shifts in
                    // register renaming instead of moving the state (moves the FMA pipe executes).
                    // Measured on the 224² MR-STAT slice: the first scalar value kernel 63.6 -> 59.6
                    // ms with two; the packed 25-slot value kernel 44.3 ms with two, 42.8 with three,
                    // 42.5 with four, 44.0 / 44.4 / 48.5 with five / six / eight; the two-wide 4 x 8
                    // tangent 380 ms with one, 272.6 with two, 250.0 with four; the scalar 5 x 5
                    // tangent 278.7 with two, 272.4 with four. The scalar value layouts keep two.
#pragma unroll ((PACKED || TAN) ? 4 : 2)
                    for (int j = 0; j < nt; j++) {
                        const int t = t0 + j;
                        const float4 tv = tv_next;
                        tv_next = __ldg(tab + min(t + 1, a.nTR - 1));
                        if constexpr (TAN) {
                            if constexpr (PACKED) {
                                if (t == 0) {
                                    st.template excite<REAL>(make_coefs2<REAL>(tv, B1, make_float2(1.f, 0.f), 1.0f, 0.0f),
                                                             0.0f, 0.0f, sub);
                                } else {
                                    st.shift(sub, a.N);
                                    st.template excite<REAL>(make_coefs2<REAL>(tv, B1, c_TR, E1_TR, beta), s1_TR, s2_TR,
                                                             sub);
                                }
                            } else {
                                if (t == 0) {
                                    st.excite(make_coefs(tv, B1, make_float2(1.f, 0.f), 1.0f, 0.0f), 0.0f, 0.0f, sub);
                                } else {
                                    st.shift(sub, a.N);
                                    st.excite(make_coefs(tv, B1, c_TR, E1_TR, beta), s1_TR, s2_TR, sub);
                                }
                            }
                            if (sampled && writer) {
                                float2* q = samples + (warp * CH + j) * VB + grp;
                                const float2 f = st.f0(0), f2 = st.f0(2);
                                q[0] = cmul(c_TE, f);
                                q[plane] = cmul(c_TE, st.f0(1));
                                q[2 * plane] = cmul(c_TE, make_float2(fmaf(s2_TE, f.x, f2.x), fmaf(s2_TE, f.y, f2.y)));
                            }
                        } else {
                            if constexpr (PACKED) {
                                if (t == 0) {
                                    st.template excite<REAL>(make_coefs2<REAL>(tv, B1, make_float2(1.f, 0.f), 1.0f, 0.0f), sub);
                                } else {
                                    st.shift(sub, a.N);
                                    st.template excite<REAL>(make_coefs2<REAL>(tv, B1, c_TR, E1_TR, beta), sub);
                                }
                            } else {
                                if (t == 0) {
                                    st.excite(make_coefs(tv, B1, make_float2(1.f, 0.f), 1.0f, 0.0f), sub);
                                } else {
                                    st.shift(sub, a.N);
                                    st.excite(make_coefs(tv, B1, c_TR, E1_TR, beta), sub);
                                }
                            }
                            if (sampled && writer) samples[(warp * CH + j) * VB + grp] = cmul(c_TE, st.f0());
                        }
                    }
                }
                if (sampled) {
                    __syncthreads();
                    // per segment, add its positions in increasing order to the tile's partial
                    // sum (the echo rows, unless the segment starts at position 0), then write
                    // the undersampling-expanded rows (fisp_kernels.cuh:246-259)
                    const uint64_t l2_keep = l2_policy_evict_last();
                    // segment bounds, the same for every thread: warps [w0, w1) on one tile
                    for (int w0 = 0; w0 < nact;) {
                        int w1 = w0 + 1;
                        while (w1 < nact && !(starts & (1u << w1))) w1++;
                        const int seg_tile = item_at(base + w0) / P;
                        const bool first = item_at(base + w0) % P == 0;
                        // a partial sum is read again by a later round (or the next CTA): keep it
                        // in L2; the tile's final sum streams out
                        const bool last = item_at(base + w1 - 1) % P == P - 1;
#pragma unroll
                        for (int qn = 0; qn < NQ; qn++) {
                            float2* out = qn == 0 ? a.echo : qn == 1 ? a.dT1 : a.dT2;
                            for (int e = threadIdx.x; e < nt * VB; e += blockDim.x) {
                                const int j = e / VB, gv = e % VB;  // VB is a compile-time power of two or 6
                                const int v = seg_tile * VB + gv;
                                if (v >= a.nvoxels) continue;
                                const float2* col = samples + qn * plane + j * VB + gv;
                                float2* row0 = out + int64_t(t0 + j) * a.uf * a.echo_stride + a.voxel_begin + v;
                                float2 acc = first ? col[w0 * CH * VB] : cadd(__ldcg(row0), col[w0 * CH * VB]);
                                for (int w = w0 + 1; w < w1; w++) acc = cadd(acc, col[w * CH * VB]);
                                for (int q = 0; q < a.uf; q++) {
                                    float2* dst = row0 + int64_t(q) * a.echo_stride;
                                    if (last) __stcs(dst, acc);
                                    else st_l2_hint(dst, acc, l2_keep);
                                }
                            }
                        }
                        w0 = w1;
                    }
                    __syncthreads();
                }
            }
            if (rep > 1) {  // close the repetition: relax to TR, dephase, spoil, wait (fisp_kernels.cuh:195-200)
                if (pok) {
                    if constexpr (TAN) {
                        st.relax(c_TR, E1_TR, s1_TR, s2_TR, sub);
                        st.shift(sub, a.N);
                        if (a.wait_spoil) st.spoil();
                        st.relax(c_W, E1_W, s1_W, s2_W, sub);
                    } else {
                        st.relax(c_TR, E1_TR, sub);
                        st.shift(sub, a.N);
                        if (a.wait_spoil) st.spoil();
                        st.relax(c_W, E1_W, sub);
                    }
                }
            }
        }
        if (BAL && base < ord->publish_u && ord->publish_u <= base + nact) {
            // the tail's partial sums are written (the summation ends with a barrier): hand them over
            if (threadIdx.x == 0) handoff_publish(ord->handoff + ord->cta);
        }
    }
}

// Range of whole tiles of CTA `cta` when `ntiles` tiles are split over `nctas` CTAs (sizes differ
// by at most one tile).
__device__ __forceinline__ int2 cta_tile_range(int ntiles, int cta, int nctas) {
    return make_int2(int(int64_t(ntiles) * cta / nctas), int(int64_t(ntiles) * (cta + 1) / nctas));
}
// One FISP simulation: a persistent grid of CTAs. Without `handoff` each CTA runs a contiguous
// range of whole voxel tiles (cta_tile_range). With `handoff` (per-CTA flags, zero at launch; the
// host asks for it when every CTA's
// share spans at least two tiles, holds at most kFispBalancedItems items and all CTAs are resident
// at once) each CTA runs an equal share of the (tile, position) items, sizes differing by at most
// one item, in the order tail, whole tiles, head (fisp_items). PACKED: the two-wide layout
// EPGPacked<K/2> (one lane per voxel).
// BAL instantiates the balanced form (launched with non-null `handoff`), the others the whole-tile
// form (`handoff` unused), so that each compiles to its own register allocation.
// REAL (packed layouts): the real-phase excitation. The host launches both forms of a packed layout;
// each reads the sequence's phase flag and the one that does not match returns at once (a branch that
// is uniform over the grid, so no host synchronisation picks the form and the pair can be captured).
template<int K, int G, bool PACKED = false, bool BAL = false, bool REAL = false>
__global__ void __launch_bounds__(256, 1) fisp_epg_kernel(FispArgs a, int ntiles, int* handoff, unsigned int* status) {
    extern __shared__ float2 samples[];  // [W][32][VB]
    if (a.skip != nullptr && *a.skip != 0) return;  // uniform over the grid
    if constexpr (PACKED) {
        if (fisp_real_phases(a) != REAL) return;
    }
    if constexpr (BAL) {
        __shared__ FispOrder ord;
        const int64_t total = int64_t(ntiles) * a.P;
        const int i0 = int(total * blockIdx.x / gridDim.x), i1 = int(total * (blockIdx.x + 1) / gridDim.x);
        const int P = a.P, n = i1 - i0;
        const int h_end = min(i1, (i0 + P - 1) / P * P);  // end of the head: the first tile's last positions
        const int t_start = max(h_end, i1 / P * P);        // start of the tail: the last tile's first positions
        const int L0 = i1 - t_start, L01 = L0 + (t_start - h_end);
        for (int u = threadIdx.x; u < n; u += blockDim.x)
            ord.item[u] = u < L0 ? t_start + u : (u < L01 ? h_end + (u - L0) : i0 + (u - L01));
        if (threadIdx.x == 0) {
            ord.wait_u = i0 % P != 0 ? L01 : n;      // n: no head, nothing to wait for
            ord.publish_u = i1 % P != 0 ? L0 : -1;   // -1: no tail, nothing to hand over
            ord.cta = blockIdx.x;
            ord.handoff = handoff;
            ord.status = status;
        }
        __syncthreads();
        fisp_items<K, G, false, PACKED, true, REAL>(a, 0, n, samples, &ord);
    } else {
        (void)handoff;
        (void)status;
        const int2 r = cta_tile_range(ntiles, blockIdx.x, gridDim.x);
        fisp_items<K, G, false, PACKED, false, REAL>(a, r.x * a.P, r.y * a.P, samples);
    }
}

// Persistent work-queue kernel for a batch of FISP simulations sharing one layout and W:
// each CTA takes (job, tile) items from `items` in order through an atomic counter until the
// queue is empty. Items are ordered longest job first, so the last wave is short.
// REAL (packed layouts): every job's phases are real, the real-phase excitation.
template<int K, int G, bool PACKED = false, bool REAL = false>
__global__ void __launch_bounds__(256, 1) fisp_queue_kernel(const FispArgs* __restrict__ jobs,
                                                            const int2* __restrict__ items, int nitems,
                                                            int* __restrict__ head) {
    extern __shared__ float2 samples[];
    __shared__ FispArgs job;
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(head, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const int2 w = items[it];
        if (threadIdx.x == 0) job = jobs[w.x];
        __syncthreads();
        // tiles w.y .. of the job, as many as the batch put in one item
        const int tiles = (job.nvoxels + 32 / G - 1) / (32 / G);
        const int t_end = min(w.y + fisp_queue_tiles_per_item(job.P, blockDim.x >> 5), tiles);
        fisp_items<K, G, false, PACKED, false, REAL>(job, w.y * job.P, t_end * job.P, samples);
        __syncthreads();  // job and s_item are rewritten by the next item
    }
}

// One FISP simulation with its T1 and T2 tangents: value, ∂/∂T1, ∂/∂T2 into a.echo, a.dT1, a.dT2.
// PACKED: the two-wide state EPGPackedTangent; REAL its real-phase form, launched beside the
// general form (the one that does not match the sequence returns at once); CUT0 its form for
// (N-1) % K == 0, which the host launches for those N.
template<int K, int G, bool PACKED = false, bool REAL = false, bool CUT0 = false>
__global__ void __launch_bounds__(256, 1) fisp_tangent_kernel(FispArgs a, int ntiles) {
    extern __shared__ float2 samples[];  // [3][W][chunk][VB]
    if constexpr (PACKED) {
        if (fisp_real_phases(a) != REAL) return;
    }
    const int2 r = cta_tile_range(ntiles, blockIdx.x, gridDim.x);
    fisp_items<K, G, true, PACKED, false, REAL, CUT0>(a, r.x * a.P, r.y * a.P, samples);
}

// Work-queue form of fisp_tangent_kernel for batches (same items and order as fisp_queue_kernel;
// REAL: every job's phases are real; CUT0: every job has (N-1) % K == 0).
template<int K, int G, bool PACKED = false, bool REAL = false, bool CUT0 = false>
__global__ void __launch_bounds__(256, 1) fisp_tangent_queue_kernel(const FispArgs* __restrict__ jobs,
                                                                    const int2* __restrict__ items, int nitems,
                                                                    int* __restrict__ head) {
    extern __shared__ float2 samples[];
    __shared__ FispArgs job;
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(head, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const int2 w = items[it];
        if (threadIdx.x == 0) job = jobs[w.x];
        __syncthreads();
        const int tiles = (job.nvoxels + 32 / G - 1) / (32 / G);
        const int t_end = min(w.y + fisp_queue_tiles_per_item(job.P, blockDim.x >> 5), tiles);
        fisp_items<K, G, true, PACKED, false, REAL, CUT0>(job, w.y * job.P, t_end * job.P, samples);
        __syncthreads();
    }
}

}  // namespace kernels

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------

namespace {

using FispKernel = void (*)(kernels::FispArgs, int);
using FispValueKernel = void (*)(kernels::FispArgs, int, int*, unsigned int*);
using FispQueueKernel = void (*)(const kernels::FispArgs*, const int2*, int, int*);

struct FispConfig {
    int K, G;
    bool packed;  // EPGPacked<K/2>: two states per two-wide instruction
    FispValueKernel fn;
    FispQueueKernel queue;
    FispValueKernel balanced;  // the balanced item split (packed layouts), else null
    // packed layouts: the real-phase forms of fn and balanced (launched beside them) and of queue
    // (launched instead of it for groups of real-phase jobs), else null
    FispValueKernel fn_real;
    FispValueKernel balanced_real;
    FispQueueKernel queue_real;
};

// Instantiated layouts: (states per lane K, lanes per voxel/position G). Coverage K·G ≥ N.
// The packed one-lane layouts come last, so the indices of the others (which a tuning table
// names) keep their meaning.
#define COMPAS_FISP(K, G) \
    {K, G, false, kernels::fisp_epg_kernel<K, G>, kernels::fisp_queue_kernel<K, G>, nullptr, nullptr, nullptr, nullptr}
#define COMPAS_FISP_PACKED(K)                                                                         \
    {K, 1, true, kernels::fisp_epg_kernel<K, 1, true>, kernels::fisp_queue_kernel<K, 1, true>,      \
     kernels::fisp_epg_kernel<K, 1, true, true>, kernels::fisp_epg_kernel<K, 1, true, false, true>,  \
     kernels::fisp_epg_kernel<K, 1, true, true, true>, kernels::fisp_queue_kernel<K, 1, true, true>}
const FispConfig kFispConfigs[] = {
    COMPAS_FISP(1, 1), COMPAS_FISP(2, 1), COMPAS_FISP(4, 1), COMPAS_FISP(6, 1), COMPAS_FISP(8, 1),
    COMPAS_FISP(12, 1), COMPAS_FISP(16, 1), COMPAS_FISP(20, 1), COMPAS_FISP(25, 1),
    COMPAS_FISP(2, 4), COMPAS_FISP(4, 2), COMPAS_FISP(4, 4), COMPAS_FISP(4, 8), COMPAS_FISP(7, 4),
    COMPAS_FISP(13, 2), COMPAS_FISP(8, 4), COMPAS_FISP(8, 8), COMPAS_FISP(8, 16), COMPAS_FISP(4, 32),
    COMPAS_FISP_PACKED(4), COMPAS_FISP_PACKED(8), COMPAS_FISP_PACKED(12), COMPAS_FISP_PACKED(16),
    COMPAS_FISP_PACKED(20), COMPAS_FISP_PACKED(26), COMPAS_FISP_PACKED(25),
};
#undef COMPAS_FISP
#undef COMPAS_FISP_PACKED

// Tangent layouts: three state vectors per (voxel, position), so at most 8 states per lane
// (8 × 18 floats); the 25-state MR-STAT case splits over 5 lanes of 5 states (6 groups per warp,
// 2 lanes idle) or 4 lanes of 7.
struct FispTangentConfig {
    int K, G;
    FispKernel fn;
    FispQueueKernel queue;
    bool packed;  // EPGPackedTangent<K/2, G>: two states per two-wide instruction
    // packed layouts: the real-phase forms of fn (launched beside it) and queue (for groups of
    // real-phase jobs), else null
    FispKernel fn_real;
    FispQueueKernel queue_real;
    // packed layouts: the four kernels above in their form for (N-1) % K == 0 (state N-1 is the
    // first state of its lane), else null
    FispKernel fn_cut0, fn_real_cut0;
    FispQueueKernel queue_cut0, queue_real_cut0;
};
#define COMPAS_FISP_TANGENT(K, G)                                                                              \
    {K, G, kernels::fisp_tangent_kernel<K, G>, kernels::fisp_tangent_queue_kernel<K, G>, false, nullptr, nullptr, \
     nullptr, nullptr, nullptr, nullptr}
#define COMPAS_FISP_TANGENT_PACKED(K, G)                                                                     \
    {K, G, kernels::fisp_tangent_kernel<K, G, true>, kernels::fisp_tangent_queue_kernel<K, G, true>, true, \
     kernels::fisp_tangent_kernel<K, G, true, true>, kernels::fisp_tangent_queue_kernel<K, G, true, true>, \
     kernels::fisp_tangent_kernel<K, G, true, false, true>, kernels::fisp_tangent_kernel<K, G, true, true, true>, \
     kernels::fisp_tangent_queue_kernel<K, G, true, false, true>, kernels::fisp_tangent_queue_kernel<K, G, true, true, true>}
// the packed layouts come last, so the indices of the others keep their meaning
const FispTangentConfig kFispTangentConfigs[] = {
    COMPAS_FISP_TANGENT(1, 1), COMPAS_FISP_TANGENT(2, 1), COMPAS_FISP_TANGENT(4, 1), COMPAS_FISP_TANGENT(8, 1),
    COMPAS_FISP_TANGENT(2, 4), COMPAS_FISP_TANGENT(4, 4), COMPAS_FISP_TANGENT(5, 5), COMPAS_FISP_TANGENT(7, 4),
    COMPAS_FISP_TANGENT(8, 4),
    COMPAS_FISP_TANGENT(4, 8), COMPAS_FISP_TANGENT(8, 8), COMPAS_FISP_TANGENT(8, 16),
    COMPAS_FISP_TANGENT_PACKED(8, 1), COMPAS_FISP_TANGENT_PACKED(4, 4), COMPAS_FISP_TANGENT_PACKED(8, 4),
    COMPAS_FISP_TANGENT_PACKED(4, 8),
};
#undef COMPAS_FISP_TANGENT
#undef COMPAS_FISP_TANGENT_PACKED
constexpr int kFispTangentConfigCount = int(sizeof(kFispTangentConfigs) / sizeof(kFispTangentConfigs[0]));

}  // namespace

int fisp_config_count() {
    return int(sizeof(kFispConfigs) / sizeof(kFispConfigs[0]));
}

bool fisp_config_info(int index, int* K, int* G) {
    if (index < 0 || index >= fisp_config_count()) return false;
    *K = kFispConfigs[index].K;
    *G = kFispConfigs[index].G;
    return true;
}

bool fisp_config_packed(int index) {
    return index >= 0 && index < fisp_config_count() && kFispConfigs[index].packed;
}

// Default layout choice for `N` states (from layout and autotuner timings on B200):
//  * many (voxel, position) pairs: all states of a voxel in one lane (G = 1, K ≥ N) — no shuffles;
//    25 states × 35 positions at 25600 voxels: 38.6 ms vs 51 ms for the best split layout;
//  * few pairs (e.g. 4096 voxels × 1 position): split the states over 4 lanes to get 4× more warps
//    (8 states: K2·G4 0.155 ms vs 0.205 ms for K8·G1);
//  * N > 25: the smallest covering split layout.
// The autotuner (tuning.cu) may override it per shape class.
FispLaunch fisp_default_launch(int N, int64_t nvoxels, int P) {
    const int64_t pairs = nvoxels * P;
    const bool wide = pairs >= 148LL * 32 * 8;
    int best = -1;
    auto waste = [&](int i) { return kFispConfigs[i].K * kFispConfigs[i].G - N; };
    // FMA-pipe time of the state update per lane and TR, in units of one state's 26 one-wide
    // operations: a two-wide instruction takes the pipe twice as long, so a pair of states costs two
    // units, an unpaired state one, and a packed layout K/2 units for K states
    auto cost = [&](int i) {
        return kFispConfigs[i].packed ? 0.5 * kFispConfigs[i].K : double(kFispConfigs[i].K);
    };
    for (int i = 0; i < fisp_config_count(); i++) {
        const auto& c = kFispConfigs[i];
        if (c.K * c.G < N) continue;
        bool preferred;
        if (N <= 26 && wide) preferred = (c.G == 1);
        else if (N <= 32 && !wide) preferred = (c.G == 4);
        else preferred = true;
        if (!preferred) continue;
        if (best < 0) {
            best = i;
        } else if (c.G == 1 && kFispConfigs[best].G == 1) {
            // one lane per voxel: the fewest issue slots, then the least padding (scalar on ties)
            if (cost(i) < cost(best) || (cost(i) == cost(best) && waste(i) < waste(best))) best = i;
        } else if (waste(i) < waste(best) || (waste(i) == waste(best) && c.G < kFispConfigs[best].G)) {
            best = i;
        }
    }
    if (best < 0) {  // nothing matched the preference: the covering layout with the least waste
        for (int i = 0; i < fisp_config_count(); i++)
            if (kFispConfigs[i].K * kFispConfigs[i].G >= N && (best < 0 || waste(i) < waste(best))) best = i;
    }
    // warps (slice positions in flight per voxel tile), from the autotuner's B200 timings at
    // 35 positions: 8 for 12+ states in one lane (25 states, 50176 voxels: 18.0 ms vs 19.8 ms
    // with 7), 6 for fewer states in one lane, 4 for states split over lanes; never more than P
    FispLaunch L {best, 1};
    const auto& c = kFispConfigs[best];
    const int w = c.G == 1 ? (c.K >= 12 ? 8 : 6) : 4;
    L.warps = std::max(1, std::min(w, P));
    return L;
}

const Array<float, 3>& fisp_excite_table(const CompasContext& ctx, const FISPSequence& seq) {
    auto& cache = *seq.cache;
    std::lock_guard<std::mutex> lock(cache.mutex);
    if (!cache.table || cache.key_rf != seq.RF_train.data() || cache.key_sp != seq.sliceprofiles.data()) {
        int nTR = int(seq.RF_train.size());
        int P = int(seq.sliceprofiles.size(0));
        COMPAS_CHECK(int(seq.sliceprofiles.size(1)) == nTR);
        // rows 0..P-1: the entries; entry P·nTR (the start of row P): the flag of a complex phase
        // (fisp_table_kernel). At least one entry per row, so the flag exists when nTR = 0.
        auto tab = std::make_shared<Array<float, 3>>(std::array<int64_t, 3> {P + 1, std::max(nTR, 1), 4}, ctx.device(),
                                                     ctx.stream());
        DeviceGuard guard(ctx.device());
        int n = nTR * P;
        COMPAS_CUDA_CHECK(cudaMemsetAsync(tab->data() + int64_t(n) * 4, 0, sizeof(float4), ctx.stream()));
        if (n > 0) {
            kernels::fisp_table_kernel<<<div_ceil(n, 256), 256, 0, ctx.stream()>>>(
                reinterpret_cast<const float2*>(seq.RF_train.data()),
                reinterpret_cast<const float2*>(seq.sliceprofiles.data()), nTR, P,
                reinterpret_cast<float4*>(tab->data()));
            check_launch("fisp_table_kernel");
        }
        cache.table = tab;
        cache.key_rf = seq.RF_train.data();
        cache.key_sp = seq.sliceprofiles.data();
        cache.real_phases = -1;
    }
    return *cache.table;
}

bool fisp_sequence_real_phases(const CompasContext& ctx, const FISPSequence& seq) {
    const auto& tab = fisp_excite_table(ctx, seq);
    auto& cache = *seq.cache;
    std::lock_guard<std::mutex> lock(cache.mutex);
    if (cache.real_phases < 0) {
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        COMPAS_CUDA_CHECK(cudaStreamIsCapturing(ctx.stream(), &capture));
        if (capture != cudaStreamCaptureStatusNone) return false;  // the general form is right for every sequence
        const int64_t flag_at = int64_t(seq.sliceprofiles.size(0)) * seq.RF_train.size() * 4;
        float flag = 1.0f;
        DeviceGuard guard(ctx.device());
        COMPAS_CUDA_CHECK(cudaMemcpyAsync(&flag, tab.data() + flag_at, sizeof(float), cudaMemcpyDeviceToHost,
                                          ctx.stream()));
        COMPAS_CUDA_CHECK(cudaStreamSynchronize(ctx.stream()));
        cache.real_phases = flag == 0.0f ? 1 : 0;
    }
    return cache.real_phases == 1;
}

kernels::FispArgs fisp_args(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                            const FISPSequence& seq, cfloat* echo, int64_t echo_stride) {
    const int nTR = int(seq.RF_train.size());
    const int P = int(seq.sliceprofiles.size(0));
    const int N = seq.max_state;
    if (N < 1 || N > 128) COMPAS_ERROR("max_state must be in [1, 128]");
    COMPAS_CHECK(seq.undersampling_factor >= 1 && seq.repetitions >= 1);
    COMPAS_CHECK(P >= 1 && int(seq.sliceprofiles.size(1)) == nTR);
    const auto& tab = fisp_excite_table(ctx, seq);

    kernels::FispArgs a;
    a.params = params.data.data();
    a.param_stride = params.data.size(1);
    a.voxel_begin = voxel_begin;
    a.nvoxels = nvoxels;
    a.table = reinterpret_cast<const float4*>(tab.data());
    a.nTR = nTR;
    a.P = P;
    a.N = N;
    a.uf = seq.undersampling_factor;
    a.reps = seq.repetitions;
    a.inversion = seq.inversion_prepulse ? 1 : 0;
    a.wait_spoil = seq.wait_spoiling ? 1 : 0;
    a.TR = seq.TR;
    a.TE = seq.TE;
    a.TW = seq.TW;
    a.TI = seq.TI;
    a.echo = reinterpret_cast<float2*>(echo);
    a.echo_stride = echo_stride;
    a.dT1 = a.dT2 = nullptr;
    a.skip = nullptr;
    return a;
}

namespace {

const FispConfig& checked_config(FispLaunch L, int N) {
    COMPAS_CHECK(L.config >= 0 && L.config < fisp_config_count());
    const auto& cfg = kFispConfigs[L.config];
    COMPAS_CHECK(cfg.K * cfg.G >= N);
    return cfg;
}

// samples of one chunk: [W][chunk][32 / G] complex per plane (kernels::kFispChunk)
size_t fisp_smem_bytes(const FispConfig& cfg, int W) {
    // [W][chunk][32 / G] samples: 64 TRs for one-lane layouts (≤ 128 KB at W ≤ 8), 32 for split ones
    const int chunk = cfg.G == 1 ? kernels::kFispChunk<1, false> : kernels::kFispChunk<2, false>;
    return size_t(W) * chunk * (32 / cfg.G) * sizeof(float2);
}

size_t fisp_tangent_smem_bytes(int G, int W) {
    return 3 * size_t(W) * (G == 1 ? 32 : 64) * (32 / G) * sizeof(float2);  // ≤ 192 KB
}

// CTAs of `fn` resident on the device at once with this block size and dynamic shared memory:
// the grid of the persistent one-simulation kernels
int resident_ctas(const void* fn, int threads, size_t smem, int device) {
    int per_sm = 1, sms = 148;
    COMPAS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    COMPAS_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    return std::max(1, per_sm) * sms;
}

// Opt in to `smem` bytes of dynamic shared memory. Without the attribute a launch may use at most
// 48 KB minus the kernel's static shared memory (the work-queue kernels keep their job's argument
// block there), so the attribute is set from 40 KB on.
void allow_smem(const void* fn, size_t smem) {
    if (smem > 40 * 1024)
        COMPAS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
}

}  // namespace

int fisp_tile_voxels(FispLaunch L) {
    COMPAS_CHECK(L.config >= 0 && L.config < fisp_config_count());
    return 32 / kFispConfigs[L.config].G;
}

void launch_fisp(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                 const FISPSequence& seq, cfloat* echo, int64_t echo_stride, FispLaunch L, const int* skip,
                 bool balance, int* handoff, int handoff_capacity) {
    const int nTR = int(seq.RF_train.size());
    const int P = int(seq.sliceprofiles.size(0));
    const int N = seq.max_state;
    if (nvoxels <= 0 || nTR <= 0) {
        (void)fisp_args(ctx, params, voxel_begin, nvoxels, seq, echo, echo_stride);  // validates
        return;
    }
    if (L.config < 0) L = fisp_default_launch(N, nvoxels, P);
    kernels::FispArgs a = fisp_args(ctx, params, voxel_begin, nvoxels, seq, echo, echo_stride);
    a.skip = skip;
    const auto& cfg = checked_config(L, N);
    const int VB = 32 / cfg.G;
    const int W = std::max(1, std::min(L.warps, 8));
    const int ntiles = div_ceil(nvoxels, VB);
    const size_t smem = fisp_smem_bytes(cfg, W);
    DeviceGuard guard(ctx.device());
    allow_smem(reinterpret_cast<const void*>(cfg.fn), smem);
    int resident = resident_ctas(reinterpret_cast<const void*>(cfg.fn), 32 * W, smem, ctx.device());
    if (cfg.fn_real != nullptr) {
        allow_smem(reinterpret_cast<const void*>(cfg.fn_real), smem);
        resident = std::min(resident, resident_ctas(reinterpret_cast<const void*>(cfg.fn_real), 32 * W, smem, ctx.device()));
    }
    const int grid = std::min(ntiles, resident);
    // The balanced split needs every CTA's share to span at least two tiles (so a CTA waits only on
    // its predecessor's first part, never on a chain), at most kFispBalancedItems items, and all
    // CTAs resident at once (the grid is at most one resident wave). It saves the idle tail of the
    // CTAs with one more whole tile: 1568 tiles x 35 positions on 148 CTAs of 8 warps run 47 rounds
    // instead of 49.
    const int64_t per_cta = (int64_t(ntiles) * P + grid - 1) / grid;
    bool balanced = balance && cfg.balanced != nullptr && grid > 1 && int64_t(ntiles) >= 2 * int64_t(grid) &&
                    per_cta <= kernels::kFispBalancedItems && (handoff == nullptr || grid <= handoff_capacity);
    if (balanced) {
        int sms = 148;
        COMPAS_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device()));
        for (FispValueKernel k : {cfg.balanced, cfg.balanced_real}) {
            if (k == nullptr) continue;
            const void* bfn = reinterpret_cast<const void*>(k);
            allow_smem(bfn, smem);
            int per_sm = 0;
            COMPAS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfn, 32 * W, smem));
            balanced = balanced && int64_t(per_sm) * sms >= grid;  // every CTA resident at once
        }
    }
    std::optional<Array<int, 1>> flags;
    if (balanced) {
        if (handoff == nullptr) {
            flags.emplace(std::array<int64_t, 1> {grid}, ctx.device(), ctx.stream());
            handoff = flags->data();
        }
        COMPAS_CUDA_CHECK(cudaMemsetAsync(handoff, 0, sizeof(int) * size_t(grid), ctx.stream()));
        // the form that does not match the sequence's phases returns without touching the flags
        cfg.balanced<<<grid, 32 * W, smem, ctx.stream()>>>(a, ntiles, handoff, ctx.status_word());
        check_launch("fisp_epg_kernel");
        if (cfg.balanced_real != nullptr) {
            cfg.balanced_real<<<grid, 32 * W, smem, ctx.stream()>>>(a, ntiles, handoff, ctx.status_word());
            check_launch("fisp_epg_kernel (real phases)");
        }
    } else {
        cfg.fn<<<grid, 32 * W, smem, ctx.stream()>>>(a, ntiles, nullptr, nullptr);
        check_launch("fisp_epg_kernel");
        if (cfg.fn_real != nullptr) {
            cfg.fn_real<<<grid, 32 * W, smem, ctx.stream()>>>(a, ntiles, nullptr, nullptr);
            check_launch("fisp_epg_kernel (real phases)");
        }
    }
}

int fisp_tangent_config_count() {
    return kFispTangentConfigCount;
}

bool fisp_tangent_config_info(int index, int* K, int* G) {
    if (index < 0 || index >= kFispTangentConfigCount) return false;
    *K = kFispTangentConfigs[index].K;
    *G = kFispTangentConfigs[index].G;
    return true;
}

bool fisp_tangent_config_packed(int index) {
    return index >= 0 && index < kFispTangentConfigCount && kFispTangentConfigs[index].packed;
}

// Tangent layout for N states: with many (voxel, position) pairs and 25-32 states the two-wide
// 4 x 8 layout, with N ≤ 8 all states in one lane; otherwise the covering layout with the least
// padding, fewer lanes on ties. The warps
// per CTA are the value kernel's (tuned_fisp_launch): 8 for the MR-STAT slice, where 7 and 5
// measured 9 % and 54 % slower (one CTA of 255-register threads per SM).
FispLaunch fisp_tangent_default_launch(int N, int64_t nvoxels, int P) {
    const bool wide = nvoxels * P >= 148LL * 32 * 8;
    int best = -1;
    // 25 to 32 states on many (voxel, position) pairs: the two-wide layout of 4 lanes x 8 states
    // (MR-STAT slice: 272.8 ms against 279.6 ms for the scalar 5 x 5 and 287 ms for 4 x 7; 96² voxels:
    // 50.1 against 54.1 ms), although its 32 slots hold up to 7 padding states
    if (wide && N > 24 && N <= 32) {
        for (int i = 0; i < kFispTangentConfigCount; i++) {
            const auto& c = kFispTangentConfigs[i];
            if (c.packed && c.K == 8 && c.G == 4) return FispLaunch {i, tuned_fisp_launch(N, nvoxels, P).warps};
        }
    }
    for (int i = 0; i < kFispTangentConfigCount; i++) {
        const auto& c = kFispTangentConfigs[i];
        if (c.K * c.G < N || (c.G == 1) != (wide && N <= 8)) continue;
        const auto& b = kFispTangentConfigs[best < 0 ? 0 : best];
        if (best < 0 || c.K * c.G < b.K * b.G) best = i;
    }
    if (best < 0)
        for (int i = 0; i < kFispTangentConfigCount; i++)
            if (kFispTangentConfigs[i].K * kFispTangentConfigs[i].G >= N) {
                best = i;
                break;
            }
    return FispLaunch {best, tuned_fisp_launch(N, nvoxels, P).warps};
}

void launch_fisp_tangent(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                         const FISPSequence& seq, cfloat* echo, cfloat* dT1, cfloat* dT2, int64_t echo_stride,
                         FispLaunch L) {
    const int nTR = int(seq.RF_train.size());
    const int P = int(seq.sliceprofiles.size(0));
    const int N = seq.max_state;
    kernels::FispArgs a = fisp_args(ctx, params, voxel_begin, nvoxels, seq, echo, echo_stride);  // validates
    if (nvoxels <= 0 || nTR <= 0) return;
    if (L.config < 0) L = fisp_tangent_default_launch(N, nvoxels, P);
    COMPAS_CHECK(L.config >= 0 && L.config < kFispTangentConfigCount);
    const auto& cfg = kFispTangentConfigs[L.config];
    COMPAS_CHECK(cfg.K * cfg.G >= N);
    a.dT1 = reinterpret_cast<float2*>(dT1);
    a.dT2 = reinterpret_cast<float2*>(dT2);
    const int VB = 32 / cfg.G;
    const int W = std::max(1, std::min(L.warps, 8));
    const int ntiles = div_ceil(nvoxels, VB);
    const size_t smem = fisp_tangent_smem_bytes(cfg.G, W);
    const bool cut0 = cfg.fn_cut0 != nullptr && (N - 1) % cfg.K == 0;
    const FispKernel fn = cut0 ? cfg.fn_cut0 : cfg.fn;
    const FispKernel fn_real = cut0 ? cfg.fn_real_cut0 : cfg.fn_real;
    DeviceGuard guard(ctx.device());
    allow_smem(reinterpret_cast<const void*>(fn), smem);
    int resident = resident_ctas(reinterpret_cast<const void*>(fn), 32 * W, smem, ctx.device());
    if (fn_real != nullptr) {
        allow_smem(reinterpret_cast<const void*>(fn_real), smem);
        resident = std::min(resident, resident_ctas(reinterpret_cast<const void*>(fn_real), 32 * W, smem, ctx.device()));
    }
    const int grid = std::min(ntiles, resident);
    fn<<<grid, 32 * W, smem, ctx.stream()>>>(a, ntiles);
    check_launch("fisp_tangent_kernel");
    if (fn_real != nullptr) {  // the form that does not match the sequence's phases returns at once
        fn_real<<<grid, 32 * W, smem, ctx.stream()>>>(a, ntiles);
        check_launch("fisp_tangent_kernel (real phases)");
    }
}

int fisp_tangent_tile_voxels(FispLaunch L) {
    COMPAS_CHECK(L.config >= 0 && L.config < kFispTangentConfigCount);
    return 32 / kFispTangentConfigs[L.config].G;
}

void launch_fisp_tangent_queue(cudaStream_t stream, int device, FispLaunch L, int max_state,
                               const kernels::FispArgs* jobs, const int2* items, int nitems, int* head, bool real) {
    if (nitems <= 0) return;
    COMPAS_CHECK(L.config >= 0 && L.config < kFispTangentConfigCount);
    const auto& cfg = kFispTangentConfigs[L.config];
    COMPAS_CHECK(cfg.K * cfg.G >= max_state);
    // every job of the launch has max_state states (the batch groups jobs by it), so the
    // slot-0 truncation form holds for all of them or for none
    const bool cut0 = cfg.queue_cut0 != nullptr && (max_state - 1) % cfg.K == 0;
    const bool use_real = real && cfg.queue_real != nullptr;
    const FispQueueKernel fn = use_real ? (cut0 ? cfg.queue_real_cut0 : cfg.queue_real) : (cut0 ? cfg.queue_cut0 : cfg.queue);
    const int W = std::max(1, std::min(L.warps, 8));
    const size_t smem = fisp_tangent_smem_bytes(cfg.G, W);
    DeviceGuard guard(device);
    allow_smem(reinterpret_cast<const void*>(fn), smem);
    int per_sm = 1, sms = 148;
    COMPAS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * W, smem));
    COMPAS_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = std::max(1, std::min(nitems, std::max(1, per_sm) * sms));
    fn<<<grid, 32 * W, smem, stream>>>(jobs, items, nitems, head);
    check_launch("fisp_tangent_queue_kernel");
}

void launch_fisp_queue(cudaStream_t stream, int device, FispLaunch L, int max_state, const kernels::FispArgs* jobs,
                       const int2* items, int nitems, int* head, bool real) {
    if (nitems <= 0) return;
    const auto& cfg = checked_config(L, max_state);
    const FispQueueKernel fn = real && cfg.queue_real != nullptr ? cfg.queue_real : cfg.queue;
    const int W = std::max(1, std::min(L.warps, 8));
    const size_t smem = fisp_smem_bytes(cfg, W);
    DeviceGuard guard(device);
    allow_smem(reinterpret_cast<const void*>(fn), smem);
    int per_sm = 1, sms = 148;
    COMPAS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * W, smem));
    COMPAS_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = std::max(1, std::min(nitems, std::max(1, per_sm) * sms));
    fn<<<grid, 32 * W, smem, stream>>>(jobs, items, nitems, head);
    check_launch("fisp_queue_kernel");
}

Array<cfloat, 2> simulate_magnetization(const CompasContext& context, TissueParameters parameters,
                                        FISPSequence sequence) {
    const int nTR = int(sequence.RF_train.size());
    const int nreadouts = nTR * sequence.undersampling_factor;
    const int nvoxels = parameters.nvoxels;
    COMPAS_CHECK(sequence.undersampling_factor >= 1);
    Array<cfloat, 2> echos({nreadouts, nvoxels}, context.device(), context.stream());
    launch_fisp(context, parameters, 0, nvoxels, sequence, echos.data(), nvoxels,
                tuned_fisp_launch(sequence.max_state, nvoxels, int(sequence.sliceprofiles.size(0))), nullptr, true);
    return echos;
}

MagnetizationTangents simulate_magnetization_tangents(const CompasContext& context, TissueParameters parameters,
                                                      FISPSequence sequence) {
    COMPAS_CHECK(sequence.undersampling_factor >= 1);
    const int nreadouts = int(sequence.RF_train.size()) * sequence.undersampling_factor;
    const int nvoxels = parameters.nvoxels;
    MagnetizationTangents out {{{nreadouts, nvoxels}, context.device(), context.stream()},
                               {{nreadouts, nvoxels}, context.device(), context.stream()},
                               {{nreadouts, nvoxels}, context.device(), context.stream()}};
    launch_fisp_tangent(context, parameters, 0, nvoxels, sequence, out.echos.data(), out.dT1.data(), out.dT2.data(),
                        nvoxels, tuned_fisp_tangent_launch(sequence.max_state, nvoxels,
                                                           int(sequence.sliceprofiles.size(0))));
    return out;
}

}  // namespace compas
