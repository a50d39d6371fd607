// pssfp.cu — pSSFP isochromat (Bloch) simulation on sm_100a.
//
// Restates src/simulate/pssfp_kernels.cuh:14-129 and src/operators/isochromat.cuh:9-128:
// per (voxel, z) an isochromat is inverted (cos πB1), relaxed, given an α/2 pulse, and then
// for each TR excited by n_RF hard-pulse Rodrigues rotations (each followed by relaxation),
// precessed, sampled (Σ_z m_x + i m_y) and precessed again.
//
// B200 layout: a thread owns ZT isochromats of one voxel and GZ lanes (a power of two)
// cover the z positions; the per-TR sum over z is a register sum plus an xor-shuffle tree.
// The RF rotation axis (Re, -Im)(RF[t]·γΔtRF[i])·B1 is the same for every z, so the
// products RF[t]·γΔtRF[i] are tabulated once per sequence; the z-dependent axis component
// and the precession angles are constant over the TR loop and hoisted out of it (the
// precession sin/cos is evaluated once per z instead of twice per TR). The rotation uses
// the unnormalised-axis Rodrigues form
//     m' = cos θ·m + (sin θ/θ)·(a×m) + ((1-cos θ)/θ²)·(a·m)·a,   θ² = a·a,
// whose coefficients sin θ/θ and (1-cos θ)/θ² are cubic Taylor polynomials in θ² (coefficients
// 1/n!) for θ ≤ 0.5 rad, accurate to 1.1e-8 relative, and cos θ = 1 - θ²·(1-cos θ)/θ², so the hot loop runs on
// the FMA pipe; larger angles use sqrt/sincos. The relaxation after each RF sample is folded into
// the rotation (E2 scales its coefficients, E1 enters as E1/E2 on the longitudinal result).
// The two-wide layouts (pssfp_tile_packed) hold the isochromats of a lane in pairs and run every
// operation as one sm_100 two-wide FP32 instruction per pair, which halves the issue slots of the
// (issue-bound) scalar update; they are the default for 3 or more z positions.
#include "common.cuh"
#include "compas/compas.h"
#include "job_args.cuh"
#include "kernels.h"

namespace compas {
namespace kernels {

// zap[0][i] = -(RF[0]/2)·γΔtRF[i] (the α/2 pulse), zap[1+t][i] = RF[t]·γΔtRF[i]
// zap[row][i] for rows 0..nTR, and after them, at entry (nTR + 1)·nRF, the flag of a complex RF
// axis: x = 1 when some entry has Im zap ≠ 0, else 0 (zeroed before the launch)
__global__ void pssfp_table_kernel(const float2* __restrict__ rf, int nTR, const float2* __restrict__ g, int nRF,
                                   float2* __restrict__ zap) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (nTR + 1) * nRF) return;
    int row = idx / nRF, i = idx % nRF;
    float2 th = row == 0 ? make_float2(-rf[0].x / 2.0f, -rf[0].y / 2.0f) : rf[row - 1];
    const float2 v = cmul(th, g[i]);
    zap[idx] = v;
    if (v.y != 0.0f) zap[int64_t(nTR + 1) * nRF].x = 1.0f;  // every writer stores the same value
}

// True when every RF sample of the sequence is real (Im zap = 0: a real RF train, as with 0-π phase
// cycling, and a real waveform). The rotation axis then has a_y = ±0 and the packed update leaves
// out its products (pssfp_tile_packed<…, REAL>).
__device__ __forceinline__ bool pssfp_real_rf(const PssfpArgs& a) {
    return __ldg(&a.zap[int64_t(a.nTR + 1) * a.nRF].x) == 0.0f;
}


struct Iso {
    float x, y, z;
};

// Per-voxel constants of rotate_relax: the Taylor coefficients of sin θ/θ and (1-cos θ)/θ² times
// E2 (magnitudes E2/(2n+1)! and E2/(2n+2)!; the series alternate in θ² and are evaluated in
// y = -θ², where every term is positive), E2 itself, E1/E2 and 1 - E1.
struct RotRelax {
    float s0, s1, s2, s3, h0, h1, h2, h3, E2, r, oneE1;
};

__device__ __forceinline__ RotRelax make_rot_relax(float E1, float E2) {
    RotRelax k;
    k.s0 = E2;
    k.s1 = E2 * (1.0f / 6.0f);
    k.s2 = E2 * (1.0f / 120.0f);
    k.s3 = E2 * (1.0f / 5040.0f);
    k.h0 = E2 * 0.5f;
    k.h1 = E2 * (1.0f / 24.0f);
    k.h2 = E2 * (1.0f / 720.0f);
    k.h3 = E2 * (1.0f / 40320.0f);
    k.E2 = E2;
    k.r = E1 / E2;
    k.oneE1 = 1.0f - E1;
    return k;
}

// E2-scaled rotation coefficients for θ² = -y: E2·cos θ, E2·sin θ/θ, E2·(1-cos θ)/θ²
struct RotCoefs {
    float c, s, h;
};

constexpr float kTaylorMax = 0.25f;  // largest θ² of the Taylor branch

// Taylor series in θ² through the cubic term (the next terms, θ⁸/9! and θ⁸/10!, are below 1.1e-8
// relative for θ² ≤ 0.25, under FP32 resolution) by Horner in y = -θ², and cos θ = 1 + y·h.
__device__ __forceinline__ RotCoefs rot_coefs_taylor(float y, const RotRelax& k) {
    RotCoefs q;
    q.s = fmaf(y, fmaf(y, fmaf(y, k.s3, k.s2), k.s1), k.s0);
    q.h = fmaf(y, fmaf(y, fmaf(y, k.h3, k.h2), k.h1), k.h0);
    q.c = fmaf(y, q.h, k.E2);
    return q;
}

__device__ __forceinline__ RotCoefs rot_coefs(float y, const RotRelax& k) {
    if (y >= -kTaylorMax) return rot_coefs_taylor(y, k);
    RotCoefs q;
    const float t2 = -y;
    const float th = sqrtf(t2);
    float sn, cs;
    sincosf(th, &sn, &cs);
    q.c = k.E2 * cs;
    q.s = k.E2 * (sn / th);
    q.h = k.E2 * ((1.0f - cs) / t2);
    return q;
}

// z component of the excitation axis of the isochromat at z (slice gradient and off-resonance
// during an RF sample), and the precession angle over the prephasing interval with `g` times the
// prephasing gradient
__device__ __forceinline__ float excite_az(const PssfpArgs& a, float z, float B0) {
    return -(a.gz_ex * z) - a.dt_ex * 6.28318530717958647692f * B0;
}
__device__ __forceinline__ float precess_angle(const PssfpArgs& a, float g, float z, float B0) {
    return -(g * a.gz_pr * z) - a.dt_pr * 6.28318530717958647692f * B0;
}

// rotation about the unnormalised axis (ax, ay, az) by |a|   (isochromat.cuh:14-73), followed by
// relaxation: transverse components times E2, longitudinal z·E1 + 1 - E1. E2 is folded into the
// rotation coefficients and E1 enters as E1/E2 on the E2-scaled longitudinal result. Every
// operation is written out (no contraction left to the compiler), in the form the packed update
// repeats on pairs of isochromats, so both give the same bits.
// REAL (a_y = ±0, pssfp_real_rf): the products with a_y are left out, as in the packed update; the
// same bits up to the sign of an exact zero.
template<bool REAL = false>
__device__ __forceinline__ void rotate_relax(Iso& m, float ax, float ay, float az, const RotCoefs& q,
                                             const RotRelax& k) {
    const float cx = REAL ? (-az) * m.y : fmaf(ay, m.z, (-az) * m.y);
    const float cy = fmaf(az, m.x, (-ax) * m.z);
    const float cz = REAL ? ax * m.y : fmaf(ax, m.y, (-ay) * m.x);
    const float hd = REAL ? q.h * fmaf(ax, m.x, az * m.z) : q.h * fmaf(ax, m.x, fmaf(ay, m.y, az * m.z));
    m.x = fmaf(q.c, m.x, fmaf(q.s, cx, hd * ax));
    m.y = REAL ? fmaf(q.c, m.y, q.s * cy) : fmaf(q.c, m.y, fmaf(q.s, cy, hd * ay));
    m.z = fmaf(k.r, fmaf(q.c, m.z, fmaf(q.s, cz, hd * az)), k.oneE1);
}

// Tangent of rotate_relax: the same linear map applied to d (without the regrowth 1 - E1) plus
// the explicit derivative (px, py, pz) of the step at the current state.
template<bool REAL = false>
__device__ __forceinline__ void rotate_relax_tangent(Iso& d, float ax, float ay, float az, const RotCoefs& q,
                                                     const RotRelax& k, float px, float py, float pz) {
    const float cx = REAL ? (-az) * d.y : fmaf(ay, d.z, (-az) * d.y);
    const float cy = fmaf(az, d.x, (-ax) * d.z);
    const float cz = REAL ? ax * d.y : fmaf(ax, d.y, (-ay) * d.x);
    const float hd = REAL ? q.h * fmaf(ax, d.x, az * d.z) : q.h * fmaf(ax, d.x, fmaf(ay, d.y, az * d.z));
    d.x = fmaf(q.c, d.x, fmaf(q.s, cx, fmaf(hd, ax, px)));
    d.y = REAL ? fmaf(q.c, d.y, fmaf(q.s, cy, py)) : fmaf(q.c, d.y, fmaf(q.s, cy, fmaf(hd, ay, py)));
    d.z = fmaf(k.r, fmaf(q.c, d.z, fmaf(q.s, cz, hd * az)), pz);
}

// One tile (128/GZ voxels) of a pSSFP simulation. Shared by the one-simulation kernel
// (tile = blockIdx.x) and the batched work-queue kernel, so both give bit-identical echoes.
// TAN: also propagate ∂m/∂T1 and ∂m/∂T2 (forward mode) and write their sums to a.dT1, a.dT2.
// Every step is affine in m: m' = D(θ)·R·m + (0, 0, 1 - E1) with D = diag(E2, E2, E1), so the
// tangent is d' = D·R·d + D_θ·R·m - (0, 0, E1_θ), and with ∂E/∂T = E·t/T² the explicit term is
// (0, 0, t/T1²·(m'_z - 1)) for T1 and (t/T2²·m'_x, t/T2²·m'_y, 0) for T2, in terms of the new
// state m'. The value goes through the same operations either way.
template<int ZT, int GZ, bool TAN = false>
__device__ __forceinline__ void pssfp_tile(const PssfpArgs& a, const int tile) {
    const int lane = threadIdx.x & 31;
    const int sub = lane % GZ;
    const int vloc = (tile * blockDim.x + threadIdx.x) / GZ;
    const bool vok = vloc < a.nvoxels;
    const int64_t vcol = a.voxel_begin + (vok ? vloc : a.nvoxels - 1);
    const float T1 = a.params[0 * a.param_stride + vcol];
    const float T2 = a.params[1 * a.param_stride + vcol];
    const float B1 = a.params[2 * a.param_stride + vcol];
    const float B0 = a.params[3 * a.param_stride + vcol];
    const float R1 = 1.0f / T1, R2 = 1.0f / T2;
    const float E1_ex = expf(-a.dt_ex * R1), E2_ex = expf(-a.dt_ex * R2);
    const float E1_pr = expf(-a.dt_pr * R1), E2_pr = expf(-a.dt_pr * R2);
    const float E1_inv = expf(-a.dt_inv * R1), E2_inv = expf(-a.dt_inv * R2);
    // tangent factors t/T1², t/T2² of each relaxation interval
    const float s1_ex = a.dt_ex * R1 * R1, s2_ex = a.dt_ex * R2 * R2;
    const float s1_pr = a.dt_pr * R1 * R1, s2_pr = a.dt_pr * R2 * R2;
    const float s1_inv = a.dt_inv * R1 * R1;

    Iso m[ZT];
    Iso d1[TAN ? ZT : 1], d2[TAN ? ZT : 1];  // ∂m/∂T1, ∂m/∂T2
    float az[ZT], cpr[ZT], spr[ZT];
    bool valid[ZT];
    const float cinv = cospif(B1);  // invert(p): z·cos(πB1)   (isochromat.cuh:100-112)
#pragma unroll
    for (int k = 0; k < ZT; k++) {
        const int zi = sub * ZT + k;
        valid[k] = zi < a.nz;
        const float z = valid[k] ? a.z[zi] : 0.0f;
        az[k] = excite_az(a, z, B0);
        sincosf(precess_angle(a, 1.0f, z, B0), &spr[k], &cpr[k]);
        m[k].x = 0.0f;
        m[k].y = 0.0f;
        m[k].z = fmaf(cinv, E1_inv, 1.0f - E1_inv);
        (void)E2_inv;
        if constexpr (TAN) {
            d1[k] = Iso {0.0f, 0.0f, s1_inv * (m[k].z - 1.0f)};
            d2[k] = Iso {0.0f, 0.0f, 0.0f};
        }
    }

    const RotRelax rr = make_rot_relax(E1_ex, E2_ex);
    auto excite = [&](int row) {
        const float2* zr = a.zap + int64_t(row) * a.nRF;
        for (int i = 0; i < a.nRF; i++) {
            const float2 zp = __ldg(zr + i);
            const float ax = zp.x * B1, ay = -zp.y * B1;
            const float naxy2 = -fmaf(ax, ax, ay * ay);
#pragma unroll
            for (int k = 0; k < ZT; k++) {
                const RotCoefs q = rot_coefs(fmaf(-az[k], az[k], naxy2), rr);
                rotate_relax(m[k], ax, ay, az[k], q, rr);
                if constexpr (TAN) {
                    rotate_relax_tangent(d1[k], ax, ay, az[k], q, rr, 0.0f, 0.0f, s1_ex * (m[k].z - 1.0f));
                    rotate_relax_tangent(d2[k], ax, ay, az[k], q, rr, s2_ex * m[k].x, s2_ex * m[k].y, 0.0f);
                }
            }
        }
    };
    // free precession by the angle (c, s) and relaxation over dt_pr
    auto precess_by = [&](int k, float c, float s) {
        const float x = m[k].x, y = m[k].y;
        m[k].x = E2_pr * fmaf(c, x, (-s) * y);
        m[k].y = E2_pr * fmaf(c, y, s * x);
        m[k].z = fmaf(m[k].z, E1_pr, 1.0f - E1_pr);
        if constexpr (TAN) {
            const float x1 = d1[k].x, y1 = d1[k].y, x2 = d2[k].x, y2 = d2[k].y;
            d1[k].x = E2_pr * fmaf(c, x1, (-s) * y1);
            d1[k].y = E2_pr * fmaf(c, y1, s * x1);
            d1[k].z = fmaf(d1[k].z, E1_pr, s1_pr * (m[k].z - 1.0f));
            d2[k].x = fmaf(s2_pr, m[k].x, E2_pr * fmaf(c, x2, (-s) * y2));
            d2[k].y = fmaf(s2_pr, m[k].y, E2_pr * fmaf(c, y2, s * x2));
            d2[k].z = d2[k].z * E1_pr;
        }
    };
    auto precess = [&]() {
#pragma unroll
        for (int k = 0; k < ZT; k++) precess_by(k, cpr[k], spr[k]);
    };

    // α/2 pulse, then re- and prephaser with twice the prephasing gradient (pssfp_kernels.cuh:73-80)
    excite(0);
#pragma unroll
    for (int k = 0; k < ZT; k++) {
        const int zi = sub * ZT + k;
        const float z = valid[k] ? a.z[zi] : 0.0f;
        float s2, c2;
        sincosf(precess_angle(a, 2.0f, z, B0), &s2, &c2);
        precess_by(k, c2, s2);
    }

    for (int t = 0; t < a.nTR; t++) {  // pssfp_kernels.cuh:83-107
        excite(t + 1);
        precess();
        float sx = 0.0f, sy = 0.0f;
#pragma unroll
        for (int k = 0; k < ZT; k++) {
            if (valid[k]) {
                sx += m[k].x;
                sy += m[k].y;
            }
        }
#pragma unroll
        for (int d = GZ / 2; d > 0; d /= 2) {
            sx += __shfl_xor_sync(0xffffffffu, sx, d, GZ);
            sy += __shfl_xor_sync(0xffffffffu, sy, d, GZ);
        }
        const int64_t at = int64_t(t) * a.echo_stride + a.voxel_begin + vloc;
        if (sub == 0 && vok) a.echo[at] = make_float2(sx, sy);
        if constexpr (TAN) {
            float t1x = 0.0f, t1y = 0.0f, t2x = 0.0f, t2y = 0.0f;
#pragma unroll
            for (int k = 0; k < ZT; k++) {
                if (valid[k]) {
                    t1x += d1[k].x;
                    t1y += d1[k].y;
                    t2x += d2[k].x;
                    t2y += d2[k].y;
                }
            }
#pragma unroll
            for (int d = GZ / 2; d > 0; d /= 2) {
                t1x += __shfl_xor_sync(0xffffffffu, t1x, d, GZ);
                t1y += __shfl_xor_sync(0xffffffffu, t1y, d, GZ);
                t2x += __shfl_xor_sync(0xffffffffu, t2x, d, GZ);
                t2y += __shfl_xor_sync(0xffffffffu, t2y, d, GZ);
            }
            if (sub == 0 && vok) {
                a.dT1[at] = make_float2(t1x, t1y);
                a.dT2[at] = make_float2(t2x, t2y);
            }
        }
        precess();
    }
}


// Two-wide form of pssfp_tile: a lane holds 2·ZP isochromats as ZP pairs, slot p in the low and
// slot p + ZP in the high half of one register pair per component, and every operation of the
// rotation, relaxation and precession is one sm_100 two-wide FP32 instruction on a pair, with the RF
// sample's axis (ax, ay) and the per-voxel coefficients broadcast to both halves. The operations are
// those of the scalar update in the same order, and the z sums run over the slots in the scalar
// order, so layout (ZP pairs, GZ lanes) gives the same bits as the scalar (2·ZP, GZ), tangents (TAN)
// included.
// REAL (every RF sample real, pssfp_real_rf): a_y = ±0, so the products a_y·m_z in the cross product's
// x, a_y·m_x in its z, a_y·m_y in a·m and hd·a_y in the new m_y are left out: 23 instructions per pair
// and RF sample instead of 27 (value; the same four per tangent). An FMA that adds ±0 to a product
// returns the rounded product, so the results are the same bits up to the sign of an exact zero.
// EXTRA = 1: one more isochromat, slot 2·ZP, in scalar registers with the scalar update (the same
// operations one-wide), so that an odd count per lane needs no padding slot (35 z on 4 lanes of 9
// instead of 10). Its update follows the pairs' (before them, ptxas spilled 40 B in the value kernel
// and 196 B in the tangent kernel; after them 4 B and 28 B).
template<int ZP, int GZ, bool TAN = false, bool REAL = false, int EXTRA = 0>
__device__ __forceinline__ void pssfp_tile_packed(const PssfpArgs& a, const int tile) {
    static_assert(EXTRA == 0 || EXTRA == 1, "at most one unpaired isochromat");
    constexpr int ZT = 2 * ZP + EXTRA;
    const int lane = threadIdx.x & 31;
    const int sub = lane % GZ;
    const int vloc = (tile * blockDim.x + threadIdx.x) / GZ;
    const bool vok = vloc < a.nvoxels;
    const int64_t vcol = a.voxel_begin + (vok ? vloc : a.nvoxels - 1);
    const float T1 = a.params[0 * a.param_stride + vcol];
    const float T2 = a.params[1 * a.param_stride + vcol];
    const float B1 = a.params[2 * a.param_stride + vcol];
    const float B0 = a.params[3 * a.param_stride + vcol];
    const float R1 = 1.0f / T1, R2 = 1.0f / T2;
    const float E1_ex = expf(-a.dt_ex * R1), E2_ex = expf(-a.dt_ex * R2);
    const float E1_pr = expf(-a.dt_pr * R1), E2_pr = expf(-a.dt_pr * R2);
    const float E1_inv = expf(-a.dt_inv * R1);
    // tangent factors t/T1², t/T2² of each relaxation interval
    const float s1_ex = a.dt_ex * R1 * R1, s2_ex = a.dt_ex * R2 * R2;
    const float s1_pr = a.dt_pr * R1 * R1, s2_pr = a.dt_pr * R2 * R2;
    const float s1_inv = a.dt_inv * R1 * R1;

    float2 mx[ZP], my[ZP], mz[ZP];      // the isochromats' magnetisation
    constexpr int ZD = TAN ? ZP : 1;
    float2 ax1[ZD], ay1[ZD], az1[ZD];   // ∂m/∂T1
    float2 ax2[ZD], ay2[ZD], az2[ZD];   // ∂m/∂T2
    float2 az[ZP], naz[ZP];             // excitation axis z component and its negation
    float2 cpr[ZP], spr[ZP], nspr[ZP];  // precession over the prephasing interval
    bool valid[ZT];
    const float cinv = cospif(B1);
    const float mz0 = fmaf(cinv, E1_inv, 1.0f - E1_inv);
#pragma unroll
    for (int p = 0; p < ZP; p++) {
        float zaz[2], zc[2], zs[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = p + h * ZP, zi = sub * ZT + k;
            valid[k] = zi < a.nz;
            const float z = valid[k] ? a.z[zi] : 0.0f;
            zaz[h] = excite_az(a, z, B0);
            sincosf(precess_angle(a, 1.0f, z, B0), &zs[h], &zc[h]);
        }
        az[p] = make_float2(zaz[0], zaz[1]);
        naz[p] = make_float2(-zaz[0], -zaz[1]);
        cpr[p] = make_float2(zc[0], zc[1]);
        spr[p] = make_float2(zs[0], zs[1]);
        nspr[p] = make_float2(-zs[0], -zs[1]);
        mx[p] = my[p] = bcast2(0.0f);
        mz[p] = bcast2(mz0);
        if constexpr (TAN) {
            ax1[p] = ay1[p] = ax2[p] = ay2[p] = az2[p] = bcast2(0.0f);
            az1[p] = bcast2(s1_inv * (mz0 - 1.0f));
        }
    }
    // the unpaired isochromat (EXTRA): magnetisation, tangents, axis z component, precession
    Iso em {0.0f, 0.0f, mz0}, ed1 {0.0f, 0.0f, s1_inv * (mz0 - 1.0f)}, ed2 {0.0f, 0.0f, 0.0f};
    float eaz = 0.0f, ecpr = 1.0f, espr = 0.0f;
    if constexpr (EXTRA) {
        const int k = 2 * ZP, zi = sub * ZT + k;
        valid[k] = zi < a.nz;
        const float z = valid[k] ? a.z[zi] : 0.0f;
        eaz = excite_az(a, z, B0);
        sincosf(precess_angle(a, 1.0f, z, B0), &espr, &ecpr);
    }

    const RotRelax rr = make_rot_relax(E1_ex, E2_ex);
    const float2 S0 = bcast2(rr.s0), S1 = bcast2(rr.s1), S2 = bcast2(rr.s2), S3 = bcast2(rr.s3);
    const float2 H0 = bcast2(rr.h0), H1 = bcast2(rr.h1), H2 = bcast2(rr.h2), H3 = bcast2(rr.h3);
    const float2 E2X = bcast2(rr.E2), RX = bcast2(rr.r), ONE_E1X = bcast2(rr.oneE1);
    const float2 S1EX = bcast2(s1_ex), S2EX = bcast2(s2_ex), NEG1 = bcast2(-1.0f);
    auto excite = [&](int row) {
        const float2* zr = a.zap + int64_t(row) * a.nRF;
        for (int i = 0; i < a.nRF; i++) {
            const float2 zp = __ldg(zr + i);
            const float ax = zp.x * B1, ay = -zp.y * B1;
            const float naxy2 = -fmaf(ax, ax, ay * ay);
            const float2 AX = bcast2(ax), AY = bcast2(ay), NAX = bcast2(-ax), NAY = bcast2(-ay);
            const float2 NAXY2 = bcast2(naxy2);
#pragma unroll
            for (int p = 0; p < ZP; p++) {
                const float2 y = fma2(naz[p], az[p], NAXY2);  // -θ² of both isochromats
                float2 c, sn, h;
                if (y.x >= -kTaylorMax && y.y >= -kTaylorMax) {
                    sn = fma2(y, fma2(y, fma2(y, S3, S2), S1), S0);
                    h = fma2(y, fma2(y, fma2(y, H3, H2), H1), H0);
                    c = fma2(y, h, E2X);
                } else {
                    const RotCoefs q0 = rot_coefs(y.x, rr), q1 = rot_coefs(y.y, rr);
                    c = make_float2(q0.c, q1.c);
                    sn = make_float2(q0.s, q1.s);
                    h = make_float2(q0.h, q1.h);
                }
                const float2 cx = REAL ? mul2(naz[p], my[p]) : fma2(AY, mz[p], mul2(naz[p], my[p]));
                const float2 cy = fma2(az[p], mx[p], mul2(NAX, mz[p]));
                const float2 cz = REAL ? mul2(AX, my[p]) : fma2(AX, my[p], mul2(NAY, mx[p]));
                const float2 hd = REAL ? mul2(h, fma2(AX, mx[p], mul2(az[p], mz[p])))
                                       : mul2(h, fma2(AX, mx[p], fma2(AY, my[p], mul2(az[p], mz[p]))));
                mx[p] = fma2(c, mx[p], fma2(sn, cx, mul2(hd, AX)));
                my[p] = REAL ? fma2(c, my[p], mul2(sn, cy)) : fma2(c, my[p], fma2(sn, cy, mul2(hd, AY)));
                mz[p] = fma2(RX, fma2(c, mz[p], fma2(sn, cz, mul2(hd, az[p]))), ONE_E1X);
                if constexpr (TAN) {
                    // the same map on the tangents plus the explicit terms at the new state:
                    // (0, 0, t/T1²·(m'_z - 1)) for T1, (t/T2²·m'_x, t/T2²·m'_y, 0) for T2
                    auto rotate = [&](float2& x, float2& yv, float2& z, float2 px, float2 py, float2 pz) {
                        const float2 tx = REAL ? mul2(naz[p], yv) : fma2(AY, z, mul2(naz[p], yv));
                        const float2 ty = fma2(az[p], x, mul2(NAX, z));
                        const float2 tz = REAL ? mul2(AX, yv) : fma2(AX, yv, mul2(NAY, x));
                        const float2 td = REAL ? mul2(h, fma2(AX, x, mul2(az[p], z)))
                                               : mul2(h, fma2(AX, x, fma2(AY, yv, mul2(az[p], z))));
                        x = fma2(c, x, fma2(sn, tx, fma2(td, AX, px)));
                        // REAL: fma2(td, ±0, py) is py exactly (py is a product or ±0)
                        yv = REAL ? fma2(c, yv, fma2(sn, ty, py)) : fma2(c, yv, fma2(sn, ty, fma2(td, AY, py)));
                        z = fma2(RX, fma2(c, z, fma2(sn, tz, mul2(td, az[p]))), pz);
                    };
                    rotate(ax1[p], ay1[p], az1[p], bcast2(0.0f), bcast2(0.0f), mul2(S1EX, add2(mz[p], NEG1)));
                    rotate(ax2[p], ay2[p], az2[p], mul2(S2EX, mx[p]), mul2(S2EX, my[p]), bcast2(0.0f));
                }
            }
            if constexpr (EXTRA) {  // the unpaired isochromat, with the scalar update (pssfp_tile)
                const RotCoefs q = rot_coefs(fmaf(-eaz, eaz, naxy2), rr);
                rotate_relax<REAL>(em, ax, ay, eaz, q, rr);
                if constexpr (TAN) {
                    rotate_relax_tangent<REAL>(ed1, ax, ay, eaz, q, rr, 0.0f, 0.0f, s1_ex * (em.z - 1.0f));
                    rotate_relax_tangent<REAL>(ed2, ax, ay, eaz, q, rr, s2_ex * em.x, s2_ex * em.y, 0.0f);
                }
            }
        }
    };
    const float2 E2P = bcast2(E2_pr), E1P = bcast2(E1_pr), ONE_E1P = bcast2(1.0f - E1_pr);
    const float2 S1P = bcast2(s1_pr), S2P = bcast2(s2_pr);
    auto precess_by = [&](int p, float2 c, float2 sn, float2 nsn) {
        const float2 x = mx[p], y = my[p];
        mx[p] = mul2(E2P, fma2(c, x, mul2(nsn, y)));
        my[p] = mul2(E2P, fma2(c, y, mul2(sn, x)));
        mz[p] = fma2(mz[p], E1P, ONE_E1P);
        if constexpr (TAN) {
            const float2 x1 = ax1[p], y1 = ay1[p], x2 = ax2[p], y2 = ay2[p];
            ax1[p] = mul2(E2P, fma2(c, x1, mul2(nsn, y1)));
            ay1[p] = mul2(E2P, fma2(c, y1, mul2(sn, x1)));
            az1[p] = fma2(az1[p], E1P, mul2(S1P, add2(mz[p], NEG1)));
            ax2[p] = fma2(S2P, mx[p], mul2(E2P, fma2(c, x2, mul2(nsn, y2))));
            ay2[p] = fma2(S2P, my[p], mul2(E2P, fma2(c, y2, mul2(sn, x2))));
            az2[p] = mul2(az2[p], E1P);
        }
    };
    // pssfp_tile's precession of the unpaired isochromat
    auto precess_extra = [&](float c, float sn) {
        if constexpr (EXTRA) {
            const float x = em.x, y = em.y;
            em.x = E2_pr * fmaf(c, x, (-sn) * y);
            em.y = E2_pr * fmaf(c, y, sn * x);
            em.z = fmaf(em.z, E1_pr, 1.0f - E1_pr);
            if constexpr (TAN) {
                const float x1 = ed1.x, y1 = ed1.y, x2 = ed2.x, y2 = ed2.y;
                ed1.x = E2_pr * fmaf(c, x1, (-sn) * y1);
                ed1.y = E2_pr * fmaf(c, y1, sn * x1);
                ed1.z = fmaf(ed1.z, E1_pr, s1_pr * (em.z - 1.0f));
                ed2.x = fmaf(s2_pr, em.x, E2_pr * fmaf(c, x2, (-sn) * y2));
                ed2.y = fmaf(s2_pr, em.y, E2_pr * fmaf(c, y2, sn * x2));
                ed2.z = ed2.z * E1_pr;
            }
        }
    };

    // α/2 pulse, then re- and prephaser with twice the prephasing gradient (pssfp_kernels.cuh:73-80)
    excite(0);
#pragma unroll
    for (int p = 0; p < ZP; p++) {
        float c2[2], s2[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int zi = sub * ZT + p + h * ZP;
            const float z = valid[p + h * ZP] ? a.z[zi] : 0.0f;
            sincosf(precess_angle(a, 2.0f, z, B0), &s2[h], &c2[h]);
        }
        precess_by(p, make_float2(c2[0], c2[1]), make_float2(s2[0], s2[1]), make_float2(-s2[0], -s2[1]));
    }
    if constexpr (EXTRA) {
        const int zi = sub * ZT + 2 * ZP;
        const float z = valid[2 * ZP] ? a.z[zi] : 0.0f;
        float c2, s2;
        sincosf(precess_angle(a, 2.0f, z, B0), &s2, &c2);
        precess_extra(c2, s2);
    }

    for (int t = 0; t < a.nTR; t++) {  // pssfp_kernels.cuh:83-107
        excite(t + 1);
#pragma unroll
        for (int p = 0; p < ZP; p++) precess_by(p, cpr[p], spr[p], nspr[p]);
        precess_extra(ecpr, espr);
        float sx = 0.0f, sy = 0.0f;
#pragma unroll
        for (int k = 0; k < ZT; k++) {
            if (valid[k]) {
                sx += k < ZP ? mx[k].x : k < 2 * ZP ? mx[k - ZP].y : em.x;
                sy += k < ZP ? my[k].x : k < 2 * ZP ? my[k - ZP].y : em.y;
            }
        }
#pragma unroll
        for (int d = GZ / 2; d > 0; d /= 2) {
            sx += __shfl_xor_sync(0xffffffffu, sx, d, GZ);
            sy += __shfl_xor_sync(0xffffffffu, sy, d, GZ);
        }
        const int64_t at = int64_t(t) * a.echo_stride + a.voxel_begin + vloc;
        if (sub == 0 && vok) a.echo[at] = make_float2(sx, sy);
        if constexpr (TAN) {
            float t1x = 0.0f, t1y = 0.0f, t2x = 0.0f, t2y = 0.0f;
#pragma unroll
            for (int k = 0; k < ZT; k++) {
                if (valid[k]) {
                    t1x += k < ZP ? ax1[k].x : k < 2 * ZP ? ax1[k - ZP].y : ed1.x;
                    t1y += k < ZP ? ay1[k].x : k < 2 * ZP ? ay1[k - ZP].y : ed1.y;
                    t2x += k < ZP ? ax2[k].x : k < 2 * ZP ? ax2[k - ZP].y : ed2.x;
                    t2y += k < ZP ? ay2[k].x : k < 2 * ZP ? ay2[k - ZP].y : ed2.y;
                }
            }
#pragma unroll
            for (int d = GZ / 2; d > 0; d /= 2) {
                t1x += __shfl_xor_sync(0xffffffffu, t1x, d, GZ);
                t1y += __shfl_xor_sync(0xffffffffu, t1y, d, GZ);
                t2x += __shfl_xor_sync(0xffffffffu, t2x, d, GZ);
                t2y += __shfl_xor_sync(0xffffffffu, t2y, d, GZ);
            }
            if (sub == 0 && vok) {
                a.dT1[at] = make_float2(t1x, t1y);
                a.dT2[at] = make_float2(t2x, t2y);
            }
        }
#pragma unroll
        for (int p = 0; p < ZP; p++) precess_by(p, cpr[p], spr[p], nspr[p]);
        precess_extra(ecpr, espr);
    }
}

// PACKED: ZT/2 pairs of isochromats per lane in the two-wide layout (pssfp_tile_packed). REAL: its
// real-RF form; the host launches both forms of a packed layout back to back, each reads the table's
// flag and the one that does not match returns at once (uniform over the grid).
template<int ZT, int GZ, bool PACKED = false, bool REAL = false>
__global__ void __launch_bounds__(128) pssfp_kernel(PssfpArgs a) {
    if (a.skip != nullptr && *a.skip != 0) return;  // uniform over the grid
    if constexpr (PACKED) {
        if (pssfp_real_rf(a) != REAL) return;
        pssfp_tile_packed<ZT / 2, GZ, false, REAL, ZT % 2>(a, blockIdx.x);
    } else {
        pssfp_tile<ZT, GZ>(a, blockIdx.x);
    }
}

// One pSSFP simulation with its T1 and T2 tangents into a.echo, a.dT1, a.dT2.
template<int ZT, int GZ, bool PACKED = false, bool REAL = false>
__global__ void __launch_bounds__(128) pssfp_tangent_kernel(PssfpArgs a) {
    if constexpr (PACKED) {
        if (pssfp_real_rf(a) != REAL) return;
        pssfp_tile_packed<ZT / 2, GZ, true, REAL, ZT % 2>(a, blockIdx.x);
    } else {
        pssfp_tile<ZT, GZ, true>(a, blockIdx.x);
    }
}

// Persistent work-queue kernel for a batch of pSSFP simulations sharing one (ZT, GZ) layout:
// CTAs of 128 threads take (job, tile) items, longest job first, through an atomic counter.
// TAN: the value and T1/T2 tangents (pssfp_tangent_kernel's work). REAL: every job's RF is real (the
// host groups jobs by their table's flag).
template<int ZT, int GZ, bool TAN = false, bool PACKED = false, bool REAL = false>
__global__ void __launch_bounds__(128) pssfp_queue_kernel(const PssfpArgs* __restrict__ jobs,
                                                          const int2* __restrict__ items, int nitems,
                                                          int* __restrict__ head) {
    __shared__ PssfpArgs job;
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(head, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const int2 w = items[it];
        if (threadIdx.x == 0) job = jobs[w.x];
        __syncthreads();
        if constexpr (PACKED) pssfp_tile_packed<ZT / 2, GZ, TAN, REAL, ZT % 2>(job, w.y);
        else pssfp_tile<ZT, GZ, TAN>(job, w.y);
        __syncthreads();
    }
}

}  // namespace kernels

namespace {
using PssfpKernel = void (*)(kernels::PssfpArgs);
using PssfpQueueKernel = void (*)(const kernels::PssfpArgs*, const int2*, int, int*);
struct PssfpConfig {
    int ZT, GZ;
    PssfpKernel fn;
    PssfpQueueKernel queue;
    PssfpKernel tangent;
    PssfpQueueKernel tangent_queue;
    bool packed;  // two-wide layout (ZT/2 pairs of isochromats per lane), value and tangent kernels
    // the real-RF forms (packed layouts, else null): fn_real and tangent_real launched beside fn and
    // tangent, the queue forms instead of theirs for groups of real-RF jobs
    PssfpKernel fn_real;
    PssfpQueueKernel queue_real;
    PssfpKernel tangent_real;
    PssfpQueueKernel tangent_queue_real;
};
#define COMPAS_PSSFP(ZT, GZ)                                                                        \
    {ZT, GZ, kernels::pssfp_kernel<ZT, GZ>, kernels::pssfp_queue_kernel<ZT, GZ>,                 \
     kernels::pssfp_tangent_kernel<ZT, GZ>, kernels::pssfp_queue_kernel<ZT, GZ, true>, false,     \
     nullptr, nullptr, nullptr, nullptr}
#define COMPAS_PSSFP_PACKED(ZT, GZ)                                                                 \
    {ZT, GZ, kernels::pssfp_kernel<ZT, GZ, true>, kernels::pssfp_queue_kernel<ZT, GZ, false, true>, \
     kernels::pssfp_tangent_kernel<ZT, GZ, true>, kernels::pssfp_queue_kernel<ZT, GZ, true, true>, true, \
     kernels::pssfp_kernel<ZT, GZ, true, true>, kernels::pssfp_queue_kernel<ZT, GZ, false, true, true>, \
     kernels::pssfp_tangent_kernel<ZT, GZ, true, true>, kernels::pssfp_queue_kernel<ZT, GZ, true, true, true>}
// packed value kernels with the scalar tangent kernels (the same bits; for layouts whose three packed
// vectors would not fit the registers)
#define COMPAS_PSSFP_PACKED_VALUE(ZT, GZ)                                                           \
    {ZT, GZ, kernels::pssfp_kernel<ZT, GZ, true>, kernels::pssfp_queue_kernel<ZT, GZ, false, true>, \
     kernels::pssfp_tangent_kernel<ZT, GZ>, kernels::pssfp_queue_kernel<ZT, GZ, true>, true,      \
     kernels::pssfp_kernel<ZT, GZ, true, true>, kernels::pssfp_queue_kernel<ZT, GZ, false, true, true>, \
     nullptr, nullptr}
const PssfpConfig kPssfpConfigs[] = {
    COMPAS_PSSFP(1, 1),  COMPAS_PSSFP(2, 1), COMPAS_PSSFP(4, 1),  COMPAS_PSSFP(8, 1),  COMPAS_PSSFP(9, 4),
    COMPAS_PSSFP(5, 8),  COMPAS_PSSFP(3, 16), COMPAS_PSSFP(2, 32), COMPAS_PSSFP(1, 32), COMPAS_PSSFP(18, 2),
    COMPAS_PSSFP(4, 4),  COMPAS_PSSFP(8, 4), COMPAS_PSSFP(4, 8),  COMPAS_PSSFP(12, 4),
    // the packed layouts come last, so the indices of the others (which a tuning table names) stay
    COMPAS_PSSFP_PACKED(2, 1), COMPAS_PSSFP_PACKED(4, 1), COMPAS_PSSFP_PACKED(10, 1), COMPAS_PSSFP_PACKED(2, 4),
    COMPAS_PSSFP_PACKED(4, 4), COMPAS_PSSFP_PACKED(6, 4), COMPAS_PSSFP_PACKED(10, 4), COMPAS_PSSFP_PACKED(6, 2),
    COMPAS_PSSFP_PACKED_VALUE(18, 2), COMPAS_PSSFP_PACKED(8, 8), COMPAS_PSSFP_PACKED(9, 4),
    COMPAS_PSSFP_PACKED(9, 1),
};
}  // namespace

int pssfp_config_count() {
    return int(sizeof(kPssfpConfigs) / sizeof(kPssfpConfigs[0]));
}

bool pssfp_config_info(int index, int* ZT, int* GZ) {
    if (index < 0 || index >= pssfp_config_count()) return false;
    *ZT = kPssfpConfigs[index].ZT;
    *GZ = kPssfpConfigs[index].GZ;
    return true;
}

bool pssfp_config_packed(int index) {
    return index >= 0 && index < pssfp_config_count() && kPssfpConfigs[index].packed;
}

// Default pSSFP layout (from timings on B200, 320 TRs of 15 RF samples): for 3 or more z positions
// the two-wide layout with the fewest slots (isochromats per lane × lanes) that cover nz, at most
// 5 pairs per lane, fewer lanes first on a tie (35 z: ZT10·GZ4 packed 9.9 ms vs 11.7 ms for the best
// scalar layout ZT9·GZ4 at 50176 voxels; 9 z: ZT10·GZ1 packed 1.64 ms vs 2.04 ms for ZT4·GZ4 at
// 16384 voxels); for 1 or 2 the scalar one-lane layout (a pair would hold one idle isochromat).
PssfpLaunch pssfp_default_launch(int nz, int64_t nvoxels) {
    (void)nvoxels;
    int best = -1;
    auto slots = [](const PssfpConfig& c) { return c.ZT * c.GZ; };
    for (int i = 0; i < pssfp_config_count(); i++) {
        const auto& c = kPssfpConfigs[i];
        const bool eligible = nz <= 2 ? (!c.packed && c.GZ == 1) : (c.packed && c.ZT / 2 <= 5);
        if (!eligible || slots(c) < nz) continue;
        if (best < 0 || slots(c) < slots(kPssfpConfigs[best]) ||
            (slots(c) == slots(kPssfpConfigs[best]) && c.GZ < kPssfpConfigs[best].GZ))
            best = i;
    }
    if (best < 0) {  // smallest covering layout of any shape
        for (int i = 0; i < pssfp_config_count(); i++) {
            const auto& c = kPssfpConfigs[i];
            if (slots(c) >= nz && (best < 0 || slots(c) < slots(kPssfpConfigs[best]))) best = i;
        }
    }
    if (best < 0) best = 7;  // 2 x 32 lanes covers nz ≤ 64
    return PssfpLaunch {best};
}

kernels::PssfpArgs pssfp_args(const CompasContext& ctx, const TissueParameters& params, int voxel_begin,
                              int nvoxels, const pSSFPSequence& seq, cfloat* echo, int64_t echo_stride) {
    const int nTR = int(seq.RF_train.size());
    const int nRF = int(seq.gamma_dt_RF.size());
    const int nz = int(seq.z.size());
    COMPAS_CHECK(nTR > 0);
    if (nz > 64) COMPAS_ERROR("pSSFP supports at most 64 z positions");
    DeviceGuard guard(ctx.device());
    std::shared_ptr<Array<cfloat, 2>> zap;
    {
        auto& cache = *seq.cache;
        std::lock_guard<std::mutex> lock(cache.mutex);
        if (!cache.table || cache.key_rf != seq.RF_train.data() || cache.key_g != seq.gamma_dt_RF.data()) {
            // rows 0..nTR: the axes; entry (nTR + 1)·nRF: the flag of a complex axis
            // (pssfp_table_kernel), at least one entry per row so that it exists when nRF = 0
            auto tab = std::make_shared<Array<cfloat, 2>>(std::array<int64_t, 2> {nTR + 2, std::max(nRF, 1)},
                                                          ctx.device(), ctx.stream());
            int n = (nTR + 1) * nRF;
            COMPAS_CUDA_CHECK(cudaMemsetAsync(tab->data() + int64_t(n), 0, sizeof(cfloat), ctx.stream()));
            if (n > 0) {
                kernels::pssfp_table_kernel<<<div_ceil(n, 256), 256, 0, ctx.stream()>>>(
                    reinterpret_cast<const float2*>(seq.RF_train.data()), nTR,
                    reinterpret_cast<const float2*>(seq.gamma_dt_RF.data()), nRF,
                    reinterpret_cast<float2*>(tab->data()));
                check_launch("pssfp_table_kernel");
            }
            cache.table = tab;
            cache.key_rf = seq.RF_train.data();
            cache.key_g = seq.gamma_dt_RF.data();
            cache.real_rf = -1;
        }
        zap = cache.table;
    }
    kernels::PssfpArgs a;
    a.params = params.data.data();
    a.param_stride = params.data.size(1);
    a.voxel_begin = voxel_begin;
    a.nvoxels = nvoxels;
    a.zap = reinterpret_cast<const float2*>(zap->data());
    a.z = seq.z.data();
    a.nTR = nTR;
    a.nRF = nRF;
    a.nz = nz;
    a.dt_ex = seq.dt.ex;
    a.dt_inv = seq.dt.inv;
    a.dt_pr = seq.dt.pr;
    a.gz_ex = seq.gamma_dt_GRz.ex;
    a.gz_pr = seq.gamma_dt_GRz.pr;
    a.echo = reinterpret_cast<float2*>(echo);
    a.echo_stride = echo_stride;
    a.dT1 = a.dT2 = nullptr;
    a.skip = nullptr;
    return a;
}

namespace {
const PssfpConfig& checked_config(PssfpLaunch L, int nz) {
    COMPAS_CHECK(L.config >= 0 && L.config < pssfp_config_count());
    const auto& cfg = kPssfpConfigs[L.config];
    if (cfg.ZT * cfg.GZ < nz) COMPAS_ERROR("pSSFP layout does not cover the z positions");
    return cfg;
}
constexpr int kPssfpThreads = 128;
}  // namespace

int pssfp_tile_voxels(PssfpLaunch L) {
    COMPAS_CHECK(L.config >= 0 && L.config < pssfp_config_count());
    return kPssfpThreads / kPssfpConfigs[L.config].GZ;
}

void launch_pssfp(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                  const pSSFPSequence& seq, cfloat* echo, int64_t echo_stride, PssfpLaunch L, const int* skip) {
    const int nz = int(seq.z.size());
    kernels::PssfpArgs a = pssfp_args(ctx, params, voxel_begin, nvoxels, seq, echo, echo_stride);
    a.skip = skip;
    if (nvoxels <= 0) return;
    if (L.config < 0) L = pssfp_default_launch(nz, nvoxels);
    const auto& cfg = checked_config(L, nz);
    const int64_t total = int64_t(nvoxels) * cfg.GZ;
    DeviceGuard guard(ctx.device());
    const unsigned grid = unsigned((total + kPssfpThreads - 1) / kPssfpThreads);
    cfg.fn<<<grid, kPssfpThreads, 0, ctx.stream()>>>(a);
    check_launch("pssfp_kernel");
    if (cfg.fn_real != nullptr) {  // the form that does not match the sequence returns at once
        cfg.fn_real<<<grid, kPssfpThreads, 0, ctx.stream()>>>(a);
        check_launch("pssfp_kernel (real RF)");
    }
}

void launch_pssfp_queue(cudaStream_t stream, int device, PssfpLaunch L, int nz, const kernels::PssfpArgs* jobs,
                        const int2* items, int nitems, int* head, bool real) {
    if (nitems <= 0) return;
    const auto& cfg = checked_config(L, nz);
    const PssfpQueueKernel fn = real && cfg.queue_real != nullptr ? cfg.queue_real : cfg.queue;
    DeviceGuard guard(device);
    int per_sm = 1, sms = 148;
    COMPAS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPssfpThreads, 0));
    COMPAS_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = std::max(1, std::min(nitems, std::max(1, per_sm) * sms));
    fn<<<grid, kPssfpThreads, 0, stream>>>(jobs, items, nitems, head);
    check_launch("pssfp_queue_kernel");
}

void launch_pssfp_tangent_queue(cudaStream_t stream, int device, PssfpLaunch L, int nz,
                                const kernels::PssfpArgs* jobs, const int2* items, int nitems, int* head, bool real) {
    if (nitems <= 0) return;
    const auto& cfg = checked_config(L, nz);
    const PssfpQueueKernel fn = real && cfg.tangent_queue_real != nullptr ? cfg.tangent_queue_real : cfg.tangent_queue;
    DeviceGuard guard(device);
    int per_sm = 1, sms = 148;
    COMPAS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPssfpThreads, 0));
    COMPAS_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = std::max(1, std::min(nitems, std::max(1, per_sm) * sms));
    fn<<<grid, kPssfpThreads, 0, stream>>>(jobs, items, nitems, head);
    check_launch("pssfp_tangent_queue_kernel");
}

bool pssfp_sequence_real_rf(const CompasContext& ctx, const pSSFPSequence& seq) {
    kernels::PssfpArgs a = pssfp_args(ctx, TissueParameters {}, 0, 0, seq, nullptr, 0);  // builds the table
    auto& cache = *seq.cache;
    std::lock_guard<std::mutex> lock(cache.mutex);
    if (cache.real_rf < 0) {
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        COMPAS_CUDA_CHECK(cudaStreamIsCapturing(ctx.stream(), &capture));
        if (capture != cudaStreamCaptureStatusNone) return false;  // the general form is right for every sequence
        float2 flag = make_float2(1.0f, 0.0f);
        DeviceGuard guard(ctx.device());
        COMPAS_CUDA_CHECK(cudaMemcpyAsync(&flag, a.zap + int64_t(a.nTR + 1) * a.nRF, sizeof(float2),
                                          cudaMemcpyDeviceToHost, ctx.stream()));
        COMPAS_CUDA_CHECK(cudaStreamSynchronize(ctx.stream()));
        cache.real_rf = flag.x == 0.0f ? 1 : 0;
    }
    return cache.real_rf == 1;
}

// Value and T1/T2 tangents in one launch, with the value kernel's layout L.
void launch_pssfp_tangent(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                          const pSSFPSequence& seq, cfloat* echo, cfloat* dT1, cfloat* dT2, int64_t echo_stride,
                          PssfpLaunch L) {
    const int nz = int(seq.z.size());
    kernels::PssfpArgs a = pssfp_args(ctx, params, voxel_begin, nvoxels, seq, echo, echo_stride);
    if (nvoxels <= 0) return;
    if (L.config < 0) L = pssfp_default_launch(nz, nvoxels);
    const auto& cfg = checked_config(L, nz);
    a.dT1 = reinterpret_cast<float2*>(dT1);
    a.dT2 = reinterpret_cast<float2*>(dT2);
    const int64_t total = int64_t(nvoxels) * cfg.GZ;
    DeviceGuard guard(ctx.device());
    const unsigned grid = unsigned((total + kPssfpThreads - 1) / kPssfpThreads);
    cfg.tangent<<<grid, kPssfpThreads, 0, ctx.stream()>>>(a);
    check_launch("pssfp_tangent_kernel");
    if (cfg.tangent_real != nullptr) {
        cfg.tangent_real<<<grid, kPssfpThreads, 0, ctx.stream()>>>(a);
        check_launch("pssfp_tangent_kernel (real RF)");
    }
}

MagnetizationTangents simulate_magnetization_tangents(const CompasContext& context, TissueParameters parameters,
                                                      pSSFPSequence sequence) {
    const int nTR = int(sequence.RF_train.size());
    const int nvoxels = parameters.nvoxels;
    MagnetizationTangents out {{{nTR, nvoxels}, context.device(), context.stream()},
                               {{nTR, nvoxels}, context.device(), context.stream()},
                               {{nTR, nvoxels}, context.device(), context.stream()}};
    launch_pssfp_tangent(context, parameters, 0, nvoxels, sequence, out.echos.data(), out.dT1.data(), out.dT2.data(),
                         nvoxels, tuned_pssfp_launch(int(sequence.z.size()), nvoxels));
    return out;
}

Array<cfloat, 2> simulate_magnetization(const CompasContext& context, TissueParameters parameters,
                                        pSSFPSequence sequence) {
    const int nTR = int(sequence.RF_train.size());
    Array<cfloat, 2> echos({nTR, parameters.nvoxels}, context.device(), context.stream());
    launch_pssfp(context, parameters, 0, parameters.nvoxels, sequence, echos.data(), parameters.nvoxels,
                 tuned_pssfp_launch(int(sequence.z.size()), parameters.nvoxels));
    return echos;
}

}  // namespace compas
