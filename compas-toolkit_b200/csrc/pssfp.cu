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
#include "common.cuh"
#include "compas/compas.h"
#include "job_args.cuh"
#include "kernels.h"

namespace compas {
namespace kernels {

// zap[0][i] = -(RF[0]/2)·γΔtRF[i] (the α/2 pulse), zap[1+t][i] = RF[t]·γΔtRF[i]
__global__ void pssfp_table_kernel(const float2* __restrict__ rf, int nTR, const float2* __restrict__ g, int nRF,
                                   float2* __restrict__ zap) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (nTR + 1) * nRF) return;
    int row = idx / nRF, i = idx % nRF;
    float2 th = row == 0 ? make_float2(-rf[0].x / 2.0f, -rf[0].y / 2.0f) : rf[row - 1];
    zap[idx] = cmul(th, g[i]);
}


struct Iso {
    float x, y, z;
};

// Per-voxel constants of rotate_relax: the Taylor coefficients of sin θ/θ and (1-cos θ)/θ² (1/n!)
// times E2, E2 itself, E1/E2 and 1 - E1.
struct RotRelax {
    float s0, s1, s2, s3, h0, h1, h2, h3, E2, r, oneE1;
};

__device__ __forceinline__ RotRelax make_rot_relax(float E1, float E2) {
    RotRelax k;
    k.s0 = E2;
    k.s1 = E2 * (-1.0f / 6.0f);
    k.s2 = E2 * (1.0f / 120.0f);
    k.s3 = E2 * (-1.0f / 5040.0f);
    k.h0 = E2 * 0.5f;
    k.h1 = E2 * (-1.0f / 24.0f);
    k.h2 = E2 * (1.0f / 720.0f);
    k.h3 = E2 * (-1.0f / 40320.0f);
    k.E2 = E2;
    k.r = E1 / E2;
    k.oneE1 = 1.0f - E1;
    return k;
}

// E2-scaled rotation coefficients for θ² = t2: E2·cos θ, E2·sin θ/θ, E2·(1-cos θ)/θ²
struct RotCoefs {
    float c, s, h;
};

__device__ __forceinline__ RotCoefs rot_coefs(float t2, const RotRelax& k) {
    RotCoefs q;
    if (t2 <= 0.25f) {
        // Taylor series in x = θ² through x³ (the next terms, x⁴/9! and x⁴/10!, are below 1.1e-8
        // relative for x ≤ 0.25, under FP32 resolution), cos θ = 1 - x·(1-cos θ)/θ²
        const float x = t2;
        q.s = fmaf(x, fmaf(x, fmaf(x, k.s3, k.s2), k.s1), k.s0);
        q.h = fmaf(x, fmaf(x, fmaf(x, k.h3, k.h2), k.h1), k.h0);
        q.c = fmaf(-x, q.h, k.E2);
    } else {
        const float th = sqrtf(t2);
        float sn, cs;
        sincosf(th, &sn, &cs);
        q.c = k.E2 * cs;
        q.s = k.E2 * (sn / th);
        q.h = k.E2 * ((1.0f - cs) / t2);
    }
    return q;
}

// rotation about the unnormalised axis (ax, ay, az) by |a|   (isochromat.cuh:14-73), followed by
// relaxation: transverse components times E2, longitudinal z·E1 + 1 - E1. E2 is folded into the
// rotation coefficients and E1 enters as E1/E2 on the E2-scaled longitudinal result.
__device__ __forceinline__ void rotate_relax(Iso& m, float ax, float ay, float az, const RotCoefs& q,
                                             const RotRelax& k) {
    const float cx = ay * m.z - az * m.y;
    const float cy = az * m.x - ax * m.z;
    const float cz = ax * m.y - ay * m.x;
    const float hd = q.h * fmaf(ax, m.x, fmaf(ay, m.y, az * m.z));
    m.x = fmaf(q.c, m.x, fmaf(q.s, cx, hd * ax));
    m.y = fmaf(q.c, m.y, fmaf(q.s, cy, hd * ay));
    m.z = fmaf(k.r, fmaf(q.c, m.z, fmaf(q.s, cz, hd * az)), k.oneE1);
}

// Tangent of rotate_relax: the same linear map applied to d (without the regrowth 1 - E1) plus
// the explicit derivative (px, py, pz) of the step at the current state.
__device__ __forceinline__ void rotate_relax_tangent(Iso& d, float ax, float ay, float az, const RotCoefs& q,
                                                     const RotRelax& k, float px, float py, float pz) {
    const float cx = ay * d.z - az * d.y;
    const float cy = az * d.x - ax * d.z;
    const float cz = ax * d.y - ay * d.x;
    const float hd = q.h * fmaf(ax, d.x, fmaf(ay, d.y, az * d.z));
    d.x = fmaf(q.c, d.x, fmaf(q.s, cx, fmaf(hd, ax, px)));
    d.y = fmaf(q.c, d.y, fmaf(q.s, cy, fmaf(hd, ay, py)));
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
    const float twopi = 6.28318530717958647692f;
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
        az[k] = -(a.gz_ex * z) - a.dt_ex * twopi * B0;
        sincosf(-(a.gz_pr * z) - a.dt_pr * twopi * B0, &spr[k], &cpr[k]);
        m[k].x = 0.0f;
        m[k].y = 0.0f;
        m[k].z = cinv * E1_inv + (1.0f - E1_inv);
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
            const float axy2 = fmaf(ax, ax, ay * ay);
#pragma unroll
            for (int k = 0; k < ZT; k++) {
                const RotCoefs q = rot_coefs(fmaf(az[k], az[k], axy2), rr);
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
        m[k].x = E2_pr * (c * x - s * y);
        m[k].y = E2_pr * (c * y + s * x);
        m[k].z = fmaf(m[k].z, E1_pr, 1.0f - E1_pr);
        if constexpr (TAN) {
            const float x1 = d1[k].x, y1 = d1[k].y, x2 = d2[k].x, y2 = d2[k].y;
            d1[k].x = E2_pr * (c * x1 - s * y1);
            d1[k].y = E2_pr * (c * y1 + s * x1);
            d1[k].z = fmaf(d1[k].z, E1_pr, s1_pr * (m[k].z - 1.0f));
            d2[k].x = fmaf(s2_pr, m[k].x, E2_pr * (c * x2 - s * y2));
            d2[k].y = fmaf(s2_pr, m[k].y, E2_pr * (c * y2 + s * x2));
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
        sincosf(-(2.0f * a.gz_pr * z) - a.dt_pr * twopi * B0, &s2, &c2);
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

template<int ZT, int GZ>
__global__ void __launch_bounds__(128) pssfp_kernel(PssfpArgs a) {
    if (a.skip != nullptr && *a.skip != 0) return;  // uniform over the grid
    pssfp_tile<ZT, GZ>(a, blockIdx.x);
}

// One pSSFP simulation with its T1 and T2 tangents into a.echo, a.dT1, a.dT2.
template<int ZT, int GZ>
__global__ void __launch_bounds__(128) pssfp_tangent_kernel(PssfpArgs a) {
    pssfp_tile<ZT, GZ, true>(a, blockIdx.x);
}

// Persistent work-queue kernel for a batch of pSSFP simulations sharing one (ZT, GZ) layout:
// CTAs of 128 threads take (job, tile) items, longest job first, through an atomic counter.
// TAN: the value and T1/T2 tangents (pssfp_tangent_kernel's work).
template<int ZT, int GZ, bool TAN = false>
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
        pssfp_tile<ZT, GZ, TAN>(job, w.y);
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
};
const PssfpConfig kPssfpConfigs[] = {
    {1, 1, kernels::pssfp_kernel<1, 1>, kernels::pssfp_queue_kernel<1, 1>,
     kernels::pssfp_tangent_kernel<1, 1>, kernels::pssfp_queue_kernel<1, 1, true>},
    {2, 1, kernels::pssfp_kernel<2, 1>, kernels::pssfp_queue_kernel<2, 1>,
     kernels::pssfp_tangent_kernel<2, 1>, kernels::pssfp_queue_kernel<2, 1, true>},
    {4, 1, kernels::pssfp_kernel<4, 1>, kernels::pssfp_queue_kernel<4, 1>,
     kernels::pssfp_tangent_kernel<4, 1>, kernels::pssfp_queue_kernel<4, 1, true>},
    {8, 1, kernels::pssfp_kernel<8, 1>, kernels::pssfp_queue_kernel<8, 1>,
     kernels::pssfp_tangent_kernel<8, 1>, kernels::pssfp_queue_kernel<8, 1, true>},
    {9, 4, kernels::pssfp_kernel<9, 4>, kernels::pssfp_queue_kernel<9, 4>,
     kernels::pssfp_tangent_kernel<9, 4>, kernels::pssfp_queue_kernel<9, 4, true>},
    {5, 8, kernels::pssfp_kernel<5, 8>, kernels::pssfp_queue_kernel<5, 8>,
     kernels::pssfp_tangent_kernel<5, 8>, kernels::pssfp_queue_kernel<5, 8, true>},
    {3, 16, kernels::pssfp_kernel<3, 16>, kernels::pssfp_queue_kernel<3, 16>,
     kernels::pssfp_tangent_kernel<3, 16>, kernels::pssfp_queue_kernel<3, 16, true>},
    {2, 32, kernels::pssfp_kernel<2, 32>, kernels::pssfp_queue_kernel<2, 32>,
     kernels::pssfp_tangent_kernel<2, 32>, kernels::pssfp_queue_kernel<2, 32, true>},
    {1, 32, kernels::pssfp_kernel<1, 32>, kernels::pssfp_queue_kernel<1, 32>,
     kernels::pssfp_tangent_kernel<1, 32>, kernels::pssfp_queue_kernel<1, 32, true>},
    {18, 2, kernels::pssfp_kernel<18, 2>, kernels::pssfp_queue_kernel<18, 2>,
     kernels::pssfp_tangent_kernel<18, 2>, kernels::pssfp_queue_kernel<18, 2, true>},
    {4, 4, kernels::pssfp_kernel<4, 4>, kernels::pssfp_queue_kernel<4, 4>,
     kernels::pssfp_tangent_kernel<4, 4>, kernels::pssfp_queue_kernel<4, 4, true>},
    {8, 4, kernels::pssfp_kernel<8, 4>, kernels::pssfp_queue_kernel<8, 4>,
     kernels::pssfp_tangent_kernel<8, 4>, kernels::pssfp_queue_kernel<8, 4, true>},
    {4, 8, kernels::pssfp_kernel<4, 8>, kernels::pssfp_queue_kernel<4, 8>,
     kernels::pssfp_tangent_kernel<4, 8>, kernels::pssfp_queue_kernel<4, 8, true>},
    {12, 4, kernels::pssfp_kernel<12, 4>, kernels::pssfp_queue_kernel<12, 4>,
     kernels::pssfp_tangent_kernel<12, 4>, kernels::pssfp_queue_kernel<12, 4, true>},
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

// Default pSSFP layout (from the autotuner's timings on B200): 4 lanes per voxel with the
// fewest isochromats per lane that cover nz (9 z: ZT4·GZ4 2.3 ms vs 3.9 ms for ZT4·GZ8 at 16384
// voxels; 35 z: ZT9·GZ4 13.8 ms vs 14.0 ms for ZT5·GZ8 at 50176 voxels); 8 lanes when that
// needs more than 12 per lane, one lane for nz ≤ 2.
PssfpLaunch pssfp_default_launch(int nz, int64_t nvoxels) {
    (void)nvoxels;
    const int want_gz = nz <= 2 ? 1 : (div_ceil(nz, 4) <= 12 ? 4 : 8);
    int best = -1;
    for (int i = 0; i < pssfp_config_count(); i++) {
        const auto& c = kPssfpConfigs[i];
        if (c.GZ != want_gz || c.ZT * c.GZ < nz) continue;
        if (best < 0 || c.ZT < kPssfpConfigs[best].ZT) best = i;
    }
    if (best < 0) {  // smallest covering layout of any shape
        for (int i = 0; i < pssfp_config_count(); i++) {
            const auto& c = kPssfpConfigs[i];
            if (c.ZT * c.GZ >= nz && (best < 0 || c.ZT * c.GZ < kPssfpConfigs[best].ZT * kPssfpConfigs[best].GZ))
                best = i;
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
            auto tab = std::make_shared<Array<cfloat, 2>>(std::array<int64_t, 2> {nTR + 1, nRF}, ctx.device(), ctx.stream());
            int n = (nTR + 1) * nRF;
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
    cfg.fn<<<unsigned((total + kPssfpThreads - 1) / kPssfpThreads), kPssfpThreads, 0, ctx.stream()>>>(a);
    check_launch("pssfp_kernel");
}

void launch_pssfp_queue(cudaStream_t stream, int device, PssfpLaunch L, int nz, const kernels::PssfpArgs* jobs,
                        const int2* items, int nitems, int* head) {
    if (nitems <= 0) return;
    const auto& cfg = checked_config(L, nz);
    DeviceGuard guard(device);
    int per_sm = 1, sms = 148;
    COMPAS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cfg.queue, kPssfpThreads, 0));
    COMPAS_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = std::max(1, std::min(nitems, std::max(1, per_sm) * sms));
    cfg.queue<<<grid, kPssfpThreads, 0, stream>>>(jobs, items, nitems, head);
    check_launch("pssfp_queue_kernel");
}

void launch_pssfp_tangent_queue(cudaStream_t stream, int device, PssfpLaunch L, int nz,
                                const kernels::PssfpArgs* jobs, const int2* items, int nitems, int* head) {
    if (nitems <= 0) return;
    const auto& cfg = checked_config(L, nz);
    DeviceGuard guard(device);
    int per_sm = 1, sms = 148;
    COMPAS_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cfg.tangent_queue, kPssfpThreads, 0));
    COMPAS_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int grid = std::max(1, std::min(nitems, std::max(1, per_sm) * sms));
    cfg.tangent_queue<<<grid, kPssfpThreads, 0, stream>>>(jobs, items, nitems, head);
    check_launch("pssfp_tangent_queue_kernel");
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
    cfg.tangent<<<unsigned((total + kPssfpThreads - 1) / kPssfpThreads), kPssfpThreads, 0, ctx.stream()>>>(a);
    check_launch("pssfp_tangent_kernel");
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
