// hermitian.cu — compute_jacobian_hermitian (Jᴴ·v), plain FP32 path.
//
// Reference math (src/jacobian/hermitian_kernels.cuh:30-92): for every voxel
//   mHv_c   = Σ_{r,k} u[c][r][k]·conj(E_k·m[r])
//   dmHv0_c = Σ_{r,k} u·conj(E_k·∂T1m[r])
//   dmHv1_c = Σ_{r,k} u·conj(E_k·∂T2m[r] + dE_k·m[r])
//   JHv = Σ_c (conj(T1ρc)·dmHv0, conj(T2ρc)·dmHv1, conj(c)·mHv, -i·conj(c)·mHv)
// Regrouped as Y_c[r] = Σ_k u[c][r][k]·conj(E_k) and Ỹ_c[r] = Σ_k (k-S/2)·u[c][r][k]·conj(E_k)
// (dE_k = (k-S/2)ΔtR2²·E_k), so mHv_c = Σ_r conj(m[r])·Y_c[r], dmHv1_c = Σ_r conj(∂T2m[r])·Y_c[r]
// + ΔtR2²·conj(m[r])·Ỹ_c[r], etc. A CTA owns 64 voxels for all readouts and coils: it
// stages a 16-readout tile of the three echo arrays once, sweeps the coils against it, and
// keeps the four per-voxel results in registers — every echo byte is read once for all
// coils, and no [R][V] temporaries are written (the reference writes two per coil).
#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"

namespace compas {
namespace kernels {

constexpr int HV_V = 64, HV_RT = 16, HV_KC = 32, HV_THREADS = 128;  // 45 KB static smem

struct HermArgs {
    const float* params;
    int64_t pstride;
    int nvoxels;
    const float2* echo;
    const float2* dT1;
    const float2* dT2;
    const float2* coils;
    const float2* u;  // [C][R][S]
    int R, S, C;
    float dt, dk_re, dk_im;
    float2* out;      // [4][V]
};

__global__ void __launch_bounds__(HV_THREADS) hermitian_simt_kernel(HermArgs a) {
    __shared__ float2 Es[HV_KC][HV_V + 1];       // conj(E_k(v)) for the k chunk
    __shared__ float2 Us[HV_RT][HV_KC + 1];      // u[c][r][k] chunk
    __shared__ float2 Me[3][HV_RT][HV_V];        // m, ∂T1 m, ∂T2 m tile
    const int tid = threadIdx.x;
    const int vl = tid % HV_V, half = tid / HV_V;
    const int v = blockIdx.x * HV_V + vl;
    const bool vok = v < a.nvoxels;
    const int vc = vok ? v : a.nvoxels - 1;
    const double twopi = 6.283185307179586476925;

    const float T1 = a.params[0 * a.pstride + vc], T2 = a.params[1 * a.pstride + vc];
    const float B0 = a.params[3 * a.pstride + vc];
    const float2 rho = make_float2(a.params[4 * a.pstride + vc], a.params[5 * a.pstride + vc]);
    const float x = a.params[6 * a.pstride + vc], y = a.params[7 * a.pstride + vc];
    const float R2 = 1.0f / T2;
    const float dscale = a.dt * R2 * R2;
    const double theta = double(a.dk_re) * x + double(a.dk_im) * y + double(a.dt) * twopi * B0;
    const float decay = -a.dt * R2;

    float2 acc[4];
#pragma unroll
    for (int f = 0; f < 4; f++) acc[f] = make_float2(0.f, 0.f);

    for (int r0 = 0; r0 < a.R; r0 += HV_RT) {
        __syncthreads();
        for (int e = tid; e < HV_RT * HV_V; e += HV_THREADS) {
            const int rr = e / HV_V, vv = e % HV_V;
            const int r = r0 + rr, vg = blockIdx.x * HV_V + vv;
            float2 m = make_float2(0.f, 0.f), d1 = m, d2 = m;
            if (r < a.R && vg < a.nvoxels) {
                const int64_t idx = int64_t(r) * a.nvoxels + vg;
                m = a.echo[idx];
                d1 = a.dT1[idx];
                d2 = a.dT2[idx];
            }
            Me[0][rr][vv] = m;
            Me[1][rr][vv] = d1;
            Me[2][rr][vv] = d2;
        }
        for (int c = 0; c < a.C; c++) {
            float2 Y[HV_RT / 2], Yt[HV_RT / 2];
#pragma unroll
            for (int i = 0; i < HV_RT / 2; i++) Y[i] = Yt[i] = make_float2(0.f, 0.f);
            for (int k0 = 0; k0 < a.S; k0 += HV_KC) {
                __syncthreads();
                {  // conj(E_k) for 32 samples × 64 voxels: this thread makes 16 samples of voxel vl
                    const int kb = k0 + half * 16;
                    const float2 st = cis_rad(theta);
                    const float sm = __expf(decay);
                    const float2 step = make_float2(sm * st.x, sm * st.y);
#pragma unroll
                    for (int h8 = 0; h8 < 2; h8++) {
                        const float s0 = float(kb + 8 * h8) - 0.5f * float(a.S);
                        const float2 ph = cis_rad(double(s0) * theta);
                        const float mg = __expf(s0 * decay);
                        float2 e = make_float2(mg * ph.x, mg * ph.y);
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            const int kk = half * 16 + 8 * h8 + j;
                            Es[kk][vl] = (k0 + kk < a.S && vok) ? cconj(e) : make_float2(0.f, 0.f);
                            e = cmul(e, step);
                        }
                    }
                }
                for (int e = tid; e < HV_RT * HV_KC; e += HV_THREADS) {
                    const int rr = e / HV_KC, kk = e % HV_KC;
                    const int r = r0 + rr, k = k0 + kk;
                    Us[rr][kk] = (r < a.R && k < a.S) ? a.u[(int64_t(c) * a.R + r) * a.S + k] : make_float2(0.f, 0.f);
                }
                __syncthreads();
                const int kn = min(HV_KC, a.S - k0);
                for (int kk = 0; kk < kn; kk++) {
                    const float2 eb = Es[kk][vl];
                    const float ks = float(k0 + kk) - 0.5f * float(a.S);
#pragma unroll
                    for (int i = 0; i < HV_RT / 2; i++) {
                        const float2 t = cmul(Us[half * (HV_RT / 2) + i][kk], eb);
                        Y[i] = cadd(Y[i], t);
                        Yt[i] = make_float2(fmaf(ks, t.x, Yt[i].x), fmaf(ks, t.y, Yt[i].y));
                    }
                }
            }
            // finalize this coil against the staged echo tile
            float2 mH = make_float2(0.f, 0.f), d0 = mH, dd1 = mH;
#pragma unroll
            for (int i = 0; i < HV_RT / 2; i++) {
                const int rr = half * (HV_RT / 2) + i;
                const float2 m = Me[0][rr][vl], m1 = Me[1][rr][vl], m2 = Me[2][rr][vl];
                mH = cadd(mH, cmulc(Y[i], m));
                d0 = cadd(d0, cmulc(Y[i], m1));
                dd1 = cadd(dd1, cadd(cmulc(Y[i], m2), cscale(dscale, cmulc(Yt[i], m))));
            }
            const float2 cc = a.coils[int64_t(c) * a.nvoxels + vc];
            acc[0] = cadd(acc[0], cmulc(d0, cscale(T1, cmul(rho, cc))));
            acc[1] = cadd(acc[1], cmulc(dd1, cscale(T2, cmul(rho, cc))));
            const float2 cm = cmulc(mH, cc);
            acc[2] = cadd(acc[2], cm);
            acc[3] = cadd(acc[3], make_float2(cm.y, -cm.x));
        }
    }
    // combine the two readout halves
    __syncthreads();
    float2* red = &Me[0][0][0];
    if (half == 1) {
#pragma unroll
        for (int f = 0; f < 4; f++) red[f * HV_V + vl] = acc[f];
    }
    __syncthreads();
    if (half == 0 && vok) {
#pragma unroll
        for (int f = 0; f < 4; f++) a.out[int64_t(f) * a.nvoxels + v] = cadd(acc[f], red[f * HV_V + vl]);
    }
}

}  // namespace kernels

void launch_jacobian_hermitian_simt(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                    const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                                    int ncoils, const cfloat* vec, const CartesianGeom& g, cfloat* JHv) {
    if (nvoxels == 0) return;
    kernels::HermArgs a {};
    a.params = params;
    a.pstride = pstride;
    a.nvoxels = nvoxels;
    a.echo = reinterpret_cast<const float2*>(echos);
    a.dT1 = reinterpret_cast<const float2*>(dT1);
    a.dT2 = reinterpret_cast<const float2*>(dT2);
    a.coils = reinterpret_cast<const float2*>(coils);
    a.u = reinterpret_cast<const float2*>(vec);
    a.R = g.nreadouts;
    a.S = g.ns;
    a.C = ncoils;
    a.dt = g.dt;
    a.dk_re = g.dk_re;
    a.dk_im = g.dk_im;
    a.out = reinterpret_cast<float2*>(JHv);
    DeviceGuard guard(ctx.device());
    kernels::hermitian_simt_kernel<<<div_ceil(nvoxels, kernels::HV_V), kernels::HV_THREADS, 0, ctx.stream()>>>(a);
    check_launch("hermitian_simt_kernel");
}

}  // namespace compas
