// spiral_hermitian.cu — Jᴴ·u on a spiral trajectory.
//
// The reference's Jᴴ·v accepts only Cartesian trajectories (compas/jacobian/hermitian.h:30,
// src/jacobian/hermitian_kernels.cuh:30-92). On a spiral, readout r of voxel v carries its own
// factor F_rvk = readout_rv · z_rv^k (the spiral signal model: spiral_view.cuh:13-73), with
// dF/dT2 = (k - S/2)·Δt·R2²·F like the Cartesian dE/dT2. With U_rv(k) = Σ_c conj(C_cv)·u[c][r][k]:
//
//   Y_rv  = Σ_k conj(F_rvk)·U_rv(k),   Ỹ_rv = Σ_k (k - S/2)·conj(F_rvk)·U_rv(k)
//   Jᴴu[0][v] = Σ_r conj(T1ρ·∂T1m_rv)·Y_rv
//   Jᴴu[1][v] = Σ_r conj(T2ρ·∂T2m_rv)·Y_rv + conj(T2ρ·ΔtR2²·m_rv)·Ỹ_rv
//   Jᴴu[2][v] = Σ_r conj(m_rv)·Y_rv,   Jᴴu[3] = -i·Jᴴu[2]
//
// One thread per voxel, 128 voxels per CTA. For each readout of its readout range and each
// group of CT coils, the CTA stages u[c][r][k0:k0+64] in shared memory; a thread forms U, the
// products with conj(F) (recomputed exactly, FP64-reduced phase, at the start of every 64-sample
// chunk and advanced by conj(z) within it) and accumulates Y and Ỹ, then folds them into its four
// outputs with the readout's m, ∂T1m, ∂T2m. Readout ranges are split over CTAs (split-K) when the
// voxel tiles alone do not fill the GPU; partial outputs are summed in a fixed order.
#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"

namespace compas {

void sum_partials(const CompasContext& ctx, const cfloat* partials, int nsplit, int64_t n, cfloat* out);

namespace kernels {

constexpr int SH_THREADS = 128, SH_KC = 64;

struct SpiralHermArgs {
    const float* params;
    int64_t pstride;
    int nvoxels;
    const float2* echo;
    const float2* dT1;
    const float2* dT2;
    const float2* coils;  // [C][V]
    const float2* u;      // [C][R][S]
    int R, S, C;
    float dt;
    const float2* k_start;
    const float2* delta_k;
    int readouts_per_split;
    float2* out;  // [splits][4][V]
};

template<int CT>
__global__ void __launch_bounds__(SH_THREADS) spiral_hermitian_kernel(SpiralHermArgs a) {
    __shared__ float2 sU[CT][SH_KC];
    const int v = blockIdx.x * SH_THREADS + threadIdx.x;
    const bool vok = v < a.nvoxels;
    const int vv = vok ? v : a.nvoxels - 1;
    const int r_begin = blockIdx.y * a.readouts_per_split;
    const int r_end = min(a.R, r_begin + a.readouts_per_split);
    const double twopi = 6.283185307179586476925, inv_2pi = 0.15915494309189533577;

    const float T1 = a.params[vv], T2 = a.params[a.pstride + vv], B0 = a.params[3 * a.pstride + vv];
    const float x = a.params[6 * a.pstride + vv], y = a.params[7 * a.pstride + vv];
    const float2 rho = make_float2(a.params[4 * a.pstride + vv], a.params[5 * a.pstride + vv]);
    const float R2 = 1.0f / T2;
    const float dec = -a.dt * R2;
    const double half = 0.5 * double(a.S) * double(a.dt);
    const float mag = expf(float(half) * R2);
    const float2 t1r = cscale(T1, rho), t2r = cscale(T2, rho);
    const float2 t2rq = cscale(a.dt * R2 * R2, t2r);

    float2 out0 = make_float2(0.f, 0.f), out1 = out0, out2 = out0;
    for (int c0 = 0; c0 < a.C; c0 += CT) {
        float2 cc[CT];  // conj(coil)
#pragma unroll
        for (int c = 0; c < CT; c++)
            cc[c] = (c0 + c < a.C) ? cconj(a.coils[int64_t(c0 + c) * a.nvoxels + vv]) : make_float2(0.f, 0.f);
        for (int r = r_begin; r < r_end; r++) {
            const float2 ks = a.k_start[r], dkr = a.delta_k[r];
            // readout factor (rewind by (S/2)Δt, prephase with Re k0·x) and the per-sample phase
            const float2 rw = cis_rad(-half * twopi * double(B0) + double(ks.x) * double(x));
            const float2 rd = cscale(mag, rw);
            const double turns = (double(dkr.x) * x + double(dkr.y) * y + double(a.dt) * twopi * B0) * inv_2pi;
            const float2 zc = cconj(cscale(__expf(dec), cis_turns(turns)));
            float2 Y = make_float2(0.f, 0.f), Yt = Y;
            for (int k0 = 0; k0 < a.S; k0 += SH_KC) {
                const int nk = min(SH_KC, a.S - k0);
                __syncthreads();
                for (int i = threadIdx.x; i < CT * SH_KC; i += SH_THREADS) {
                    const int c = i / SH_KC, kk = i % SH_KC;
                    sU[c][kk] = (c0 + c < a.C && kk < nk) ? a.u[(int64_t(c0 + c) * a.R + r) * a.S + k0 + kk]
                                                          : make_float2(0.f, 0.f);
                }
                __syncthreads();
                // conj(F) at the chunk start: exact, then the recurrence within the chunk
                const float2 ph = cis_turns(double(k0) * turns);
                const float m0 = __expf(float(k0) * dec);
                float2 G = cconj(cmul(rd, make_float2(m0 * ph.x, m0 * ph.y)));
                for (int kk = 0; kk < nk; kk++) {
                    float2 U = make_float2(0.f, 0.f);
#pragma unroll
                    for (int c = 0; c < CT; c++) U = cfma(cc[c], sU[c][kk], U);
                    const float2 t = cmul(U, G);
                    const float w = float(k0 + kk) - 0.5f * float(a.S);
                    Y = cadd(Y, t);
                    Yt = make_float2(fmaf(w, t.x, Yt.x), fmaf(w, t.y, Yt.y));
                    G = cmul(G, zc);
                }
            }
            if (vok) {
                const int64_t idx = int64_t(r) * a.nvoxels + v;
                const float2 me = a.echo[idx], d1 = a.dT1[idx], d2 = a.dT2[idx];
                out0 = cadd(out0, cmulc(Y, cmul(t1r, d1)));
                out1 = cadd(out1, cadd(cmulc(Y, cmul(t2r, d2)), cmulc(Yt, cmul(t2rq, me))));
                out2 = cadd(out2, cmulc(Y, me));
            }
        }
    }
    if (vok) {
        float2* o = a.out + int64_t(blockIdx.y) * 4 * a.nvoxels;
        o[v] = out0;
        o[a.nvoxels + v] = out1;
        o[2 * int64_t(a.nvoxels) + v] = out2;
        o[3 * int64_t(a.nvoxels) + v] = make_float2(out2.y, -out2.x);  // -i·out2
    }
}

}  // namespace kernels

void launch_jacobian_hermitian_spiral(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                      const cfloat* echos, const cfloat* dT1, const cfloat* dT2,
                                      const cfloat* coils, int ncoils, const cfloat* vec, int nreadouts, int ns,
                                      float dt, const cfloat* k_start, const cfloat* delta_k, cfloat* JHv,
                                      Precision prec) {
    if (nvoxels == 0) return;
    if (prec == Precision::SplitBF16 &&
        launch_jacobian_hermitian_spiral_tc(ctx, params, pstride, nvoxels, echos, dT1, dT2, coils, ncoils, vec,
                                            nreadouts, ns, dt, k_start, delta_k, JHv))
        return;
    DeviceGuard guard(ctx.device());
    if (int64_t(ncoils) * nreadouts * ns == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(JHv, 0, sizeof(cfloat) * 4 * size_t(nvoxels), ctx.stream()));
        return;
    }
    kernels::SpiralHermArgs a {};
    a.params = params;
    a.pstride = pstride;
    a.nvoxels = nvoxels;
    a.echo = reinterpret_cast<const float2*>(echos);
    a.dT1 = reinterpret_cast<const float2*>(dT1);
    a.dT2 = reinterpret_cast<const float2*>(dT2);
    a.coils = reinterpret_cast<const float2*>(coils);
    a.u = reinterpret_cast<const float2*>(vec);
    a.R = nreadouts;
    a.S = ns;
    a.C = ncoils;
    a.dt = dt;
    a.k_start = reinterpret_cast<const float2*>(k_start);
    a.delta_k = reinterpret_cast<const float2*>(delta_k);
    // split the readouts over CTAs until ~8 CTAs per SM are in flight (≥ 8 readouts per split)
    const int vtiles = div_ceil(nvoxels, kernels::SH_THREADS);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device());
    const int want = div_ceil(8 * sms, vtiles);
    const int splits_max = std::max(1, nreadouts / 8);
    int splits = std::max(1, std::min(want, splits_max));
    a.readouts_per_split = div_ceil(nreadouts, splits);
    splits = div_ceil(nreadouts, a.readouts_per_split);
    const int64_t n = 4 * int64_t(nvoxels);
    Array<cfloat, 2> partials({splits > 1 ? splits : 0, n}, ctx.device(), ctx.stream());
    a.out = reinterpret_cast<float2*>(splits > 1 ? partials.data() : JHv);
    const int ct = ncoils <= 1 ? 1 : ncoils <= 2 ? 2 : ncoils <= 4 ? 4 : 8;
    dim3 grid(vtiles, splits);
    switch (ct) {
        case 1: kernels::spiral_hermitian_kernel<1><<<grid, kernels::SH_THREADS, 0, ctx.stream()>>>(a); break;
        case 2: kernels::spiral_hermitian_kernel<2><<<grid, kernels::SH_THREADS, 0, ctx.stream()>>>(a); break;
        case 4: kernels::spiral_hermitian_kernel<4><<<grid, kernels::SH_THREADS, 0, ctx.stream()>>>(a); break;
        default: kernels::spiral_hermitian_kernel<8><<<grid, kernels::SH_THREADS, 0, ctx.stream()>>>(a); break;
    }
    check_launch("spiral_hermitian_kernel");
    if (splits > 1) sum_partials(ctx, partials.data(), splits, n, JHv);
}

}  // namespace compas
