// signal.cu — magnetization_to_signal (Cartesian, spiral) and J·v, plain FP32 path.
//
// Cartesian signal (reference: src/trajectories/signal_kernels.cuh:137-167,
// compas/trajectories/cartesian_view.cuh:28-63) and J·v (src/jacobian/product_kernels.cuh:
// 7-67) are both contractions over voxels of a streamed operand A[r][v] with a generated
// operand B[(c,k)][v] = coil[c][v]·E_k(v):
//   E_k(v) = exp((k - S/2)·(-Δt/T2 + iΘ_v)),  Θ_v = Δk_re·x + Δk_im·y + 2πΔt·B0.
// For the signal the reference's readout rewind/prephaser times the sample factor equals
// E_k(v)·exp(i(S/2)Δk_im·y) exactly, so A = echo and the per-voxel ρ and y-term go into B.
// For J·v the two sums Σ_v P·E and Σ_v Q·dE/dT2 share E because dE/dT2 = (k-S/2)ΔtR2²·E:
//   Jv[c][r][k] = Σ_v coil·E_k·(P[r][v] + (k-S/2)·Q'[r][v]),  Q' = Δt R2² Q.
// The phase (k-S/2)·Θ_v reaches hundreds of radians; it is reduced modulo 2π in FP64
// before the FP32 sincos, so B carries ~1e-7 relative error instead of the ~1e-5–1e-4
// of an FP32 phase.
//
// Kernel shape: a CTA computes a 128 (readouts) × 64 (samples) tile of one coil over a
// voxel range (split-K over voxels, partial tiles summed in fixed order by a second
// kernel); 256 threads, 8×4 complex register micro-tile, 16-voxel shared-memory chunks.
#include "common.cuh"
#include "compas/compas.h"
#include "job_args.cuh"
#include "kernels.h"

namespace compas {
namespace kernels {

constexpr int SG_RT = 128, SG_KT = 64, SG_VT = 16, SG_THREADS = 256;

enum class GenMode { Signal, Jacobian };

struct SignalArgs {
    const float* params;
    int64_t pstride;
    int nvoxels;
    const float2* echo;  // [R][V]   (Jacobian: echos)
    const float2* dT1;   // Jacobian only
    const float2* dT2;   // Jacobian only
    const float2* vec;   // Jacobian only [4][V]
    const float2* coils; // [C][V]
    int R, S, C;
    float dt, dk_re, dk_im;
    int vchunk;          // voxels per split
    float2* out;         // partials [splits][C][R][S]
};

// E_k(v) for k = k0..k0+3 with exact start (FP64 phase reduction) and a 3-step recurrence
__device__ __forceinline__ void sample_factors4(float a_decay, double theta, int S, int k0, float2 out[4]) {
    const float s0 = float(k0) - 0.5f * float(S);
    const float2 ph = cis_rad(double(s0) * theta);
    const float mag = __expf(s0 * a_decay);
    float2 e = make_float2(mag * ph.x, mag * ph.y);
    const float2 st = cis_rad(theta);
    const float sm = __expf(a_decay);
    const float2 step = make_float2(sm * st.x, sm * st.y);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        out[j] = e;
        e = cmul(e, step);
    }
}

template<GenMode MODE>
__global__ void __launch_bounds__(SG_THREADS, 2) signal_gemm_kernel(SignalArgs a) {
    __shared__ float2 As[SG_VT][SG_RT + 1];
    __shared__ float2 Aq[MODE == GenMode::Jacobian ? SG_VT : 1][SG_RT + 1];
    __shared__ float2 Bs[SG_VT][SG_KT + 1];
    const int tid = threadIdx.x;
    const int k_tile = blockIdx.x * SG_KT, r_tile = blockIdx.y * SG_RT;
    const int c = blockIdx.z % a.C, split = blockIdx.z / a.C;
    const int v_begin = split * a.vchunk, v_end = min(a.nvoxels, v_begin + a.vchunk);
    const int ty = tid / 16, tx = tid % 16;

    float2 acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = make_float2(0.f, 0.f);

    const double twopi = 6.283185307179586476925;
    for (int v0 = v_begin; v0 < v_end; v0 += SG_VT) {
        // ---- operand A: 128 readouts × 16 voxels
#pragma unroll
        for (int i = 0; i < (SG_RT * SG_VT) / SG_THREADS; i++) {
            const int e = tid + i * SG_THREADS;
            const int rr = e / SG_VT, vv = e % SG_VT;
            const int r = r_tile + rr, v = v0 + vv;
            float2 x = make_float2(0.f, 0.f), q = make_float2(0.f, 0.f);
            if (r < a.R && v < v_end) {
                const int64_t idx = int64_t(r) * a.nvoxels + v;
                if constexpr (MODE == GenMode::Signal) {
                    x = a.echo[idx];
                } else {
                    // P = v0 T1 ρ ∂T1m + v1 T2 ρ ∂T2m + v2 m + v3 i m;  Q' = Δt R2² v1 T2 ρ m
                    const float T1 = a.params[0 * a.pstride + v], T2 = a.params[1 * a.pstride + v];
                    const float2 rho = make_float2(a.params[4 * a.pstride + v], a.params[5 * a.pstride + v]);
                    const float2 me = a.echo[idx], d1 = a.dT1[idx], d2 = a.dT2[idx];
                    const float2 w0 = a.vec[v], w1 = a.vec[a.nvoxels + v];
                    const float2 w2 = a.vec[2 * int64_t(a.nvoxels) + v], w3 = a.vec[3 * int64_t(a.nvoxels) + v];
                    const float2 t1r = cscale(T1, rho), t2r = cscale(T2, rho);
                    x = cmul(cmul(w0, t1r), d1);
                    x = cadd(x, cmul(cmul(w1, t2r), d2));
                    x = cadd(x, cmul(w2, me));
                    x = cadd(x, cmul(make_float2(-w3.y, w3.x), me));
                    const float R2 = 1.0f / T2;
                    q = cscale(a.dt * R2 * R2, cmul(cmul(w1, t2r), me));
                }
            }
            As[vv][rr] = x;
            if constexpr (MODE == GenMode::Jacobian) Aq[vv][rr] = q;
        }
        // ---- operand B: coil · E_k (· ρ · e^{i(S/2)Δk_im y} for the signal), 64 samples × 16 voxels
        {
            const int vv = tid % SG_VT, kg = tid / SG_VT;  // 16 groups × 4 samples
            const int v = v0 + vv;
            float2 f[4];
            if (v < v_end) {
                const float T2 = a.params[1 * a.pstride + v], B0 = a.params[3 * a.pstride + v];
                const float x = a.params[6 * a.pstride + v], y = a.params[7 * a.pstride + v];
                const double theta = double(a.dk_re) * x + double(a.dk_im) * y + double(a.dt) * twopi * B0;
                sample_factors4(-a.dt / T2, theta, a.S, k_tile + 4 * kg, f);
                float2 w = a.coils[int64_t(c) * a.nvoxels + v];
                if constexpr (MODE == GenMode::Signal) {
                    const float2 rho = make_float2(a.params[4 * a.pstride + v], a.params[5 * a.pstride + v]);
                    w = cmul(w, rho);
                    if (a.dk_im != 0.0f) w = cmul(w, cis_rad(0.5 * double(a.S) * double(a.dk_im) * y));
                }
#pragma unroll
                for (int j = 0; j < 4; j++) f[j] = cmul(f[j], w);
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) f[j] = make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) Bs[vv][4 * kg + j] = f[j];
        }
        __syncthreads();
        // ---- 8 × 4 complex micro-tile
#pragma unroll 4
        for (int vv = 0; vv < SG_VT; vv++) {
            float2 b[4];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[vv][tx * 4 + j];
            if constexpr (MODE == GenMode::Jacobian) {
                float2 b2[4];
#pragma unroll
                for (int j = 0; j < 4; j++) b2[j] = cscale(float(k_tile + tx * 4 + j) - 0.5f * float(a.S), b[j]);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const float2 p = As[vv][ty * 8 + i], q = Aq[vv][ty * 8 + i];
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[i][j] = cfma(q, b2[j], cfma(p, b[j], acc[i][j]));
                }
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const float2 p = As[vv][ty * 8 + i];
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[i][j] = cfma(p, b[j], acc[i][j]);
                }
            }
        }
        __syncthreads();
    }
    float2* out = a.out + (int64_t(split) * a.C + c) * int64_t(a.R) * a.S;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int r = r_tile + ty * 8 + i;
        if (r >= a.R) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int k = k_tile + tx * 4 + j;
            if (k < a.S) out[int64_t(r) * a.S + k] = acc[i][j];
        }
    }
}

// out[i] = Σ_s partials[s][i], fixed order
__global__ void sum_partials_kernel(const float2* __restrict__ partials, int nsplit, int64_t n, float2* __restrict__ out) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        float2 s = partials[i];
        for (int p = 1; p < nsplit; p++) s = cadd(s, partials[int64_t(p) * n + i]);
        out[i] = s;
    }
}

// ---- spiral: per readout r, s[c][r][k] = Σ_v coil·A[r][v]·z_rv^k  (signal_kernels.cuh:274-345)
//
// A block owns one readout, SP_THREADS·SP_KPT consecutive samples and CT coils; each thread
// keeps SP_KPT samples × CT coils of accumulators. Voxels are staged SP_VCH at a time in shared
// memory with everything that depends on the voxel only: A = ρ·rewind·prephaser·m, Θ_rv in
// turns (FP64), the decay -Δt R2, the per-sample step z_rv = e^{-Δt R2 + iΘ_rv} and the coil
// values. Per voxel a thread then forms its start factor z^{k0} (FP64-reduced phase) once and
// advances it by z along its samples, so the work per staged voxel is CT·SP_KPT complex FMAs
// plus SP_KPT complex products. Every (coil, sample) accumulates the voxels in the same order
// whatever CT is, so the result does not depend on the coil grouping.
constexpr int SP_THREADS = 128, SP_KPT = 8, SP_VCH = 64;

// One block of the spiral signal: samples bx·SP_THREADS·SP_KPT.., readout r, coils cz·CT..
// Shared by the one-operation kernel (blockIdx) and the batched kernel: bit-identical results.
template<int CT, bool JAC = false>
__device__ __forceinline__ void spiral_tile(const SpiralArgs& a, const int bx, const int r, const int cz) {
    __shared__ float2 sA[SP_VCH];
    __shared__ float2 sAQ[JAC ? SP_VCH : 1];  // J·v: the (k - S/2)-weighted source
    __shared__ double sTurns[SP_VCH];
    __shared__ float sDecay[SP_VCH];
    __shared__ float2 sStep[SP_VCH];
    __shared__ float2 sCoil[CT][SP_VCH];
    const int c0 = cz * CT;
    const int k0 = (bx * SP_THREADS + threadIdx.x) * SP_KPT;
    const double twopi = 6.283185307179586476925, inv_2pi = 0.15915494309189533577;
    const float2 ks = a.k_start[r], dkr = a.delta_k[r];
    float2 acc[CT][SP_KPT];
#pragma unroll
    for (int c = 0; c < CT; c++)
#pragma unroll
        for (int j = 0; j < SP_KPT; j++) acc[c][j] = make_float2(0.f, 0.f);

    for (int v0 = 0; v0 < a.nvoxels; v0 += SP_VCH) {
        for (int i = threadIdx.x; i < SP_VCH; i += SP_THREADS) {
            const int v = v0 + i;
            float2 A = make_float2(0.f, 0.f), AQ = make_float2(0.f, 0.f), step = make_float2(0.f, 0.f);
            double turns = 0.0;
            float dec = 0.0f;
            if (v < a.nvoxels) {
                const float T2 = a.params[1 * a.pstride + v], B0 = a.params[3 * a.pstride + v];
                const float x = a.params[6 * a.pstride + v], y = a.params[7 * a.pstride + v];
                const float2 rho = make_float2(a.params[4 * a.pstride + v], a.params[5 * a.pstride + v]);
                const float R2 = 1.0f / T2;
                // rewind by (S/2)Δt and prephase with Re k0·x   (spiral_view.cuh:13-59)
                const double half = 0.5 * double(a.S) * double(a.dt);
                const float2 rw = cis_rad(-half * twopi * double(B0) + double(ks.x) * double(x));
                const float mag = expf(float(half) * R2);
                if constexpr (!JAC) {
                    A = cmul(cmul(a.echo[int64_t(r) * a.nvoxels + v], cscale(mag, rw)), rho);
                } else {
                    // J·v source (product_kernels.cuh:56-60 with the spiral factor): P = T1ρv0·∂T1m +
                    // T2ρv1·∂T2m + (v2 + i v3)·m and Q = ΔtR2²·T2ρv1·m, both times the readout factor
                    const float T1 = a.params[v];
                    const int64_t idx = int64_t(r) * a.nvoxels + v;
                    const float2 me = a.echo[idx], d1 = a.dT1[idx], d2 = a.dT2[idx];
                    const float2 w0 = a.vec[v], w1 = a.vec[a.nvoxels + v];
                    const float2 w2 = a.vec[2 * int64_t(a.nvoxels) + v], w3 = a.vec[3 * int64_t(a.nvoxels) + v];
                    const float2 c1 = cmul(w0, cscale(T1, rho)), c2 = cmul(w1, cscale(T2, rho));
                    const float2 cm = make_float2(w2.x - w3.y, w2.y + w3.x);
                    const float2 P = cadd(cadd(cmul(c1, d1), cmul(c2, d2)), cmul(cm, me));
                    const float2 Q = cmul(cscale(a.dt * R2 * R2, c2), me);
                    const float2 rd = cscale(mag, rw);
                    A = cmul(rd, P);
                    AQ = cmul(rd, Q);
                }
                turns = (double(dkr.x) * x + double(dkr.y) * y + double(a.dt) * twopi * B0) * inv_2pi;
                dec = -a.dt * R2;
                step = cscale(__expf(dec), cis_turns(turns));
            }
            sA[i] = A;
            if constexpr (JAC) sAQ[i] = AQ;
            sTurns[i] = turns;
            sDecay[i] = dec;
            sStep[i] = step;
#pragma unroll
            for (int c = 0; c < CT; c++)
                sCoil[c][i] = (v < a.nvoxels && c0 + c < a.C) ? a.coils[int64_t(c0 + c) * a.nvoxels + v]
                                                                : make_float2(0.f, 0.f);
        }
        __syncthreads();
        if (k0 < a.S) {
            const int nv = min(SP_VCH, a.nvoxels - v0);
            for (int i = 0; i < nv; i++) {
                const float2 ph = cis_turns(double(k0) * sTurns[i]);
                const float m0 = __expf(float(k0) * sDecay[i]);
                const float2 z0 = make_float2(m0 * ph.x, m0 * ph.y);
                float2 e = cmul(sA[i], z0);
                const float2 step = sStep[i];
                float2 coil[CT];
#pragma unroll
                for (int c = 0; c < CT; c++) coil[c] = sCoil[c][i];
                if constexpr (!JAC) {
#pragma unroll
                    for (int j = 0; j < SP_KPT; j++) {
#pragma unroll
                        for (int c = 0; c < CT; c++) acc[c][j] = cfma(coil[c], e, acc[c][j]);
                        e = cmul(e, step);
                    }
                } else {
                    float2 f = cmul(sAQ[i], z0);
#pragma unroll
                    for (int j = 0; j < SP_KPT; j++) {
                        const float kk = float(k0 + j) - 0.5f * float(a.S);
                        const float2 t = make_float2(fmaf(kk, f.x, e.x), fmaf(kk, f.y, e.y));
#pragma unroll
                        for (int c = 0; c < CT; c++) acc[c][j] = cfma(coil[c], t, acc[c][j]);
                        e = cmul(e, step);
                        f = cmul(f, step);
                    }
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int c = 0; c < CT; c++) {
        if (c0 + c >= a.C) continue;
#pragma unroll
        for (int j = 0; j < SP_KPT; j++) {
            const int k = k0 + j;
            if (k < a.S) a.signal[(int64_t(c0 + c) * a.R + r) * a.S + k] = acc[c][j];
        }
    }
}

template<int CT>
__global__ void __launch_bounds__(SP_THREADS) signal_spiral_kernel(SpiralArgs a) {
    spiral_tile<CT>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// J·v on a spiral trajectory (no counterpart in the reference, whose Jacobians are Cartesian only)
template<int CT>
__global__ void __launch_bounds__(SP_THREADS) jacobian_spiral_kernel(SpiralArgs a) {
    spiral_tile<CT, true>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

__device__ __forceinline__ int job_of_block(const int* __restrict__ offsets, int njobs, int b) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(offsets + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Batched spiral signal: flattened block b → job j (cta_offsets[j] ≤ b < cta_offsets[j+1]) and the
// block (l % nx, (l / nx) % R, l / (nx·R)) of that job's own grid, l = b - cta_offsets[j].
template<int CT>
__global__ void __launch_bounds__(SP_THREADS) signal_spiral_batch_kernel(const SpiralArgs* __restrict__ jobs,
                                                                        const int* __restrict__ cta_offsets,
                                                                        int njobs) {
    __shared__ SpiralArgs job;
    __shared__ int3 blk;
    if (threadIdx.x == 0) {
        const int j = job_of_block(cta_offsets, njobs, blockIdx.x);
        job = jobs[j];
        const int nx = (job.S + SP_THREADS * SP_KPT - 1) / (SP_THREADS * SP_KPT);
        const int l = blockIdx.x - cta_offsets[j];
        blk = make_int3(l % nx, (l / nx) % job.R, l / (nx * job.R));
    }
    __syncthreads();
    spiral_tile<CT>(job, blk.x, blk.y, blk.z);
}

// Batched sum of split-K partials: flattened 256-thread block b → job j, element
// (b - block_offsets[j])·256 + t; same per-element order as sum_partials_kernel.
__global__ void sum_partials_batch_kernel(const PartialSum* __restrict__ jobs, const int* __restrict__ block_offsets,
                                          int njobs) {
    const int j = job_of_block(block_offsets, njobs, blockIdx.x);
    const PartialSum p = jobs[j];
    const int64_t i = int64_t(blockIdx.x - block_offsets[j]) * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    float2 s = p.partials[i];
    for (int q = 1; q < p.nsplit; q++) s = cadd(s, p.partials[int64_t(q) * p.n + i]);
    p.out[i] = s;
}

}  // namespace kernels

void sum_partials(const CompasContext& ctx, const cfloat* partials, int nsplit, int64_t n, cfloat* out) {
    DeviceGuard guard(ctx.device());
    const int blocks = int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)));
    kernels::sum_partials_kernel<<<blocks, 256, 0, ctx.stream()>>>(reinterpret_cast<const float2*>(partials), nsplit,
                                                                    n, reinterpret_cast<float2*>(out));
    check_launch("sum_partials_kernel");
}

namespace {

template<kernels::GenMode MODE>
void run_signal_gemm(const CompasContext& ctx, kernels::SignalArgs a, cfloat* out) {
    DeviceGuard guard(ctx.device());
    const int ktiles = div_ceil(a.S, kernels::SG_KT), rtiles = div_ceil(a.R, kernels::SG_RT);
    const int64_t tiles = int64_t(ktiles) * rtiles * a.C;
    // enough CTAs for ~3 per SM, at least 64 voxel chunks per split
    int splits = int(std::max<int64_t>(1, (148 * 3 + tiles - 1) / tiles));
    splits = std::min(splits, std::max(1, a.nvoxels / (64 * kernels::SG_VT)));
    a.vchunk = div_ceil(div_ceil(a.nvoxels, splits), kernels::SG_VT) * kernels::SG_VT;
    splits = div_ceil(a.nvoxels, a.vchunk);
    const int64_t n = int64_t(a.C) * a.R * a.S;
    Array<cfloat, 2> partials({splits > 1 ? splits : 0, n}, ctx.device(), ctx.stream());
    a.out = reinterpret_cast<float2*>(splits > 1 ? partials.data() : out);
    dim3 grid(ktiles, rtiles, a.C * splits);
    kernels::signal_gemm_kernel<MODE><<<grid, kernels::SG_THREADS, 0, ctx.stream()>>>(a);
    check_launch("signal_gemm_kernel");
    if (splits > 1) sum_partials(ctx, partials.data(), splits, n, out);
}

}  // namespace

void launch_signal_cartesian_simt(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                  const cfloat* echos, const cfloat* coils, int ncoils, const CartesianGeom& g,
                                  cfloat* signal) {
    if (int64_t(ncoils) * g.nreadouts * g.ns == 0) return;
    if (nvoxels == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(signal, 0, sizeof(cfloat) * size_t(ncoils) * g.nreadouts * g.ns, ctx.stream()));
        return;
    }
    kernels::SignalArgs a {};
    a.params = params;
    a.pstride = pstride;
    a.nvoxels = nvoxels;
    a.echo = reinterpret_cast<const float2*>(echos);
    a.coils = reinterpret_cast<const float2*>(coils);
    a.R = g.nreadouts;
    a.S = g.ns;
    a.C = ncoils;
    a.dt = g.dt;
    a.dk_re = g.dk_re;
    a.dk_im = g.dk_im;
    run_signal_gemm<kernels::GenMode::Signal>(ctx, a, signal);
}

void launch_jacobian_simt(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                          const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils, int ncoils,
                          const cfloat* vec, const CartesianGeom& g, cfloat* Jv) {
    if (int64_t(ncoils) * g.nreadouts * g.ns == 0) return;
    if (nvoxels == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(Jv, 0, sizeof(cfloat) * size_t(ncoils) * g.nreadouts * g.ns, ctx.stream()));
        return;
    }
    kernels::SignalArgs a {};
    a.params = params;
    a.pstride = pstride;
    a.nvoxels = nvoxels;
    a.echo = reinterpret_cast<const float2*>(echos);
    a.dT1 = reinterpret_cast<const float2*>(dT1);
    a.dT2 = reinterpret_cast<const float2*>(dT2);
    a.vec = reinterpret_cast<const float2*>(vec);
    a.coils = reinterpret_cast<const float2*>(coils);
    a.R = g.nreadouts;
    a.S = g.ns;
    a.C = ncoils;
    a.dt = g.dt;
    a.dk_re = g.dk_re;
    a.dk_im = g.dk_im;
    run_signal_gemm<kernels::GenMode::Jacobian>(ctx, a, Jv);
}

void launch_signal_spiral_simt(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                               const cfloat* echos, const cfloat* coils, int ncoils, int nreadouts, int ns, float dt,
                               const cfloat* k_start, const cfloat* delta_k, cfloat* signal) {
    if (int64_t(ncoils) * nreadouts * ns == 0) return;
    kernels::SpiralArgs a {};
    a.params = params;
    a.pstride = pstride;
    a.nvoxels = nvoxels;
    a.echo = reinterpret_cast<const float2*>(echos);
    a.coils = reinterpret_cast<const float2*>(coils);
    a.R = nreadouts;
    a.S = ns;
    a.C = ncoils;
    a.dt = dt;
    a.k_start = reinterpret_cast<const float2*>(k_start);
    a.delta_k = reinterpret_cast<const float2*>(delta_k);
    a.signal = reinterpret_cast<float2*>(signal);
    DeviceGuard guard(ctx.device());
    const int ct = spiral_coil_group(ncoils);
    dim3 grid(div_ceil(ns, kernels::SP_THREADS * kernels::SP_KPT), nreadouts, div_ceil(ncoils, ct));
    switch (ct) {
        case 1: kernels::signal_spiral_kernel<1><<<grid, kernels::SP_THREADS, 0, ctx.stream()>>>(a); break;
        case 2: kernels::signal_spiral_kernel<2><<<grid, kernels::SP_THREADS, 0, ctx.stream()>>>(a); break;
        case 4: kernels::signal_spiral_kernel<4><<<grid, kernels::SP_THREADS, 0, ctx.stream()>>>(a); break;
        default: kernels::signal_spiral_kernel<8><<<grid, kernels::SP_THREADS, 0, ctx.stream()>>>(a); break;
    }
    check_launch("signal_spiral_kernel");
}

// Coils per block for `ncoils` coils: minimises (blocks per readout) × (modelled instructions
// per staged voxel and thread), where a block of CT coils costs 4·CT·8 FMAs for the products,
// 8 complex steps and ~50 instructions for the start factor and shared-memory loads.
void launch_jacobian_spiral_simt(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                 const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                                 int ncoils, const cfloat* vec, int nreadouts, int ns, float dt,
                                 const cfloat* k_start, const cfloat* delta_k, cfloat* Jv) {
    if (int64_t(ncoils) * nreadouts * ns == 0) return;
    kernels::SpiralArgs a {};
    a.params = params;
    a.pstride = pstride;
    a.nvoxels = nvoxels;
    a.echo = reinterpret_cast<const float2*>(echos);
    a.dT1 = reinterpret_cast<const float2*>(dT1);
    a.dT2 = reinterpret_cast<const float2*>(dT2);
    a.vec = reinterpret_cast<const float2*>(vec);
    a.coils = reinterpret_cast<const float2*>(coils);
    a.R = nreadouts;
    a.S = ns;
    a.C = ncoils;
    a.dt = dt;
    a.k_start = reinterpret_cast<const float2*>(k_start);
    a.delta_k = reinterpret_cast<const float2*>(delta_k);
    a.signal = reinterpret_cast<float2*>(Jv);
    DeviceGuard guard(ctx.device());
    const int ct = spiral_coil_group(ncoils);
    dim3 grid(div_ceil(ns, kernels::SP_THREADS * kernels::SP_KPT), nreadouts, div_ceil(ncoils, ct));
    switch (ct) {
        case 1: kernels::jacobian_spiral_kernel<1><<<grid, kernels::SP_THREADS, 0, ctx.stream()>>>(a); break;
        case 2: kernels::jacobian_spiral_kernel<2><<<grid, kernels::SP_THREADS, 0, ctx.stream()>>>(a); break;
        case 4: kernels::jacobian_spiral_kernel<4><<<grid, kernels::SP_THREADS, 0, ctx.stream()>>>(a); break;
        default: kernels::jacobian_spiral_kernel<8><<<grid, kernels::SP_THREADS, 0, ctx.stream()>>>(a); break;
    }
    check_launch("jacobian_spiral_kernel");
}

int spiral_coil_group(int ncoils) {
    int best = 1;
    double best_cost = 1e300;
    for (int ct : {1, 2, 4, 8}) {
        const double cost = double(div_ceil(std::max(ncoils, 1), ct)) * (32.0 * ct + 48.0 + 50.0);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = ct;
        }
    }
    return best;
}

int spiral_block_count(int ncoils, int nreadouts, int ns) {
    const int kper = kernels::SP_THREADS * kernels::SP_KPT;
    return div_ceil(ns, kper) * nreadouts * div_ceil(ncoils, spiral_coil_group(ncoils));
}

void launch_signal_spiral_batch(cudaStream_t stream, int device, int coil_group, const kernels::SpiralArgs* jobs,
                                const int* cta_offsets, int njobs, int ctas) {
    if (njobs <= 0 || ctas <= 0) return;
    DeviceGuard guard(device);
    switch (coil_group) {
        case 1: kernels::signal_spiral_batch_kernel<1><<<ctas, kernels::SP_THREADS, 0, stream>>>(jobs, cta_offsets, njobs); break;
        case 2: kernels::signal_spiral_batch_kernel<2><<<ctas, kernels::SP_THREADS, 0, stream>>>(jobs, cta_offsets, njobs); break;
        case 4: kernels::signal_spiral_batch_kernel<4><<<ctas, kernels::SP_THREADS, 0, stream>>>(jobs, cta_offsets, njobs); break;
        case 8: kernels::signal_spiral_batch_kernel<8><<<ctas, kernels::SP_THREADS, 0, stream>>>(jobs, cta_offsets, njobs); break;
        default: COMPAS_ERROR("invalid spiral coil grouping");
    }
    check_launch("signal_spiral_batch_kernel");
}

void launch_sum_partials_batch(cudaStream_t stream, int device, const kernels::PartialSum* jobs,
                               const int* block_offsets, int njobs, int blocks) {
    if (njobs <= 0 || blocks <= 0) return;
    DeviceGuard guard(device);
    kernels::sum_partials_batch_kernel<<<blocks, 256, 0, stream>>>(jobs, block_offsets, njobs);
    check_launch("sum_partials_batch_kernel");
}

bool launch_signal_spiral_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                             const cfloat* echos, const cfloat* coils, int ncoils, int nreadouts, int ns, float dt,
                             const cfloat* k_start, const cfloat* delta_k, cfloat* signal);
bool launch_jacobian_spiral_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                               const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                               int ncoils, const cfloat* vec, int nreadouts, int ns, float dt, const cfloat* k_start,
                               const cfloat* delta_k, cfloat* Jv);

void launch_signal_spiral(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                          const cfloat* echos, const cfloat* coils, int ncoils, int nreadouts, int ns, float dt,
                          const cfloat* k_start, const cfloat* delta_k, cfloat* signal, Precision prec) {
    if (prec == Precision::SplitBF16 && launch_signal_spiral_tc(ctx, params, pstride, nvoxels, echos, coils, ncoils,
                                                                nreadouts, ns, dt, k_start, delta_k, signal))
        return;
    launch_signal_spiral_simt(ctx, params, pstride, nvoxels, echos, coils, ncoils, nreadouts, ns, dt, k_start, delta_k,
                              signal);
}

void launch_jacobian_spiral(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                            const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils, int ncoils,
                            const cfloat* vec, int nreadouts, int ns, float dt, const cfloat* k_start,
                            const cfloat* delta_k, cfloat* Jv, Precision prec) {
    if (prec == Precision::SplitBF16 && launch_jacobian_spiral_tc(ctx, params, pstride, nvoxels, echos, dT1, dT2,
                                                                  coils, ncoils, vec, nreadouts, ns, dt, k_start,
                                                                  delta_k, Jv))
        return;
    launch_jacobian_spiral_simt(ctx, params, pstride, nvoxels, echos, dT1, dT2, coils, ncoils, vec, nreadouts, ns, dt,
                                k_start, delta_k, Jv);
}

}  // namespace compas

