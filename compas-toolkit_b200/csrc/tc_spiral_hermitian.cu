// tc_spiral_hermitian.cu — Jᴴ·u on a spiral trajectory on tcgen05 tensor cores, split-BF16.
//
// Jᴴu (the FP32 form is spiral_hermitian.cu; signal model: spiral_view.cuh:13-73) needs, per
// readout r and voxel v,
//   Y_rv = Σ_k conj(F_rvk)·U_rv(k),  Ỹ_rv = Σ_k (k - S/2)·conj(F_rvk)·U_rv(k),
//   F_rvk = rd_rv·z_rv^k,  U_rv(k) = Σ_c conj(C_cv)·u[c][r][k].
// With k = 128t + j and ct_t = conj(rd·z^{128t}):
//   Y_rv = Σ_c conj(C_cv)·Σ_t ct_t·G[v][(c,t)],
//   Ỹ_rv = Σ_c conj(C_cv)·Σ_t ct_t·((128t - S/2)·G[v][(c,t)] + G̃[v][(c,t)]),
//   G[v][(c,t)] = Σ_j conj(z_v^j)·u[c][r][128t + j],   G̃[v][(c,t)] = Σ_j j·conj(z_v^j)·u[c][r][128t + j],
// so per readout one GEMM with M = 128 voxels (TMEM lanes), K = the 128 in-tile samples j and
// N = 32 columns per coil (G_re, G_im, G̃_re, G̃_im for each of T ≤ 8 sample tiles) × CT ≤ 8 coils.
// A = conj(z^j) is generated (exact FP64-reduced start every 16 samples, complex step between),
// B = u and j·u are converted from the residual, ct_t comes from a small prep kernel's table.
// The readout's contribution then folds into each voxel's four results in the epilogue:
//   Jᴴu[0] += conj(T1ρ·∂T1m)·Y,  Jᴴu[1] += conj(T2ρ·∂T2m)·Y + conj(ΔtR2²·T2ρ·m)·Ỹ,  Jᴴu[2] += conj(m)·Y,
//   Jᴴu[3] = -i·Jᴴu[2].
// CTA: 128 voxels × CT coils × a readout range; 4 stages of 32 samples per readout; two TMEM
// accumulators (512 columns) alternate between readouts so the epilogue of readout r overlaps the
// MMAs of readout r + 1. Warps 0-7 generate A, 8-15 convert u, 16 issues the MMAs, 17-20 run the
// epilogue (one TMEM lane quarter each). Every wait is bounded.
#include <cuda_bf16.h>

#include <cstdlib>
#include <mutex>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {

void sum_partials(const CompasContext& ctx, const cfloat* partials, int nsplit, int64_t n, cfloat* out);

namespace kernels {

constexpr int TX_M = 128;          // voxels per CTA (TMEM lanes)
constexpr int TX_COLS = 32;        // complex samples j per stage (one 128-byte swizzle row)
constexpr int TX_KST = 128 / TX_COLS;  // stages per readout
constexpr int TX_TMAX = 8, TX_CTMAX = 8;
constexpr int TX_N = 32 * TX_CTMAX;    // 256 real columns: 32 per coil
constexpr int TX_STAGES = 2;
constexpr int TX_A_WARPS = 8, TX_B_WARPS = 8, TX_E_WARPS = 4;
constexpr int TX_MMA_WARP = TX_A_WARPS + TX_B_WARPS;
constexpr int TX_THREADS = (TX_A_WARPS + TX_B_WARPS + 1 + TX_E_WARPS) * 32;  // 672
constexpr int TX_A_BYTES = TX_M * TX_COLS * 4;   // 16 KB per hi/lo plane
constexpr int TX_B_BYTES = TX_N * TX_COLS * 4;   // 32 KB per hi/lo plane
constexpr int TX_STAGE = 2 * TX_A_BYTES + 2 * TX_B_BYTES;
constexpr int TX_SMEM = TX_STAGES * TX_STAGE + 1024 + 128;

struct TxArgs {
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
    int T, CT;                 // sample tiles (≤ 8), coils per CTA (≤ 8)
    int r_first, r_end;        // readouts [r_first, r_end) of this launch
    int readouts_per_split;    // readouts of one CTA
    int nsplit_launch;         // readout splits of this launch (gridDim.z)
    int partial0;              // first partial slot of this launch
    const float2* ct;          // [readouts of the launch][T][V] conj(rd·z^{128t})
    float2* out;               // [partials][4][V]
    unsigned int* status;
};

// ct[rr][t][v] = conj(rd_rv·z_rv^{128t}) for the launch's readouts, thread = (voxel, readout)
__global__ void tc_spiral_hermitian_prep_kernel(TxArgs a, float2* __restrict__ ct) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int rr = blockIdx.y, r = a.r_first + rr;
    if (v >= a.nvoxels) return;
    const double twopi = 6.283185307179586476925, inv_2pi = 0.15915494309189533577;
    const double half = 0.5 * double(a.S) * double(a.dt);
    const float2 ks = a.k_start[r], dkr = a.delta_k[r];
    const float T2 = a.params[a.pstride + v], B0 = a.params[3 * a.pstride + v];
    const float x = a.params[6 * a.pstride + v], y = a.params[7 * a.pstride + v];
    const float R2 = 1.0f / T2;
    const float dec = -a.dt * R2;
    // readout factor: rewind by (S/2)Δt, prephase with Re k0·x   (spiral_view.cuh:13-59)
    const float2 rd = cscale(expf(float(half) * R2), cis_rad(-half * twopi * double(B0) + double(ks.x) * double(x)));
    const double turns = (double(dkr.x) * x + double(dkr.y) * y + double(a.dt) * twopi * B0) * inv_2pi;
    for (int t = 0; t < a.T; t++) {
        const float2 ph = cis_turns(double(128 * t) * turns);
        const float mg = __expf(float(128 * t) * dec);
        ct[(int64_t(rr) * a.T + t) * a.nvoxels + v] = cconj(cmul(rd, make_float2(mg * ph.x, mg * ph.y)));
    }
}

__global__ void __launch_bounds__(TX_THREADS, 1) tc_spiral_hermitian_kernel(TxArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TX_STAGES * TX_STAGE);
    uint64_t* empty = full + TX_STAGES;
    uint64_t* acc_full = empty + TX_STAGES;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int v0 = blockIdx.x * TX_M;
    const int c0 = blockIdx.y * a.CT;
    const int split = blockIdx.z;
    const int rr_begin = split * a.readouts_per_split;  // readouts within the launch
    const int nread = max(0, min(a.readouts_per_split, a.r_end - (a.r_first + rr_begin)));
    const int nstages = nread * TX_KST;
    const int N = 32 * a.CT;
    const double twopi = 6.283185307179586476925, inv_2pi = 0.15915494309189533577;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TX_STAGES; s++) {
            tc::mbar_init(&full[s], (TX_A_WARPS + TX_B_WARPS) * 32);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            tc::mbar_init(&acc_full[b], 1);
            tc::mbar_init(&acc_empty[b], TX_E_WARPS * 32);
        }
        tc::mbar_init(done, 1);
        *abort_flag = 0;
        tc::fence_mbarrier_init();
    }
    if (warp == TX_MMA_WARP) tc::tmem_alloc(tmem_slot, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < TX_A_WARPS) {
        // ---------------- A: conj(z_v^j) for voxel row v, samples j = 32s + 16h .. +15 of each stage
        const int v = v0 + 32 * (warp & 3) + lane;
        const int row = 32 * (warp & 3) + lane;
        const int h = warp >> 2;
        const bool vok = v < a.nvoxels;
        float x = 0.f, y = 0.f, B0 = 0.f, dec = 0.f;
        if (vok) {
            x = a.params[6 * a.pstride + v];
            y = a.params[7 * a.pstride + v];
            B0 = a.params[3 * a.pstride + v];
            dec = -a.dt / a.params[a.pstride + v];
        }
        const float sm = __expf(dec);
        for (int g = 0; g < nstages; g++) {
            const int buf = g % TX_STAGES;
            const int rr = rr_begin + g / TX_KST, s = g % TX_KST;
            float2 e = make_float2(0.f, 0.f), zc = e;
            if (vok) {
                const float2 dkr = a.delta_k[a.r_first + rr];
                const double turns = (double(dkr.x) * x + double(dkr.y) * y + double(a.dt) * twopi * B0) * inv_2pi;
                const int j0 = TX_COLS * s + 16 * h;
                const float2 ph = cis_turns(double(j0) * turns);
                const float m0 = __expf(float(j0) * dec);
                e = make_float2(m0 * ph.x, -m0 * ph.y);  // conj(z^{j0})
                const float2 st = cis_turns(turns);
                zc = make_float2(sm * st.x, -sm * st.y);  // conj(z)
            }
            if (!tc::mbar_wait(&empty[buf], ((g / TX_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
            if (*(volatile int*)abort_flag) break;
            unsigned char* Ah = smem + buf * TX_STAGE;
            unsigned char* Al = Ah + TX_A_BYTES;
#pragma unroll
            for (int q = 0; q < 4; q++) {  // 4 chunks of 4 samples
                uint32_t hh[4], ll[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    tc::split2(e.x, e.y, hh[i], ll[i]);
                    e = cmul(e, zc);
                }
                const uint32_t off = tc::sw128_offset(row, 4 * h + q);
                *reinterpret_cast<uint4*>(Ah + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
                *reinterpret_cast<uint4*>(Al + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
        }
    } else if (warp < TX_MMA_WARP) {
        // ---------------- B: rows n = 32c + 4t + q of u[c][r][128t + j] — q = 0 (u_re, -u_im),
        // 1 (u_im, u_re), 2 and 3 the same of j·u; thread = (4-sample quad, (c, t) pairs p, p + 32)
        const int tb = threadIdx.x - 32 * TX_A_WARPS;
        const int quad = tb & 7, p0 = tb >> 3;
        const int npairs = a.CT * a.T;
        const bool vec16 = (a.S & 1) == 0 && (reinterpret_cast<uintptr_t>(a.u) & 15) == 0;
        float2 un[2][4];
        auto load = [&](int g, float2 (&dst)[2][4]) {
            const int r = a.r_first + rr_begin + g / TX_KST, s = g % TX_KST;
#pragma unroll
            for (int pi = 0; pi < 2; pi++) {
                const int p = p0 + 32 * pi;
                const int c = p / a.T, t = p - c * a.T;
                const int k = 128 * t + TX_COLS * s + 4 * quad;
#pragma unroll
                for (int i = 0; i < 4; i++) dst[pi][i] = make_float2(0.f, 0.f);
                if (p < npairs && c0 + c < a.C) {
                    const float2* urow = a.u + (int64_t(c0 + c) * a.R + r) * a.S;
                    if (vec16 && k + 4 <= a.S) {
                        const float4 x0 = __ldg(reinterpret_cast<const float4*>(urow + k));
                        const float4 x1 = __ldg(reinterpret_cast<const float4*>(urow + k + 2));
                        dst[pi][0] = make_float2(x0.x, x0.y);
                        dst[pi][1] = make_float2(x0.z, x0.w);
                        dst[pi][2] = make_float2(x1.x, x1.y);
                        dst[pi][3] = make_float2(x1.z, x1.w);
                    } else {
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            if (k + i < a.S) dst[pi][i] = __ldg(urow + k + i);
                    }
                }
            }
        };
        // the next stage's u is requested as soon as a stage is handed to the MMA
        if (nstages > 0) load(0, un);
        for (int g = 0; g < nstages; g++) {
            const int buf = g % TX_STAGES;
            const int s = g % TX_KST;
            if (!tc::mbar_wait(&empty[buf], ((g / TX_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
            if (*(volatile int*)abort_flag) break;
            unsigned char* Bh = smem + buf * TX_STAGE + 2 * TX_A_BYTES;
            unsigned char* Bl = Bh + TX_B_BYTES;
#pragma unroll
            for (int pi = 0; pi < 2; pi++) {
                const int p = p0 + 32 * pi;
                if (p >= npairs) break;
                const int c = p / a.T, t = p - c * a.T;
                uint32_t h0[4], l0[4], h1[4], l1[4], h2[4], l2[4], h3[4], l3[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float2 w = un[pi][i];
                    const float jf = float(TX_COLS * s + 4 * quad + i);
                    uint32_t hx, lx, hs, ls;
                    // one split per value: (x, -y) flips the upper sign bit, (y, x) swaps the halves
                    tc::split2(w.x, w.y, hx, lx);
                    tc::split2(jf * w.x, jf * w.y, hs, ls);
                    h0[i] = hx ^ 0x80000000u;
                    l0[i] = lx ^ 0x80000000u;
                    h1[i] = __byte_perm(hx, 0, 0x1032);
                    l1[i] = __byte_perm(lx, 0, 0x1032);
                    h2[i] = hs ^ 0x80000000u;
                    l2[i] = ls ^ 0x80000000u;
                    h3[i] = __byte_perm(hs, 0, 0x1032);
                    l3[i] = __byte_perm(ls, 0, 0x1032);
                }
                const int n = 32 * c + 4 * t;
                const uint32_t o0 = tc::sw128_offset(n, quad), o1 = tc::sw128_offset(n + 1, quad);
                const uint32_t o2 = tc::sw128_offset(n + 2, quad), o3 = tc::sw128_offset(n + 3, quad);
                *reinterpret_cast<uint4*>(Bh + o0) = make_uint4(h0[0], h0[1], h0[2], h0[3]);
                *reinterpret_cast<uint4*>(Bl + o0) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
                *reinterpret_cast<uint4*>(Bh + o1) = make_uint4(h1[0], h1[1], h1[2], h1[3]);
                *reinterpret_cast<uint4*>(Bl + o1) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
                *reinterpret_cast<uint4*>(Bh + o2) = make_uint4(h2[0], h2[1], h2[2], h2[3]);
                *reinterpret_cast<uint4*>(Bl + o2) = make_uint4(l2[0], l2[1], l2[2], l2[3]);
                *reinterpret_cast<uint4*>(Bh + o3) = make_uint4(h3[0], h3[1], h3[2], h3[3]);
                *reinterpret_cast<uint4*>(Bl + o3) = make_uint4(l3[0], l3[1], l3[2], l3[3]);
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
            if (g + 1 < nstages) load(g + 1, un);
        }
    } else if (warp == TX_MMA_WARP) {
        // ---------------- MMA issuer (one lane): per readout 4 stages into accumulator rr & 1
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16_f32(TX_M, N);
            for (int ri = 0; ri < nread && !*(volatile int*)abort_flag; ri++) {
                const int ab = ri & 1;
                if (ri >= 2 && !tc::mbar_wait(&acc_empty[ab], ((ri >> 1) - 1) & 1, a.status)) {
                    *abort_flag = 1;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t d = tmem + uint32_t(ab * 256);
                for (int s = 0; s < TX_KST; s++) {
                    const int g = ri * TX_KST + s;
                    const int buf = g % TX_STAGES;
                    if (!tc::mbar_wait(&full[buf], (g / TX_STAGES) & 1, a.status)) *abort_flag = 1;
                    if (*(volatile int*)abort_flag) break;
                    tc::tc_fence_after();
                    const uint32_t base = tc::smem_u32(smem + buf * TX_STAGE);
                    const uint32_t ah = base, al = base + TX_A_BYTES;
                    const uint32_t bh = base + 2 * TX_A_BYTES, bl = bh + TX_B_BYTES;
#pragma unroll
                    for (int k16 = 0; k16 < 2 * TX_COLS / 16; k16++) {
                        const uint32_t koff = k16 * 32;
                        const uint64_t dah = tc::sw128_kmajor_desc(ah + koff), dal = tc::sw128_kmajor_desc(al + koff);
                        const uint64_t dbh = tc::sw128_kmajor_desc(bh + koff), dbl = tc::sw128_kmajor_desc(bl + koff);
                        tc::mma_bf16(d, dah, dbh, idesc, (s > 0 || k16 > 0) ? 1u : 0u);
                        tc::mma_bf16(d, dah, dbl, idesc, 1u);
                        tc::mma_bf16(d, dal, dbh, idesc, 1u);
                    }
                    tc::mma_commit(&empty[buf]);
                }
                tc::mma_commit(&acc_full[ab]);
            }
            tc::mma_commit(done);
            tc::mbar_wait(done, 0, a.status);  // all MMAs complete before TMEM is released
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: thread = voxel = TMEM lane 32·quarter + lane
        const int quarter = warp & 3;
        const int v = v0 + 32 * quarter + lane;
        const bool vok = v < a.nvoxels;
        const int vc = vok ? v : a.nvoxels - 1;
        const float T1 = a.params[vc], T2 = a.params[a.pstride + vc];
        const float2 rho = make_float2(a.params[4 * a.pstride + vc], a.params[5 * a.pstride + vc]);
        const float R2 = 1.0f / T2;
        const float2 t1r = cscale(T1, rho), t2r = cscale(T2, rho);
        const float2 t2rq = cscale(a.dt * R2 * R2, t2r);
        float2 out0 = make_float2(0.f, 0.f), out1 = out0, out2 = out0;
        bool ok = true;
        for (int ri = 0; ri < nread; ri++) {
            const int ab = ri & 1;
            const int rr = rr_begin + ri, r = a.r_first + rr;
            // this readout's factors (loads in flight while the accumulator fills)
            float2 ctv[TX_TMAX];
#pragma unroll
            for (int t = 0; t < TX_TMAX; t++)
                ctv[t] = (vok && t < a.T) ? a.ct[(int64_t(rr) * a.T + t) * a.nvoxels + v] : make_float2(0.f, 0.f);
            float2 me = make_float2(0.f, 0.f), d1 = me, d2 = me;
            if (vok) {
                const int64_t idx = int64_t(r) * a.nvoxels + v;
                me = a.echo[idx];
                d1 = a.dT1[idx];
                d2 = a.dT2[idx];
            }
            const bool waited = tc::mbar_wait(&acc_full[ab], (ri >> 1) & 1, a.status);
            tc::tc_fence_after();
            if (!__all_sync(0xffffffffu, waited && !*(volatile int*)abort_flag)) {
                *abort_flag = 1;
                ok = false;
                break;
            }
            float2 Y = make_float2(0.f, 0.f), Yt = Y;
            for (int c = 0; c < a.CT; c++) {
                float2 X = make_float2(0.f, 0.f), Xt = X;
#pragma unroll
                for (int hf = 0; hf < 2; hf++) {  // sample tiles 4·hf .. 4·hf + 3 (16 columns)
                    if (4 * hf >= a.T) break;
                    float dv[16];
                    tc::tmem_load16(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(ab * 256 + 32 * c + 16 * hf), dv);
#pragma unroll
                    for (int tt = 0; tt < 4; tt++) {
                        const int t = 4 * hf + tt;
                        if (t >= a.T) break;
                        const float2 G = make_float2(dv[4 * tt], dv[4 * tt + 1]);
                        const float2 Gt = make_float2(dv[4 * tt + 2], dv[4 * tt + 3]);
                        const float w = float(128 * t) - 0.5f * float(a.S);
                        X = cadd(X, cmul(ctv[t], G));
                        Xt = cadd(Xt, cmul(ctv[t], make_float2(fmaf(w, G.x, Gt.x), fmaf(w, G.y, Gt.y))));
                    }
                }
                // conj(coil) of this voxel (a small table that stays in L1)
                const float2 ccv = (vok && c0 + c < a.C) ? cconj(__ldg(a.coils + int64_t(c0 + c) * a.nvoxels + v))
                                                         : make_float2(0.f, 0.f);
                Y = cadd(Y, cmul(ccv, X));
                Yt = cadd(Yt, cmul(ccv, Xt));
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&acc_empty[ab]);
            out0 = cadd(out0, cmulc(Y, cmul(t1r, d1)));
            out1 = cadd(out1, cadd(cmulc(Y, cmul(t2r, d2)), cmulc(Yt, cmul(t2rq, me))));
            out2 = cadd(out2, cmulc(Y, me));
        }
        if (ok && vok && !*(volatile int*)abort_flag) {
            const int slot = a.partial0 + blockIdx.y * a.nsplit_launch + split;
            float2* o = a.out + int64_t(slot) * 4 * a.nvoxels;
            o[v] = out0;
            o[a.nvoxels + v] = out1;
            o[2 * int64_t(a.nvoxels) + v] = out2;
            o[3 * int64_t(a.nvoxels) + v] = make_float2(out2.y, -out2.x);  // -i·out2
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == TX_MMA_WARP) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

}  // namespace kernels

// readout splits within one readout chunk of the spiral Jᴴ·v contraction: the tuned count (at most
// one readout each), else the fewest splits, each of at least 4 readouts, whose grid of voxel tiles ×
// coil groups × splits (one CTA per SM) spans two waves or more with the last wave at least 95 %
// full, or failing that the best-filled grid of at most 16 splits (30000 voxels at 16 coils: 470
// CTAs per split are 3.2 waves, 79 % of the SM time in use; 3 splits: 9.5 waves, 95 %). Returned as
// the count the launches run (every split non-empty). Each readout's accumulation is drained
// separately, so the count changes only the partial sums.
int tc_spiral_hermitian_splits(int device, int nvoxels, int R, int S, int C) {
    const int T = div_ceil(std::max(S, 1), kernels::TX_M);
    const int chunk = spiral_table_chunk(int64_t(T) * nvoxels * int64_t(sizeof(float2)), R);
    const TcTuning tuning = tuned_tc(TcKind::SpiralHermitian, R, nvoxels, int64_t(C) * S);
    int splits = 1;
    if (tuning.splits > 0) {
        splits = std::max(1, std::min(tuning.splits, chunk));
    } else {
        const int64_t base = int64_t(div_ceil(C, kernels::TX_CTMAX)) * div_ceil(std::max(nvoxels, 1), kernels::TX_M);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int most = std::max(1, std::min(16, div_ceil(chunk, 4)));
        double best_fill = -1.0;
        for (int s = 1; s <= most; s++) {
            const int64_t ctas = base * s;
            const int64_t waves = (ctas + sms - 1) / sms;
            const double fill = double(ctas) / double(waves * sms);
            if (ctas >= 2 * sms && fill >= 0.95) {
                splits = s;
                break;
            }
            if (fill > best_fill + 1e-9) {
                best_fill = fill;
                splits = s;
            }
        }
    }
    return div_ceil(chunk, div_ceil(chunk, splits));
}

bool launch_jacobian_hermitian_spiral_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                         const cfloat* echos, const cfloat* dT1, const cfloat* dT2,
                                         const cfloat* coils, int ncoils, const cfloat* vec, int nreadouts, int ns,
                                         float dt, const cfloat* k_start, const cfloat* delta_k, cfloat* JHv) {
    if (!tensor_cores_available(ctx.device())) return false;
    const int T = div_ceil(std::max(ns, 1), 128);
    if (T > kernels::TX_TMAX) return false;  // readouts of more than 1024 samples: FP32 kernel
    if (nvoxels == 0) return true;
    DeviceGuard guard(ctx.device());
    const int64_t n = 4 * int64_t(nvoxels);
    if (int64_t(ncoils) * nreadouts * ns == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(JHv, 0, sizeof(cfloat) * size_t(n), ctx.stream()));
        return true;
    }
    kernels::TxArgs a {};
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
    a.T = T;
    a.status = ctx.status_word();
    const int groups = div_ceil(ncoils, kernels::TX_CTMAX);
    a.CT = div_ceil(ncoils, groups);
    const int vtiles = div_ceil(nvoxels, kernels::TX_M);
    // readouts in chunks whose ct table ([readouts][T][V] complex) stays near 1 GB
    // (COMPAS_B200_SPIRAL_TABLE_BYTES overrides the budget; it changes only the order in which the
    // readouts' contributions are summed)
    const int chunk = spiral_table_chunk(int64_t(T) * nvoxels * int64_t(sizeof(float2)), nreadouts);
    const int nchunks = div_ceil(nreadouts, chunk);
    const int splits = tc_spiral_hermitian_splits(ctx.device(), nvoxels, nreadouts, ns, ncoils);
    // per chunk: its readouts in `splits` near-equal parts (the last chunk may be a readout shorter)
    auto chunk_splits = [&](int rc, int* per_split) {
        *per_split = div_ceil(rc, std::min(splits, rc));
        return div_ceil(rc, *per_split);
    };
    int nparts = 0;
    for (int ci = 0; ci < nchunks; ci++) {
        int per_split = 0;
        nparts += groups * chunk_splits(std::min(chunk, nreadouts - ci * chunk), &per_split);
    }
    Array<cfloat, 2> partials({nparts > 1 ? nparts : 0, n}, ctx.device(), ctx.stream());
    a.out = reinterpret_cast<float2*>(nparts > 1 ? partials.data() : JHv);
    Array<cfloat, 2> table({std::min(chunk, nreadouts), int64_t(T) * nvoxels}, ctx.device(), ctx.stream());
    a.ct = reinterpret_cast<const float2*>(table.data());
    static std::once_flag once;
    std::call_once(once, [] {
        COMPAS_CUDA_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(kernels::tc_spiral_hermitian_kernel),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, kernels::TX_SMEM));
    });
    a.partial0 = 0;
    for (int ci = 0; ci < nchunks; ci++) {
        a.r_first = ci * chunk;
        const int rc = std::min(chunk, nreadouts - a.r_first);
        a.r_end = a.r_first + rc;
        a.nsplit_launch = chunk_splits(rc, &a.readouts_per_split);
        kernels::tc_spiral_hermitian_prep_kernel<<<dim3(div_ceil(nvoxels, 128), rc), 128, 0, ctx.stream()>>>(
            a, reinterpret_cast<float2*>(table.data()));
        // every split of the launch has readouts (chunk_splits)
        kernels::tc_spiral_hermitian_kernel<<<dim3(vtiles, groups, a.nsplit_launch), kernels::TX_THREADS,
                                              kernels::TX_SMEM, ctx.stream()>>>(a);
        check_launch("tc_spiral_hermitian_kernel");
        a.partial0 += groups * a.nsplit_launch;
    }
    if (nparts > 1) sum_partials(ctx, partials.data(), nparts, n, JHv);
    return true;
}

}  // namespace compas
