// tc_spiral.cu — split-BF16 tcgen05 kernels for the spiral signal and the spiral J·v.
//
// Spiral signal (reference: src/trajectories/signal_kernels.cuh:274-345, spiral_view.cuh:13-73):
//   s[c][r][k] = Σ_v C[c][v]·A_rv·z_rv^k,  A_rv = ρ_v·m[r][v]·rewind_rv,  z_rv = e^{-Δt R2 + iΘ_rv}.
// Writing the sample as k = 128·t + j gives z^k = z^{128t}·z^j, so for one readout
//   s[c][r][128t + j] = Σ_v P[j][v]·W[v][(t, c)],   P[j][v] = z_rv^j,   W[v][(t, c)] = z_rv^{128t}·A_rv·C[c][v]
// is one GEMM with M = 128 (j, the TMEM lanes), N = 2·T·CT real columns (all T sample tiles × CT
// coils of the readout at once) and K = the voxels: the generated tile P serves every sample tile,
// and the sample-tile offset z^{128t} moves into the small per-voxel operand W.
// A CTA owns one readout, CT coils and a voxel range (split-K, ≤ 512 K16 steps per split so the
// tensor core's FP32 accumulation stays accurate; partial tiles are summed in a fixed order):
//   warps 0-7   generate P for 128 samples × 32 complex columns per stage: 16 consecutive samples
//               per thread from an exact start z^{16g} (phase reduced modulo 2π in FP64) and the
//               complex step z; split FP32 → BF16 hi + lo into the 128-byte-swizzled K-major tile;
//   warps 8-15  form W for every sample tile t: the base z^{128t}·source (exact, FP64-reduced
//               phase) comes from a small prep kernel's table for the launch's readouts, times each
//               coil; real-ified as the rows (W_re, -W_im), (W_im, W_re);
//   warp 16     allocates 256 TMEM columns and one lane issues 3 tcgen05.mma per K16 step
//               (hi·hi + hi·lo + lo·hi, FP32 accumulation);
//   warps 0-15  afterwards read the accumulator (lane = sample j) and write the tile.
// J·v on a spiral (no counterpart in the reference) uses two columns per voxel: with source P_rv
// for z^k and Q_rv for (k - S/2)·z^k (P, Q as in the FP32 spiral J·v),
//   (k - S/2)·z^k = z^{128t}·[(128t - S/2)·z^j + j·z^j],
// so the A columns are z^j and j·z^j and the W rows z^{128t}·C·(P + (128t - S/2)·Q) and z^{128t}·C·Q.
// Every wait is bounded.
#include <cuda_bf16.h>

#include <cstdlib>
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {

void sum_partials(const CompasContext& ctx, const cfloat* partials, int nsplit, int64_t n, cfloat* out);

namespace kernels {

constexpr int TS_M = 128;        // samples j per tile (TMEM lanes)
constexpr int TS_COLS = 32;      // complex K columns per stage (one 128-byte swizzle row)
constexpr int TS_NMAX = 256;     // real N columns (2·T·CT)
constexpr int TS_STAGES = 2;
constexpr int TS_A_WARPS = 8, TS_B_WARPS = 8;
constexpr int TS_MMA_WARP = TS_A_WARPS + TS_B_WARPS;
constexpr int TS_PRODUCERS = (TS_A_WARPS + TS_B_WARPS) * 32;  // 512
constexpr int TS_THREADS = TS_PRODUCERS + 32;                 // 544
constexpr int TS_A_BYTES = TS_M * TS_COLS * 2 * 2;            // 16 KB per hi/lo plane
constexpr int TS_B_BYTES = TS_NMAX * TS_COLS * 2 * 2;         // 32 KB per hi/lo plane
constexpr int TS_STAGE = 2 * TS_A_BYTES + 2 * TS_B_BYTES;
constexpr int TS_SMEM = TS_STAGES * TS_STAGE + 1024 + 128;

struct TsArgs {
    const float* params;
    int64_t pstride;
    int nvoxels;
    const float2* echo;
    const float2* dT1;  // J·v only
    const float2* dT2;
    const float2* vec;  // J·v only: [4][V]
    const float2* coils;
    int R, S, C;
    float dt;
    const float2* k_start;
    const float2* delta_k;
    int T, CT;     // sample tiles per readout, coils per CTA (2·T·CT ≤ 256)
    int vchunk;    // voxels per split (a multiple of the voxels per stage)
    int r_first;   // first readout of this launch (blockIdx.x = r - r_first)
    const float2* base;  // [readouts of the launch][TERMS][T][V] z^{128t}·source (tc_spiral_base_kernel)
    float2* out;   // [splits][C][R][S]
    unsigned int* status;
};

// The per-voxel operand factors of one launch's readouts: thread = (voxel, readout). Source
// (signal: ρ·m·rewind; J·v: rewind·P and rewind·Q'), then for every sample tile t the exact
// z^{128t} (phase reduced modulo 2π in FP64) times the source (J·v: times P + (128t - S/2)·Q' and Q').
template<bool JAC>
__global__ void tc_spiral_base_kernel(TsArgs a, float2* __restrict__ base) {
    constexpr int TERMS = JAC ? 2 : 1;
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int rr = blockIdx.y, r = a.r_first + rr;
    if (v >= a.nvoxels) return;
    const double twopi = 6.283185307179586476925, inv_2pi = 0.15915494309189533577;
    const double hdt = 0.5 * double(a.S) * double(a.dt);
    const float2 ks = a.k_start[r], dkr = a.delta_k[r];
    const int64_t idx = int64_t(r) * a.nvoxels + v;
    const float T2 = a.params[a.pstride + v], B0 = a.params[3 * a.pstride + v];
    const float x = a.params[6 * a.pstride + v], y = a.params[7 * a.pstride + v];
    const float2 rho = make_float2(a.params[4 * a.pstride + v], a.params[5 * a.pstride + v]);
    const float2 me = a.echo[idx];
    const float R2 = 1.0f / T2;
    const float dec = -a.dt * R2;
    const double turns = (double(dkr.x) * x + double(dkr.y) * y + double(a.dt) * twopi * B0) * inv_2pi;
    // rewind by (S/2)Δt and prephase with Re k0·x   (spiral_view.cuh:13-59)
    const float2 rw = cis_rad(-hdt * twopi * double(B0) + double(ks.x) * double(x));
    const float2 rd = cscale(expf(float(hdt) * R2), rw);
    float2 s0, s1 = make_float2(0.f, 0.f);
    if constexpr (!JAC) {
        s0 = cmul(cmul(me, rd), rho);
    } else {
        const float T1 = a.params[v];
        const float2 w0 = a.vec[v], w1 = a.vec[a.nvoxels + v];
        const float2 w2 = a.vec[2 * int64_t(a.nvoxels) + v], w3 = a.vec[3 * int64_t(a.nvoxels) + v];
        const float2 c1 = cmul(w0, cscale(T1, rho)), c2 = cmul(w1, cscale(T2, rho));
        const float2 cm = make_float2(w2.x - w3.y, w2.y + w3.x);
        s0 = cmul(rd, cadd(cadd(cmul(c1, a.dT1[idx]), cmul(c2, a.dT2[idx])), cmul(cm, me)));
        s1 = cmul(rd, cmul(cscale(a.dt * R2 * R2, c2), me));
    }
    for (int t = 0; t < a.T; t++) {
        const float2 ph = cis_turns(double(128 * t) * turns);
        const float mg = __expf(float(128 * t) * dec);
        const float2 zt = make_float2(mg * ph.x, mg * ph.y);
        const int64_t o = ((int64_t(rr) * TERMS) * a.T + t) * a.nvoxels + v;
        if constexpr (!JAC) {
            base[o] = cmul(zt, s0);
        } else {
            base[o] = cmul(zt, cadd(s0, cscale(float(128 * t) - 0.5f * float(a.S), s1)));
            base[o + int64_t(a.T) * a.nvoxels] = cmul(zt, s1);
        }
    }
}

template<bool JAC>
__global__ void __launch_bounds__(TS_THREADS, 1) tc_spiral_kernel(TsArgs a) {
    constexpr int TERMS = JAC ? 2 : 1;
    constexpr int VPS = TS_COLS / TERMS;  // voxels per stage
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TS_STAGES * TS_STAGE);
    uint64_t* empty = full + TS_STAGES;
    uint64_t* done = empty + TS_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = a.r_first + blockIdx.x;
    const int c0 = blockIdx.y * a.CT;
    const int split = blockIdx.z;
    const int v_begin = split * a.vchunk;
    const int v_end = min(a.nvoxels, v_begin + a.vchunk);
    const int nstages = max(1, (v_end - v_begin + VPS - 1) / VPS);
    const int N = (2 * a.T * a.CT + 15) / 16 * 16;  // MMA columns; those past 2·T·CT are never read
    const double twopi = 6.283185307179586476925, inv_2pi = 0.15915494309189533577;
    const float2 dkr = a.delta_k[r];

    if (threadIdx.x == 0) {
        for (int s = 0; s < TS_STAGES; s++) {
            tc::mbar_init(&full[s], TS_PRODUCERS);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(done, 1);
        *abort_flag = 0;
        tc::fence_mbarrier_init();
    }
    if (warp == TS_MMA_WARP) tc::tmem_alloc(tmem_slot, 256);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // column jc = lane of this stage: voxel v_begin + it·VPS + jc / TERMS, term jc % TERMS
    const int jc = lane;
    const int term = jc % TERMS;
    const uint32_t col_off = uint32_t(jc & 3) * 4;
    auto voxel = [&](int it) { return v_begin + it * VPS + jc / TERMS; };

    if (warp < TS_A_WARPS) {
        // ---------------- P producer: samples j = 16g .. 16g + 15 of column jc
        const int g = warp;
        float4 pn;  // {x, y, B0, T2} of the next stage's voxel
        auto load = [&](int it, float4& p) {
            const int v = voxel(it);
            p = v < v_end ? make_float4(a.params[6 * a.pstride + v], a.params[7 * a.pstride + v],
                                        a.params[3 * a.pstride + v], a.params[a.pstride + v])
                          : make_float4(0.f, 0.f, 0.f, 0.f);
        };
        load(0, pn);
        for (int it = 0; it < nstages; it++) {
            const int buf = it % TS_STAGES;
            const float4 pc = pn;
            if (it + 1 < nstages) load(it + 1, pn);
            float2 z = make_float2(0.f, 0.f), step = z;
            if (voxel(it) < v_end) {
                const float dec = -a.dt / pc.w;
                const double turns = (double(dkr.x) * pc.x + double(dkr.y) * pc.y + double(a.dt) * twopi * pc.z) * inv_2pi;
                const float2 ph = cis_turns(double(16 * g) * turns);
                const float m0 = __expf(float(16 * g) * dec);
                z = make_float2(m0 * ph.x, m0 * ph.y);
                step = cscale(__expf(dec), cis_turns(turns));
            }
            if (!tc::mbar_wait(&empty[buf], ((it / TS_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
            if (*(volatile int*)abort_flag) break;
            unsigned char* Ah = smem + buf * TS_STAGE;
            unsigned char* Al = Ah + TS_A_BYTES;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int j = 16 * g + i;
                float2 e = z;
                if (JAC && term == 1) e = make_float2(float(j) * z.x, float(j) * z.y);
                uint32_t h, l;
                tc::split2(e.x, e.y, h, l);
                const uint32_t off = tc::sw128_offset(j, jc >> 2) + col_off;
                *reinterpret_cast<uint32_t*>(Ah + off) = h;
                *reinterpret_cast<uint32_t*>(Al + off) = l;
                z = cmul(z, step);
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
        }
    } else if (warp < TS_MMA_WARP && JAC && a.CT >= 4) {
        // J·v with at least four coils per CTA: 16-byte rows (J·v 26.4 -> 21.9 ms at 16 coils,
        // 30000 voxels x 760 x 1000; the per-column form below is faster for the signal and for
        // fewer coils)
        // ---------------- W producer: sample tiles t = warp - 8, warp, …; lane = (column quad
        // q = lane & 7, coil subset cs = lane >> 3): columns 4q .. 4q + 3 of the coils cs, cs + 4, …,
        // so every row is written as 16-byte chunks. The bases z^{128t}·source come from the prep
        // kernel's table; the first sample tile's bases and the first four coils of the subset are
        // requested for the next stage as soon as a stage is handed to the MMA.
        constexpr int CPRE = 4;
        const int q = lane & 7, cs = lane >> 3;
        const int t0 = warp - TS_A_WARPS;
        auto col_voxel = [&](int it, int i) { return v_begin + it * VPS + (4 * q + i) / TERMS; };
        auto col_base = [&](int i) {  // base table row of column 4q + i (its term)
            return a.base + (int64_t(blockIdx.x) * TERMS + (4 * q + i) % TERMS) * a.T * a.nvoxels;
        };
        float2 bn[4], cvn[CPRE][4];
        auto load = [&](int it) {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int v = col_voxel(it, i);
                const bool ok = v < v_end;
                bn[i] = (ok && t0 < a.T) ? __ldg(col_base(i) + int64_t(t0) * a.nvoxels + v) : make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < CPRE; k++) {
                    const int c = cs + 4 * k;
                    cvn[k][i] = (ok && c < a.CT && c0 + c < a.C) ? __ldg(a.coils + int64_t(c0 + c) * a.nvoxels + v)
                                                                 : make_float2(0.f, 0.f);
                }
            }
        };
        load(0);
        for (int it = 0; it < nstages; it++) {
            const int buf = it % TS_STAGES;
            // bn and cvn hold this stage's values until the next stage's load (after the hand-over)
            if (!tc::mbar_wait(&empty[buf], ((it / TS_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
            if (*(volatile int*)abort_flag) break;
            unsigned char* Bh = smem + buf * TS_STAGE + 2 * TS_A_BYTES;
            unsigned char* Bl = Bh + TS_B_BYTES;
            // W = coil·base of the four columns → rows (W_re, -W_im), (W_im, W_re): one split per value,
            // the upper sign bit flipped for the first row and the halves swapped for the second
            auto emit = [&](int t, int c, const float2 (&W)[4]) {
                uint32_t h[4], l[4];
#pragma unroll
                for (int i = 0; i < 4; i++) tc::split2(W[i].x, W[i].y, h[i], l[i]);
                const int row = 2 * (t * a.CT + c);
                const uint32_t o0 = tc::sw128_offset(row, q), o1 = tc::sw128_offset(row + 1, q);
                *reinterpret_cast<uint4*>(Bh + o0) =
                    make_uint4(h[0] ^ 0x80000000u, h[1] ^ 0x80000000u, h[2] ^ 0x80000000u, h[3] ^ 0x80000000u);
                *reinterpret_cast<uint4*>(Bl + o0) =
                    make_uint4(l[0] ^ 0x80000000u, l[1] ^ 0x80000000u, l[2] ^ 0x80000000u, l[3] ^ 0x80000000u);
                *reinterpret_cast<uint4*>(Bh + o1) =
                    make_uint4(__byte_perm(h[0], 0, 0x1032), __byte_perm(h[1], 0, 0x1032), __byte_perm(h[2], 0, 0x1032),
                               __byte_perm(h[3], 0, 0x1032));
                *reinterpret_cast<uint4*>(Bl + o1) =
                    make_uint4(__byte_perm(l[0], 0, 0x1032), __byte_perm(l[1], 0, 0x1032), __byte_perm(l[2], 0, 0x1032),
                               __byte_perm(l[3], 0, 0x1032));
            };
            for (int t = t0; t < a.T; t += TS_B_WARPS) {
                float2 base[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int v = col_voxel(it, i);
                    base[i] = t == t0 ? bn[i] : (v < v_end ? __ldg(col_base(i) + int64_t(t) * a.nvoxels + v)
                                                           : make_float2(0.f, 0.f));
                }
#pragma unroll
                for (int k = 0; k < CPRE; k++) {
                    const int c = cs + 4 * k;
                    if (c >= a.CT) break;
                    float2 W[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) W[i] = cmul(cvn[k][i], base[i]);
                    emit(t, c, W);
                }
                // more than 16 coils per CTA (readouts of at most 896 samples): the rest loaded here
                for (int c = cs + 4 * CPRE; c < a.CT; c += 4) {
                    float2 W[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const int v = col_voxel(it, i);
                        const float2 cw = (v < v_end && c0 + c < a.C) ? __ldg(a.coils + int64_t(c0 + c) * a.nvoxels + v)
                                                                      : make_float2(0.f, 0.f);
                        W[i] = cmul(cw, base[i]);
                    }
                    emit(t, c, W);
                }
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
            if (it + 1 < nstages) load(it + 1);
        }
    } else if (warp < TS_MMA_WARP) {
        // ---------------- W producer: sample tiles t = warp - 8, warp, … of column jc. The bases
        // z^{128t}·source come from the prep kernel's table; the base and the first 16 coil factors
        // of the next stage are requested as soon as a stage is handed to the MMA.
        constexpr int CPRE = 16;
        const int t0 = warp - TS_A_WARPS;
        const float2* brow = a.base + (int64_t(blockIdx.x) * TERMS + term) * a.T * a.nvoxels;
        float2 bn = make_float2(0.f, 0.f), cv[CPRE];
        auto load = [&](int it) {
            const int v = voxel(it);
            const bool ok = v < v_end;
            bn = (ok && t0 < a.T) ? __ldg(brow + int64_t(t0) * a.nvoxels + v) : make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < CPRE; c++)
                cv[c] = (ok && c < a.CT && c0 + c < a.C) ? __ldg(a.coils + int64_t(c0 + c) * a.nvoxels + v)
                                                         : make_float2(0.f, 0.f);
        };
        load(0);
        for (int it = 0; it < nstages; it++) {
            const int buf = it % TS_STAGES;
            const int v = voxel(it);
            const bool vok = v < v_end;
            const float2 b0 = bn;
            if (!tc::mbar_wait(&empty[buf], ((it / TS_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
            if (*(volatile int*)abort_flag) break;
            unsigned char* Bh = smem + buf * TS_STAGE + 2 * TS_A_BYTES;
            unsigned char* Bl = Bh + TS_B_BYTES;
            // W = coil·base → rows (W_re, -W_im), (W_im, W_re): one split, the upper sign bit flipped
            // for the first row and the halves swapped for the second
            auto emit = [&](int t, int c, float2 W) {
                uint32_t h, l;
                tc::split2(W.x, W.y, h, l);
                const int row = 2 * (t * a.CT + c);
                const uint32_t o0 = tc::sw128_offset(row, jc >> 2) + col_off;
                const uint32_t o1 = tc::sw128_offset(row + 1, jc >> 2) + col_off;
                *reinterpret_cast<uint32_t*>(Bh + o0) = h ^ 0x80000000u;
                *reinterpret_cast<uint32_t*>(Bl + o0) = l ^ 0x80000000u;
                *reinterpret_cast<uint32_t*>(Bh + o1) = __byte_perm(h, 0, 0x1032);
                *reinterpret_cast<uint32_t*>(Bl + o1) = __byte_perm(l, 0, 0x1032);
            };
            for (int t = t0; t < a.T; t += TS_B_WARPS) {
                const float2 base = t == t0 ? b0 : (vok ? __ldg(brow + int64_t(t) * a.nvoxels + v) : make_float2(0.f, 0.f));
#pragma unroll
                for (int c = 0; c < CPRE; c++) {
                    if (c >= a.CT) break;
                    emit(t, c, cmul(cv[c], base));
                }
                // more than 16 coils per CTA (readouts of at most 896 samples): groups of 8
                for (int cb = CPRE; cb < a.CT; cb += 8) {
                    float2 cw[8];
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const int cc = c0 + cb + c;
                        cw[c] = (vok && cb + c < a.CT && cc < a.C) ? __ldg(a.coils + int64_t(cc) * a.nvoxels + v)
                                                                   : make_float2(0.f, 0.f);
                    }
#pragma unroll
                    for (int c = 0; c < 8; c++)
                        if (cb + c < a.CT) emit(t, cb + c, cmul(cw[c], base));
                }
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
            if (it + 1 < nstages) load(it + 1);
        }
    } else {
        // ---------------- MMA issuer (one lane)
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16_f32(TS_M, N);
            for (int it = 0; it < nstages; it++) {
                const int buf = it % TS_STAGES;
                if (!tc::mbar_wait(&full[buf], (it / TS_STAGES) & 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::tc_fence_after();
                const uint32_t base = tc::smem_u32(smem + buf * TS_STAGE);
                const uint32_t ah = base, al = base + TS_A_BYTES;
                const uint32_t bh = base + 2 * TS_A_BYTES, bl = bh + TS_B_BYTES;
#pragma unroll
                for (int k16 = 0; k16 < 2 * TS_COLS / 16; k16++) {
                    const uint32_t koff = k16 * 32;  // 16 bf16 = 32 bytes along K inside the swizzle atom
                    const uint64_t dah = tc::sw128_kmajor_desc(ah + koff), dal = tc::sw128_kmajor_desc(al + koff);
                    const uint64_t dbh = tc::sw128_kmajor_desc(bh + koff), dbl = tc::sw128_kmajor_desc(bl + koff);
                    tc::mma_bf16(tmem, dah, dbh, idesc, (it > 0 || k16 > 0) ? 1u : 0u);
                    tc::mma_bf16(tmem, dah, dbl, idesc, 1u);
                    tc::mma_bf16(tmem, dal, dbh, idesc, 1u);
                }
                tc::mma_commit(&empty[buf]);
            }
            tc::mma_commit(done);
            tc::mbar_wait(done, 0, a.status);  // the MMAs finish before the TMEM is released
        }
        __syncwarp();
    }

    if (warp < TS_MMA_WARP) {
        // ---------------- epilogue: lane = sample j of quarter warp%4; the quarter's four warps take
        // alternate 8-column chunks (4 (t, c) pairs each)
        const bool waited = tc::mbar_wait(done, 0, a.status);
        tc::tc_fence_after();
        const bool ok = !tc::bar_red_or(1, TS_PRODUCERS, !(waited && !*(volatile int*)abort_flag));
        if (ok) {
            const int quarter = warp & 3;
            const int j = quarter * 32 + lane;
            float2* outp = a.out + int64_t(split) * a.C * a.R * a.S;
            for (int ch = warp >> 2; ch < N / 8; ch += 4) {
                float v[8];
                tc::tmem_load8(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(ch * 8), v);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int p = ch * 4 + i;  // (t, c) pair
                    const int t = p / a.CT, c = p - t * a.CT;
                    const int k = 128 * t + j;
                    if (t < a.T && k < a.S && c0 + c < a.C)
                        outp[(int64_t(c0 + c) * a.R + r) * a.S + k] = make_float2(v[2 * i], v[2 * i + 1]);
                }
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == TS_MMA_WARP) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 256);
    }
}

}  // namespace kernels

// readouts per chunk of a spiral contraction whose per-readout table takes `per_readout_bytes`: the
// tables of one chunk stay near 1 GB (COMPAS_B200_SPIRAL_TABLE_BYTES overrides the budget)
int spiral_table_chunk(int64_t per_readout_bytes, int R) {
    int64_t budget = int64_t(1) << 30;
    if (const char* e = std::getenv("COMPAS_B200_SPIRAL_TABLE_BYTES")) budget = std::max<int64_t>(1, std::atoll(e));
    const int64_t most = std::max<int64_t>(1, std::min<int64_t>(R, budget / std::max<int64_t>(1, per_readout_bytes)));
    // as many chunks as the budget needs, of equal size (759 readouts: 380 + 379, not 559 + 200)
    const int64_t nchunks = std::max<int64_t>(1, (int64_t(R) + most - 1) / most);
    return int(std::max<int64_t>(1, (int64_t(R) + nchunks - 1) / nchunks));
}

// voxel splits of the spiral signal / J·v contraction: at least enough for ≤ 512 K16 steps each
// (4096 voxels of the signal, 2048 of J·v); then the tuned count (≤ 64, ≥ one voxel stage each), or
// else enough CTAs to fill the GPU twice (≥ 8 stages each); returned as the count the launch runs
int tc_spiral_splits(int device, int nvoxels, int R, int S, int C, bool jac) {
    const int T = div_ceil(std::max(S, 1), kernels::TS_M);
    const int ct_max = std::max(1, kernels::TS_NMAX / (2 * T));
    const int groups = div_ceil(C, ct_max);
    const int vps = jac ? 16 : 32;
    const int min_splits = div_ceil(std::max(nvoxels, 1), jac ? 2048 : 4096);
    const TcTuning tuning = tuned_tc(jac ? TcKind::SpiralJacobian : TcKind::SpiralSignal, R, nvoxels, int64_t(C) * S);
    int splits = min_splits;
    if (tuning.splits > 0) {
        splits = std::max(min_splits, std::min({tuning.splits, 64, div_ceil(std::max(nvoxels, 1), vps)}));
    } else {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int64_t ctas = int64_t(R) * groups;
        if (ctas * splits < 2 * sms)
            splits = std::max(splits, int(std::min<int64_t>(div_ceil(2 * sms, int(ctas)), div_ceil(nvoxels, 8 * vps))));
    }
    // the count the launch runs: voxels per split rounded up to whole stages, every split non-empty
    const int vchunk = div_ceil(div_ceil(std::max(nvoxels, 1), splits), vps) * vps;
    return div_ceil(std::max(nvoxels, 1), vchunk);
}

namespace {

template<bool JAC>
void set_smem_attribute() {
    static std::once_flag once;
    std::call_once(once, [] {
        COMPAS_CUDA_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(kernels::tc_spiral_kernel<JAC>),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, kernels::TS_SMEM));
    });
}

bool launch_tc_spiral(const CompasContext& ctx, kernels::TsArgs a, bool jac) {
    if (!tensor_cores_available(ctx.device())) return false;
    const int T = div_ceil(std::max(a.S, 1), kernels::TS_M);
    if (2 * T > kernels::TS_NMAX) return false;  // readouts of more than 16384 samples: FP32 kernel
    DeviceGuard guard(ctx.device());
    if (int64_t(a.C) * a.R * a.S == 0) return true;
    if (a.nvoxels == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(a.out, 0, sizeof(float2) * size_t(a.C) * a.R * a.S, ctx.stream()));
        return true;
    }
    a.status = ctx.status_word();
    a.T = T;
    // coils per CTA: as many as fit 2·T·CT ≤ 256 real columns, spread evenly over the coil groups
    const int ct_max = std::max(1, kernels::TS_NMAX / (2 * T));
    const int groups = div_ceil(a.C, ct_max);
    a.CT = div_ceil(a.C, groups);
    const int vps = jac ? 16 : 32;
    int splits = tc_spiral_splits(ctx.device(), a.nvoxels, a.R, a.S, a.C, jac);
    a.vchunk = div_ceil(div_ceil(a.nvoxels, splits), vps) * vps;
    splits = div_ceil(a.nvoxels, a.vchunk);
    const int64_t n = int64_t(a.C) * a.R * a.S;
    float2* out = a.out;
    Array<cfloat, 2> partials({splits > 1 ? splits : 0, n}, ctx.device(), ctx.stream());
    if (splits > 1) a.out = reinterpret_cast<float2*>(partials.data());
    // readouts in chunks whose base table ([readouts][TERMS][T][V] complex) stays near 1 GB
    // (COMPAS_B200_SPIRAL_TABLE_BYTES overrides the budget; results do not depend on it)
    const int terms = jac ? 2 : 1;
    const int chunk = spiral_table_chunk(int64_t(terms) * T * a.nvoxels * int64_t(sizeof(float2)), a.R);
    Array<cfloat, 2> base({std::min(chunk, a.R), int64_t(terms) * T * a.nvoxels}, ctx.device(), ctx.stream());
    a.base = reinterpret_cast<const float2*>(base.data());
    if (jac) set_smem_attribute<true>();
    else set_smem_attribute<false>();
    for (int r0 = 0; r0 < a.R; r0 += chunk) {
        a.r_first = r0;
        const int rc = std::min(chunk, a.R - r0);
        const dim3 pgrid(div_ceil(a.nvoxels, 128), rc);
        const dim3 grid(rc, groups, splits);
        float2* bp = reinterpret_cast<float2*>(base.data());
        if (jac) {
            kernels::tc_spiral_base_kernel<true><<<pgrid, 128, 0, ctx.stream()>>>(a, bp);
            kernels::tc_spiral_kernel<true><<<grid, kernels::TS_THREADS, kernels::TS_SMEM, ctx.stream()>>>(a);
        } else {
            kernels::tc_spiral_base_kernel<false><<<pgrid, 128, 0, ctx.stream()>>>(a, bp);
            kernels::tc_spiral_kernel<false><<<grid, kernels::TS_THREADS, kernels::TS_SMEM, ctx.stream()>>>(a);
        }
        check_launch("tc_spiral_base_kernel / tc_spiral_kernel");
    }
    if (splits > 1) sum_partials(ctx, partials.data(), splits, n, reinterpret_cast<cfloat*>(out));
    return true;
}

kernels::TsArgs spiral_args(const float* params, int64_t pstride, int nvoxels, const cfloat* echos,
                            const cfloat* coils, int ncoils, int nreadouts, int ns, float dt, const cfloat* k_start,
                            const cfloat* delta_k, cfloat* out) {
    kernels::TsArgs a {};
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
    a.out = reinterpret_cast<float2*>(out);
    return a;
}

}  // namespace

bool launch_signal_spiral_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                             const cfloat* echos, const cfloat* coils, int ncoils, int nreadouts, int ns, float dt,
                             const cfloat* k_start, const cfloat* delta_k, cfloat* signal) {
    return launch_tc_spiral(
        ctx, spiral_args(params, pstride, nvoxels, echos, coils, ncoils, nreadouts, ns, dt, k_start, delta_k, signal),
        false);
}

bool launch_jacobian_spiral_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                               const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                               int ncoils, const cfloat* vec, int nreadouts, int ns, float dt, const cfloat* k_start,
                               const cfloat* delta_k, cfloat* Jv) {
    auto a = spiral_args(params, pstride, nvoxels, echos, coils, ncoils, nreadouts, ns, dt, k_start, delta_k, Jv);
    a.dT1 = reinterpret_cast<const float2*>(dT1);
    a.dT2 = reinterpret_cast<const float2*>(dT2);
    a.vec = reinterpret_cast<const float2*>(vec);
    return launch_tc_spiral(ctx, a, true);
}

}  // namespace compas
