// tc_hermitian.cu — compute_jacobian_hermitian (Jᴴ·v) on tcgen05 tensor cores, split-BF16.
//
// Reference math: src/jacobian/hermitian_kernels.cuh:30-92 (see hermitian.cu for the
// regrouping). For every voxel v and (readout r, coil c) pair p:
//   Y_p(v) = Σ_k u[c][r][k]·conj(E_k(v)),   Ỹ_p(v) = Σ_k (k - S/2)·u[c][r][k]·conj(E_k(v))
// is a GEMM with M = voxels, N = pairs, K = samples. A CTA owns 128 voxels (the 128 TMEM
// lanes), so the follow-up contraction over coils and readouts
//   Z_r = Σ_c conj(C_c)·Y_rc,  Z̃_r = Σ_c conj(C_c)·Ỹ_rc,
//   mHv += conj(m[r])·Z_r,  dmHv0 += conj(∂T1m[r])·Z_r,  dmHv1 += conj(∂T2m[r])·Z_r + ΔtR2²·conj(m[r])·Z̃_r
// happens inside each epilogue thread; the per-voxel results never leave registers, every echo
// element is read once for all coils, and no [R][V] temporary is written (the reference writes
// two FP32 [2][R][V] arrays per coil and re-reads the echoes per coil).
//
// Real-ified operands (re/im interleaved along K = 2S):
//   A'[v]  = (Re ē_k, Im ē_k) with ē = conj(E_k(v))     — 256 voxels (a CTA pair) × 32 samples per stage
//   B'[n]  for n = h·128 + type·32 + q, pair p = h·32 + q of the 64-pair tile:
//          type 0 (u_re, -u_im) → Y_re, 1 (u_im, u_re) → Y_im, 2 and 3 the same of (k-S/2)·u → Ỹ_re, Ỹ_im
// A does not depend on the pair tile, so a small kernel writes it once per call as the swizzled
// BF16 hi/lo shared-memory images of every (voxel tile, 32-sample stage): E_k exactly at every
// 16th sample (phase reduced modulo 2π in FP64) and the complex recurrence in between. The
// contraction then loads each stage's A with one bulk copy.
// D[128 voxels][256] accumulates in TMEM; two accumulators (512 columns) alternate between
// consecutive pair tiles so the epilogue of tile t overlaps the MMAs of tile t+1.
// Warp roles (576 threads): 0-7 epilogue (warps w and w+4 share TMEM lanes 32(w%4).. = voxels
// and split each tile's pairs), 8-15 convert u (B), 16 allocates TMEM and issues the MMAs,
// 17 loads A. All waits are bounded.
#include <cuda_bf16.h>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {

void sum_partials(const CompasContext& ctx, const cfloat* partials, int nsplit, int64_t n, cfloat* out);

namespace kernels {

constexpr int TH_M = 128, TH_N = 256, TH_K = 64, TH_PAIRS = 64;
constexpr int TH_THREADS = 576;  // 8 epilogue + 8 B warps + MMA warp + copy warp
constexpr int TH_MMA_WARP = 16, TH_COPY_WARP = 17;
constexpr int TH_B_THREADS = 256;
constexpr int TH_STAGES = 3;
constexpr int TH_A_BYTES = TH_M * TH_K * 2;           // 16 KB per plane: this CTA's 128 voxels
constexpr int TH_BH_BYTES = (TH_N / 2) * TH_K * 2;    // 16 KB per plane: this CTA's 128 of the 256 B rows
constexpr int TH_STAGE_BYTES = 2 * TH_A_BYTES + 2 * TH_BH_BYTES;
constexpr int TH_SMEM = TH_STAGES * TH_STAGE_BYTES + 1024 + 256;
constexpr int TH_APACK_BLOCK = 2 * TH_A_BYTES;  // hi + lo image of one (voxel tile, stage)

struct ThArgs {
    const float* params;
    int64_t pstride;
    int nvoxels;
    const float2* echo;
    const float2* dT1;
    const float2* dT2;
    const float2* coils;  // [C][V]
    const float2* u;      // [C][R][S]
    int R, S, C;
    float dt, dk_re, dk_im;
    int tiles_per_split;  // pair tiles handled by one CTA
    const unsigned char* apack;  // [voxel tiles][stages] A images
    float2* out;          // [splits][4][V]
    unsigned int* status;
};

// A images: thread = (voxel row t of tile blockIdx.x, 16-sample segment blockIdx.y) writes
// conj(E_k(v)) for k = 16·seg .. 16·seg + 15 (zero past S or past the last voxel)
__global__ void __launch_bounds__(128) tc_hermitian_pack_kernel(ThArgs a) {
    const int t = threadIdx.x;
    const int v = blockIdx.x * TH_M + t;
    const int seg = blockIdx.y;
    const int kstages = (a.S + 31) / 32;
    const double twopi = 6.283185307179586476925;
    float2 e = make_float2(0.f, 0.f), step = e;
    const bool vok = v < a.nvoxels;
    if (vok) {
        const float T2 = a.params[a.pstride + v], B0 = a.params[3 * a.pstride + v];
        const float x = a.params[6 * a.pstride + v], y = a.params[7 * a.pstride + v];
        const double theta = double(a.dk_re) * x + double(a.dk_im) * y + double(a.dt) * twopi * B0;
        const float decay = -a.dt / T2;
        const float2 st = cis_rad(theta);
        const float sm = __expf(decay);
        step = make_float2(sm * st.x, sm * st.y);
        const int kb = seg * 16;
        const float s0 = float(kb) - 0.5f * float(a.S);
        const float2 ph = cis_rad(double(s0) * theta);
        const float mg = __expf(s0 * decay);
        e = make_float2(mg * ph.x, mg * ph.y);
    }
    unsigned char* blk = const_cast<unsigned char*>(a.apack) + (int64_t(blockIdx.x) * kstages + seg / 2) * TH_APACK_BLOCK;
#pragma unroll
    for (int cq = 0; cq < 4; cq++) {  // 4 chunks of 4 samples
        uint32_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const bool kok = vok && (seg * 16 + 4 * cq + i) < a.S;
            tc::split2(kok ? e.x : 0.0f, kok ? -e.y : 0.0f, h[i], l[i]);
            e = cmul(e, step);
        }
        const uint32_t off = tc::sw128_offset(t, (seg & 1) * 4 + cq);
        *reinterpret_cast<uint4*>(blk + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(blk + TH_A_BYTES + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

// One CTA pair (cluster of 2) per pair of voxel tiles and pair-tile range: each CTA loads its own
// voxel tile's A and converts half of B — the four rows of 32 of the tile's 64 pairs, so it reads
// only those pairs' u — and the leader issues M = 256 MMAs over both. Producers of both CTAs
// arrive on the leader's barriers; the leader's commits arrive on both CTAs' barriers.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TH_THREADS, 1) tc_hermitian_kernel(ThArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TH_STAGES * TH_STAGE_BYTES);
    uint64_t* empty = full + TH_STAGES;
    uint64_t* afull = empty + TH_STAGES;
    uint64_t* acc_full = afull + TH_STAGES;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = tc::cluster_ctarank();
    const int vt = blockIdx.x;  // this CTA's voxel tile
    const int v0 = vt * TH_M;
    const int split = blockIdx.y;
    const int npairs = a.R * a.C;
    const int ntiles_total = (npairs + TH_PAIRS - 1) / TH_PAIRS;
    const int tile_begin = split * a.tiles_per_split;
    const int tile_end = min(ntiles_total, tile_begin + a.tiles_per_split);
    const int ntiles = max(0, tile_end - tile_begin);
    const int kstages = (a.S + 31) / 32;  // 32 samples (64 K) per stage
    const int nstages = ntiles * kstages;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TH_STAGES; s++) {
            tc::mbar_init(&full[s], 2 * TH_B_THREADS + 1);  // B of both CTAs + the peer's A landed
            tc::mbar_init(&empty[s], 1);
            tc::mbar_init(&afull[s], 1);
        }
        for (int s = 0; s < 2; s++) {
            tc::mbar_init(&acc_full[s], 1);
            tc::mbar_init(&acc_empty[s], 2 * 256);  // epilogue threads of both CTAs
        }
        tc::mbar_init(done, 1);
        *abort_flag = 0;
        tc::fence_mbarrier_init();
    }
    if (warp == TH_MMA_WARP) tc::tmem_alloc_pair(tmem_slot, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::cluster_sync();  // both CTAs' barriers exist before either arrives on the other's
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < 8) {
        // ---------------- epilogue: thread = voxel = TMEM lane 32·(warp%4) + lane; warps w and
        // w+4 take alternate 8-pair chunks of every tile
        const int t = threadIdx.x & 127;
        const int v = v0 + t;
        const bool vok = v < a.nvoxels;
        const int vc = vok ? v : (a.nvoxels - 1);
        const float T1 = a.params[vc], T2 = a.params[a.pstride + vc];
        const float2 rho = make_float2(a.params[4 * a.pstride + vc], a.params[5 * a.pstride + vc]);
        const float R2 = 1.0f / T2;
        const float dscale = a.dt * R2 * R2;
        const int quarter = warp & 3, parity = warp >> 2;
        // Σ_r over conj(∂T1m)·Z, conj(∂T2m)·Z + ΔtR2²·conj(m)·Z̃, conj(m)·Z
        float2 acc[3];
#pragma unroll
        for (int f = 0; f < 3; f++) acc[f] = make_float2(0.f, 0.f);
        // echoes of readout r: those of a chunk's first readout are requested one chunk ahead,
        // the second readout's (4-7 coils) at the start of the chunk, further ones (fewer than 4
        // coils) when needed
        auto load_echo = [&](int r, float2& e0, float2& e1, float2& e2) {
            e0 = e1 = e2 = make_float2(0.f, 0.f);
            if (vok && r < a.R) {
                const int64_t idx = int64_t(r) * a.nvoxels + v;
                e0 = __ldg(a.echo + idx);
                e1 = __ldg(a.dT1 + idx);
                e2 = __ldg(a.dT2 + idx);
            }
        };
        float2 m[2], m1[2], m2[2], mn, m1n, m2n;
        if (ntiles > 0) load_echo((tile_begin * TH_PAIRS + parity * 8) / a.C, m[0], m1[0], m2[0]);
        bool ok = true;
        for (int tl = 0; tl < ntiles; tl++) {
            const int abuf = tl & 1;
            const bool waited = tc::mbar_wait(&acc_full[abuf], (tl >> 1) & 1, a.status);
            tc::tc_fence_after();
            if (!__all_sync(0xffffffffu, waited && !*(volatile int*)abort_flag)) {
                *abort_flag = 1;
                ok = false;
                break;
            }
            const uint32_t tbase = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(abuf * 256);
            const int p0 = (tile_begin + tl) * TH_PAIRS;
#pragma unroll 1
            for (int ch = parity; ch < TH_PAIRS / 8; ch += 2) {  // 8 pairs at a time
                const int pb = p0 + ch * 8;
                const int rb = pb / a.C;
                if ((pb + 7) / a.C > rb) load_echo(rb + 1, m[1], m1[1], m2[1]);
                {
                    const bool more = ch + 2 < TH_PAIRS / 8;
                    const int tln = more ? tl : tl + 1, chn = more ? ch + 2 : parity;
                    if (tln < ntiles) load_echo(((tile_begin + tln) * TH_PAIRS + chn * 8) / a.C, mn, m1n, m2n);
                }
                // coil factor of each pair (a small table that stays in L1)
                float2 cc[8];
                {
                    int c = pb - rb * a.C;
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        cc[i] = (vok && pb + i < npairs) ? __ldg(a.coils + int64_t(c) * a.nvoxels + v)
                                                         : make_float2(0.f, 0.f);
                        if (++c == a.C) c = 0;
                    }
                }
                float yr[8], yi[8], tr[8], ti[8];
                // columns: [pair half][Y_re, Y_im, Ỹ_re, Ỹ_im][32 pairs]
                const uint32_t cb = tbase + uint32_t((ch >> 2) * 128 + (ch & 3) * 8);
                tc::tmem_load8x4(cb, cb + 32, cb + 64, cb + 96, yr, yi, tr, ti);
                int r = rb, c = pb - rb * a.C;
                float2 Z = make_float2(0.f, 0.f), Zt = Z;
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    Z = cadd(Z, cmulc(make_float2(yr[i], yi[i]), cc[i]));
                    Zt = cadd(Zt, cmulc(make_float2(tr[i], ti[i]), cc[i]));
                    const bool next_r = ++c == a.C;
                    if (next_r || i == 7) {
                        // fold readout r's coil sum into the voxel's results
                        float2 me, d1, d2;
                        if (r == rb) {
                            me = m[0], d1 = m1[0], d2 = m2[0];
                        } else if (r == rb + 1) {
                            me = m[1], d1 = m1[1], d2 = m2[1];
                        } else {
                            load_echo(r, me, d1, d2);
                        }
                        acc[0] = cadd(acc[0], cmulc(Z, d1));
                        acc[1] = cadd(acc[1], cadd(cmulc(Z, d2), cscale(dscale, cmulc(Zt, me))));
                        acc[2] = cadd(acc[2], cmulc(Z, me));
                        Z = Zt = make_float2(0.f, 0.f);
                    }
                    if (next_r) {
                        c = 0;
                        ++r;
                    }
                }
                m[0] = mn;
                m1[0] = m1n;
                m2[0] = m2n;
            }
            tc::tc_fence_before();
            tc::mbar_arrive_cluster(&acc_empty[abuf], 0);
        }
        // combine the two warps of each lane quarter through shared memory (stage buffer 0,
        // free once every tile has been consumed) and write the four results
        float2* red = reinterpret_cast<float2*>(smem);
        tc::bar_sync(2, 256);  // epilogue warps only: all MMAs consumed
        if (parity == 1) {
#pragma unroll
            for (int f = 0; f < 3; f++) red[f * 128 + t] = acc[f];
        }
        tc::bar_sync(2, 256);
        if (parity == 0 && ok && vok && !*(volatile int*)abort_flag) {
#pragma unroll
            for (int f = 0; f < 3; f++) acc[f] = cadd(acc[f], red[f * 128 + t]);
            // conj(T1ρ·C)·… : the ρ factors of the T1 / T2 blocks, taken out of the coil sums
            const float2 r1 = cscale(T1, rho), r2 = cscale(T2, rho);
            float2* o = a.out + int64_t(split) * 4 * a.nvoxels;
            o[v] = cmulc(acc[0], r1);
            o[a.nvoxels + v] = cmulc(acc[1], r2);
            o[2 * int64_t(a.nvoxels) + v] = acc[2];
            o[3 * int64_t(a.nvoxels) + v] = make_float2(acc[2].y, -acc[2].x);  // -i·mHv
        }
    } else if (warp < 16) {
        // ---------------- B producer: the CTA's 32 pairs of the tile (rank·32 ..), all four rows
        // each: (u_re,-u_im) → Y_re, (u_im,u_re) → Y_im and the same of (k-S/2)·u → Ỹ_re, Ỹ_im.
        // thread = (pair q, 4-sample quad sq): 8 lanes cover one pair's 32 samples, so each load
        // instruction reads 4 contiguous 128-byte pieces of u
        const int t = threadIdx.x - 256;
        const int sq = t & 7, q = t >> 3;
        const int pl = int(rank) * 32 + q;  // pair within the tile
        // u is loaded two stages ahead: stage g + 2 is requested once stage g is converted
        const bool vec16 = (a.S & 1) == 0 && (reinterpret_cast<uintptr_t>(a.u) & 15) == 0;  // 16-byte aligned rows
        float2 uv[4], uv1[4];
        auto load_u = [&](int g, float2 (&dst)[4]) {
            const int tl = g / kstages, ks = g - tl * kstages;
            const int p = (tile_begin + tl) * TH_PAIRS + pl;
            const bool pok = p < npairs;
            const int r = pok ? p / a.C : 0, c = pok ? p - r * a.C : 0;
            const float2* urow = a.u + (int64_t(c) * a.R + r) * a.S;
            const int kb = ks * 32 + sq * 4;
            if (pok && vec16 && kb + 4 <= a.S) {
                const float4 x0 = __ldg(reinterpret_cast<const float4*>(urow + kb));
                const float4 x1 = __ldg(reinterpret_cast<const float4*>(urow + kb + 2));
                dst[0] = make_float2(x0.x, x0.y);
                dst[1] = make_float2(x0.z, x0.w);
                dst[2] = make_float2(x1.x, x1.y);
                dst[3] = make_float2(x1.z, x1.w);
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++) dst[i] = (pok && kb + i < a.S) ? __ldg(urow + kb + i) : make_float2(0.f, 0.f);
            }
        };
        if (nstages > 0) load_u(0, uv);
        if (nstages > 1) load_u(1, uv1);
        for (int g = 0; g < nstages; g++) {
            const int buf = g % TH_STAGES;
            const int ks = g % kstages;
            if (!tc::mbar_wait(&empty[buf], ((g / TH_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
            if (*(volatile int*)abort_flag) break;
            unsigned char* Bh = smem + buf * TH_STAGE_BYTES + 2 * TH_A_BYTES;
            unsigned char* Bl = Bh + TH_BH_BYTES;
            const int kb = ks * 32 + sq * 4;
            // one hi/lo split per value: the split of (x, -y) is the split of (x, y) with the upper
            // sign bit flipped, the split of (y, x) the same pair with halves swapped
            uint32_t h0[4], l0[4], h1[4], l1[4], h2[4], l2[4], h3[4], l3[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float2 w = uv[i];
                const float ksf = float(kb + i) - 0.5f * float(a.S);
                uint32_t h, l, hs, ls;
                tc::split2(w.x, w.y, h, l);
                tc::split2(ksf * w.x, ksf * w.y, hs, ls);
                h0[i] = h ^ 0x80000000u;
                l0[i] = l ^ 0x80000000u;
                h1[i] = __byte_perm(h, 0, 0x1032);
                l1[i] = __byte_perm(l, 0, 0x1032);
                h2[i] = hs ^ 0x80000000u;
                l2[i] = ls ^ 0x80000000u;
                h3[i] = __byte_perm(hs, 0, 0x1032);
                l3[i] = __byte_perm(ls, 0, 0x1032);
            }
            // local row = type·32 + q (global B row rank·128 + type·32 + q), 16-byte chunk sq
            const uint32_t o0 = tc::sw128_offset(0 * 32 + q, sq), o1 = tc::sw128_offset(1 * 32 + q, sq);
            const uint32_t o2 = tc::sw128_offset(2 * 32 + q, sq), o3 = tc::sw128_offset(3 * 32 + q, sq);
            *reinterpret_cast<uint4*>(Bh + o0) = make_uint4(h0[0], h0[1], h0[2], h0[3]);
            *reinterpret_cast<uint4*>(Bl + o0) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
            *reinterpret_cast<uint4*>(Bh + o1) = make_uint4(h1[0], h1[1], h1[2], h1[3]);
            *reinterpret_cast<uint4*>(Bl + o1) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
            *reinterpret_cast<uint4*>(Bh + o2) = make_uint4(h2[0], h2[1], h2[2], h2[3]);
            *reinterpret_cast<uint4*>(Bl + o2) = make_uint4(l2[0], l2[1], l2[2], l2[3]);
            *reinterpret_cast<uint4*>(Bh + o3) = make_uint4(h3[0], h3[1], h3[2], h3[3]);
            *reinterpret_cast<uint4*>(Bl + o3) = make_uint4(l3[0], l3[1], l3[2], l3[3]);
            tc::fence_async_shared();
            tc::mbar_arrive_cluster(&full[buf], 0);
#pragma unroll
            for (int i = 0; i < 4; i++) uv[i] = uv1[i];
            if (g + 2 < nstages) load_u(g + 2, uv1);
        }
    } else if (warp == TH_COPY_WARP) {
        // ---------------- A: one bulk copy (hi + lo, 32 KB) per stage into this CTA's buffer
        if (lane == 0) {
            const unsigned char* src = a.apack + int64_t(vt) * kstages * TH_APACK_BLOCK;
            int issued[TH_STAGES];
            for (int s = 0; s < TH_STAGES; s++) issued[s] = -1;
            for (int g = 0; g < nstages; g++) {
                const int buf = g % TH_STAGES;
                if (!tc::mbar_wait(&empty[buf], ((g / TH_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::mbar_arrive_expect_tx(&afull[buf], TH_APACK_BLOCK);
                tc::bulk_copy_g2s(smem + buf * TH_STAGE_BYTES, src + int64_t(g % kstages) * TH_APACK_BLOCK,
                                  TH_APACK_BLOCK, &afull[buf]);
                issued[buf] = g;
            }
            // copies still in flight land before the CTA can finish (bounded)
            for (int s = 0; s < TH_STAGES; s++)
                if (issued[s] >= 0) tc::mbar_wait(&afull[s], (issued[s] / TH_STAGES) & 1, a.status);
        }
    } else if (rank == 0) {
        // ---------------- MMA issuer (leader, warp 16, one lane): M = 256 over both CTAs
        if (lane == 0) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(2 * TH_M, TH_N);
            int g = 0;
            for (int tl = 0; tl < ntiles && !*(volatile int*)abort_flag; tl++) {
                const int abuf = tl & 1;
                if (tl >= 2 && !tc::mbar_wait(&acc_empty[abuf], ((tl >> 1) - 1) & 1, a.status)) {
                    *abort_flag = 1;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t d = tmem + uint32_t(abuf * 256);
                for (int ks = 0; ks < kstages; ks++, g++) {
                    const int buf = g % TH_STAGES;
                    if (!tc::mbar_wait(&full[buf], (g / TH_STAGES) & 1, a.status)) *abort_flag = 1;
                    if (!tc::mbar_wait(&afull[buf], (g / TH_STAGES) & 1, a.status)) *abort_flag = 1;
                    if (*(volatile int*)abort_flag) break;
                    tc::tc_fence_after();
                    const uint32_t base = tc::smem_u32(smem + buf * TH_STAGE_BYTES);
                    const uint32_t ah = base, al = base + TH_A_BYTES;
                    const uint32_t bh = base + 2 * TH_A_BYTES, bl = bh + TH_BH_BYTES;
#pragma unroll
                    for (int k16 = 0; k16 < TH_K / 16; k16++) {
                        const uint32_t koff = k16 * 32;
                        const uint64_t dah = tc::sw128_kmajor_desc(ah + koff), dal = tc::sw128_kmajor_desc(al + koff);
                        const uint64_t dbh = tc::sw128_kmajor_desc(bh + koff), dbl = tc::sw128_kmajor_desc(bl + koff);
                        tc::mma_bf16_pair(d, dah, dbh, idesc, (ks > 0 || k16 > 0) ? 1u : 0u);
                        tc::mma_bf16_pair(d, dah, dbl, idesc, 1u);
                        tc::mma_bf16_pair(d, dal, dbh, idesc, 1u);
                    }
                    tc::mma_commit_pair(&empty[buf]);
                }
                tc::mma_commit_pair(&acc_full[abuf]);
            }
            tc::mma_commit_pair(done);
            tc::mbar_wait(done, 0, a.status);  // all MMAs complete before TMEM is released
        }
        __syncwarp();
    } else {
        // ---------------- peer, warp 16: tell the leader when each stage's A has landed here
        if (lane == 0) {
            for (int g = 0; g < nstages; g++) {
                const int buf = g % TH_STAGES;
                if (!tc::mbar_wait(&afull[buf], (g / TH_STAGES) & 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::mbar_arrive_cluster(&full[buf], 0);
            }
            tc::mbar_wait(done, 0, a.status);
        }
        __syncwarp();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::cluster_sync();  // neither CTA leaves while the other may still signal it or read TMEM
    if (warp == TH_MMA_WARP) {
        tc::tc_fence_after();
        tc::tmem_dealloc_pair(tmem, 512);
    }
}

}  // namespace kernels

// pair-tile splits of the Cartesian Jᴴ·v contraction: the tuned count (at most one split per pair
// tile), else the count (≥ 4 tiles per split, ≤ 16 splits) that leaves the least idle part of the
// last wave of one CTA per SM. Each pair tile's accumulation is drained separately, so the count
// changes only the partial sums.
int tc_hermitian_splits(int device, int nvoxels, int R, int S, int C) {
    const int vtiles = 2 * div_ceil(nvoxels, 2 * kernels::TH_M);
    const int ptiles = div_ceil(C * R, kernels::TH_PAIRS);
    const TcTuning tuning = tuned_tc(TcKind::CartesianHermitian, R, nvoxels, int64_t(C) * S);
    int splits = 1;
    if (tuning.splits > 0) {
        splits = std::max(1, std::min(tuning.splits, ptiles));
    } else {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        double best = -1.0;
        for (int sp = 1; sp <= std::max(1, std::min(16, ptiles / 4)); sp++) {
            const int64_t ctas = int64_t(vtiles) * sp;
            const int64_t waves = (ctas + sms - 1) / sms;
            const double eff = double(ctas) / double(waves * sms) - 0.002 * sp;
            if (eff > best + 1e-9) {
                best = eff;
                splits = sp;
            }
        }
    }
    return div_ceil(ptiles, div_ceil(ptiles, splits));  // the count the launch runs (none empty)
}

bool launch_jacobian_hermitian_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                  const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                                  int ncoils, const cfloat* vec, const CartesianGeom& g, cfloat* JHv) {
    if (!tensor_cores_available(ctx.device())) return false;
    if (nvoxels == 0) return true;
    DeviceGuard guard(ctx.device());
    if (int64_t(ncoils) * g.nreadouts * g.ns == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(JHv, 0, sizeof(cfloat) * 4 * size_t(nvoxels), ctx.stream()));
        return true;
    }
    kernels::ThArgs a {};
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
    a.status = ctx.status_word();
    const int vtiles = 2 * div_ceil(nvoxels, 2 * kernels::TH_M);  // whole CTA pairs
    const int ptiles = div_ceil(ncoils * g.nreadouts, kernels::TH_PAIRS);
    const int kstages = div_ceil(g.ns, 32);
    int splits = tc_hermitian_splits(ctx.device(), nvoxels, g.nreadouts, g.ns, ncoils);
    a.tiles_per_split = div_ceil(ptiles, splits);
    splits = div_ceil(ptiles, a.tiles_per_split);
    const int64_t n = 4 * int64_t(nvoxels);
    Array<cfloat, 2> partials({splits > 1 ? splits : 0, n}, ctx.device(), ctx.stream());
    Array<unsigned char> apack({int64_t(vtiles) * kstages * kernels::TH_APACK_BLOCK}, ctx.device(), ctx.stream());
    a.apack = apack.data();
    a.out = reinterpret_cast<float2*>(splits > 1 ? partials.data() : JHv);
    static bool attr_set = false;
    if (!attr_set) {
        COMPAS_CUDA_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(kernels::tc_hermitian_kernel),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, kernels::TH_SMEM));
        attr_set = true;
    }
    kernels::tc_hermitian_pack_kernel<<<dim3(vtiles, 2 * kstages), kernels::TH_M, 0, ctx.stream()>>>(a);
    check_launch("tc_hermitian_pack_kernel");
    dim3 grid(vtiles, splits);
    kernels::tc_hermitian_kernel<<<grid, kernels::TH_THREADS, kernels::TH_SMEM, ctx.stream()>>>(a);
    check_launch("tc_hermitian_kernel");
    if (splits > 1) sum_partials(ctx, partials.data(), splits, n, JHv);
    return true;
}

}  // namespace compas
