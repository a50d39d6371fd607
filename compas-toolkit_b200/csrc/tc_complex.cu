// tc_complex.cu — split-BF16 tcgen05 tensor-core kernels for the Cartesian signal and J·v.
//
// Both operations are voxel contractions of a streamed operand A with a generated operand B
// (see signal.cu for the algebra, reference src/trajectories/signal_kernels.cuh:137-167 and
// src/jacobian/product_kernels.cuh:7-67):
//   signal: out[c][r][k] = Σ_v echo[r][v] · F_{c,k}(v),        F = coil·ρ·E_k·e^{i(S/2)Δk_im y}
//   J·v:    out[c][r][k] = Σ_v P[r][v]·F_{c,k}(v) + Q'[r][v]·(k-S/2)·F_{c,k}(v),  F = coil·E_k
// The complex contraction is real-ified by interleaving re/im along K: the streamed row
// (A_re, A_im) per complex term, the generated rows (F_re, -F_im) and (F_im, F_re) per output pair
// j = (c, k), so one real GEMM D[2j + re/im][readout] yields the complex tile.
//
// Precision: every operand x is split as x = hi + lo (two BF16s, |x - hi - lo| ≤ 2⁻¹⁸|x|) and the
// product is accumulated in FP32 TMEM as hi·hi + hi·lo + lo·hi (three tcgen05.mma per K step);
// the dropped lo·lo term is ≤ 2⁻¹⁶ relative, giving ~1e-5 relative L2 against FP64.
//
// Per call, small kernels first write per-voxel tables (the E_k step, E_k itself at every
// TC_PPG-th sample with the phase reduced in FP64, coil·w, the J·v coefficients) and pack the
// streamed operand once as the split, swizzled shared-memory images the contraction consumes.
// The contraction runs on CTA pairs (cluster of 2, tcgen05 cta_group::2): one MMA spans both SMs'
// tensor cores with M = 256 generated rows (128 (coil, sample) pairs × re/im; each CTA generates
// its 128) and N = nr readouts (each CTA holds nr/2; nr, a multiple of 16 up to 256, gives the fewest
// readout tiles and then the least padding, e.g. 224 for 1120 readouts).
// CTA organisation (576 threads, 1 CTA/SM, 192 KB shared memory in 3 stages of 64 KB):
//   warps 0-15  generate this CTA's 128 rows (64 pairs × 64 K per stage): thread = (2 voxels,
//               group of TC_PPG pairs); a group starts from the exact E_k table value × coil·w and
//               steps along k with the complex recurrence. Afterwards they drain the TMEM
//               accumulator through shared memory into coalesced rows of the output;
//   warp 16     allocates 512 TMEM columns (both CTAs); in the leader one lane issues the 12 MMAs
//               per stage, in the peer one lane tells the leader when its streamed half has landed;
//   warp 17     one lane loads each stage's half readout tile (hi and lo planes) by bulk copies.
// Stages hand over through mbarriers (full, in the leader: producers of both CTAs → MMA; afull:
// copy landed; empty, in both: tcgen05.commit multicast → producers and copy). Every 512 K16 steps
// (128 stages) the producers fold the TMEM accumulator into an FP32 running sum held in the other
// half of the CTA's 512 TMEM columns, which bounds the tensor core's accumulation error for any
// voxel count. The voxel range is split over CTA pairs (split-K) only to fill the GPU; partial
// tiles are summed in a fixed order. Every wait is bounded.
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "compas/compas.h"
#include "job_args.cuh"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {

void sum_partials(const CompasContext& ctx, const cfloat* partials, int nsplit, int64_t n, cfloat* out);

namespace kernels {

constexpr int TC_M = 128, TC_N = 256, TC_K = 64;  // real-ified tile of one CTA (M = 256 per CTA pair)
constexpr int TC_PAIRS = TC_N / 2;                 // complex (c, k) pairs per tile
constexpr int TC_PPG = 2;                          // consecutive pairs per producer thread
constexpr int TC_B_THREADS = 512;                  // 16 producer warps: 16 voxel halves × 32 groups
constexpr int TC_MMA_WARP = 16, TC_COPY_WARP = 17;
constexpr int TC_THREADS = 576;
constexpr int TC_STAGES = 3;
constexpr int TC_A_BYTES = TC_M * TC_K * 2;         // 16 KB slot per hi/lo plane: this CTA's ≤ 128 readouts
constexpr int TC_BH_BYTES = (TC_N / 2) * TC_K * 2;  // 16 KB per hi/lo plane: this CTA's 128 generated rows
constexpr int TC_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TC_BH_BYTES;
constexpr int TC_SMEM = TC_STAGES * TC_STAGE_BYTES + 1024 /*align*/ + 128 /*barriers*/;
// TMEM of a CTA: the MMA accumulator (columns 0 .. nr-1) and the running FP32 sum of the finished
// accumulation chunks (columns TC_SUM_COL ..); a chunk is TC_CHUNK_STAGES stages = 512 K16 steps
constexpr int TC_TMEM_COLS = 512, TC_SUM_COL = 256;
constexpr int TC_CHUNK_STAGES = 128;
static_assert(TC_PAIRS / 2 == (TC_B_THREADS / 16) * TC_PPG, "a CTA's producer groups cover half the pair tile");
static_assert((TC_PAIRS / 2) * (2 * 256 + 2) * 4 <= TC_STAGES * TC_STAGE_BYTES, "output tile fits the stage buffers");

// one thread per voxel: the E_k step, E_k at the restart points, coil·w for every coil and
// (J·v) the four complex coefficients of P and Q' — once per call instead of per CTA and stage
template<bool JAC>
__device__ __forceinline__ void tc_prep_voxel(const TcArgs& a, const int v) {
    if (v >= a.nvoxels) return;
    const double twopi = 6.283185307179586476925;
    const float T1 = a.params[v], T2 = a.params[a.pstride + v], B0 = a.params[3 * a.pstride + v];
    const float x = a.params[6 * a.pstride + v], y = a.params[7 * a.pstride + v];
    const float2 rho = make_float2(a.params[4 * a.pstride + v], a.params[5 * a.pstride + v]);
    // Θ_v = Δk_re·x + Δk_im·y + 2πΔt·B0 (rad per sample), decay -Δt/T2 per sample
    const double theta = double(a.dk_re) * x + double(a.dk_im) * y + double(a.dt) * twopi * B0;
    const float decay = -a.dt / T2;
    const float2 st = cis_rad(theta);
    const float sm = __expf(decay);
    const_cast<float2*>(a.vstep)[v] = make_float2(sm * st.x, sm * st.y);
    // E_k = e^{(k - S/2)(decay + iΘ)} at k = q·egk, the phase argument reduced modulo 2π in FP64
    float2* estart = const_cast<float2*>(a.estart);
    const int nq = a.S / a.egk;
    for (int q = 0; q < nq; q++) {
        const float ks = float(q * a.egk) - 0.5f * float(a.S);
        const float2 ph = cis_rad(double(ks) * theta);
        const float mg = __expf(ks * decay);
        estart[int64_t(q) * a.nvoxels + v] = make_float2(mg * ph.x, mg * ph.y);
    }
    float2 w = make_float2(1.f, 0.f);
    if constexpr (!JAC) {
        w = rho;
        if (a.dk_im != 0.0f) w = cmul(w, cis_rad(0.5 * double(a.S) * double(a.dk_im) * y));
    }
    float2* coilw = const_cast<float2*>(a.coilw);
    for (int c = 0; c < a.C; c++) coilw[int64_t(c) * a.nvoxels + v] = cmul(a.coils[int64_t(c) * a.nvoxels + v], w);
    if constexpr (JAC) {
        // P = c1·∂T1m + c2·∂T2m + cm·m,  Q' = cq·m   (product_kernels.cuh:56-60, dE/dT2 folded)
        const float2 w0 = a.vec[v], w1 = a.vec[a.nvoxels + v];
        const float2 w2 = a.vec[2 * int64_t(a.nvoxels) + v], w3 = a.vec[3 * int64_t(a.nvoxels) + v];
        const float2 c1 = cmul(w0, cscale(T1, rho)), c2 = cmul(w1, cscale(T2, rho));
        const float2 cm = make_float2(w2.x - w3.y, w2.y + w3.x);
        const float R2 = 1.0f / T2;
        const float2 cq = cscale(a.dt * R2 * R2, c2);
        float4* jcoef = const_cast<float4*>(a.jcoef);
        jcoef[2 * int64_t(v)] = make_float4(c1.x, c1.y, c2.x, c2.y);
        jcoef[2 * int64_t(v) + 1] = make_float4(cm.x, cm.y, cq.x, cq.y);
    }
}

template<bool JAC>
__global__ void tc_prep_kernel(TcArgs a) {
    tc_prep_voxel<JAC>(a, blockIdx.x * blockDim.x + threadIdx.x);
}

// Pack the streamed operand (echoes, or the J·v sources) once per call as the shared-memory images
// the contraction consumes: element (readout r, column g) with g = 32·stage + j (signal: voxel g;
// J·v: voxel g/2, term g%2 = P or Q') is split into hi/lo BF16 and stored at the swizzled position
// of row r % (nr/2), column j in block (readout tile r / nr, half (r % nr) / (nr/2), stage). Rows
// past R and columns past V are zero. Each CTA of a pair then loads its half of a stage with two
// bulk copies (hi, lo).
// Thread = one 16-byte chunk (4 columns) of one row: 4 voxels (signal) or 2 voxels × 2 terms
// (J·v); a warp reads contiguous echo rows and writes whole 128-byte rows of 4 blocks.
template<bool JAC>
__device__ __forceinline__ void tc_pack_a(const TcArgs& a, const int cg, const int rp) {
    if (cg >= a.apack_stages * 8) return;
    const int stage = cg >> 3, chunk = cg & 7;
    float2 e[4];
#pragma unroll
    for (int i = 0; i < 4; i++) e[i] = make_float2(0.f, 0.f);
    if (rp < a.R) {
        const int64_t row = int64_t(rp) * a.nvoxels;
        if constexpr (!JAC) {
            const int v0 = stage * 32 + chunk * 4;
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (v0 + i < a.nvoxels) e[i] = __ldg(a.echo + row + v0 + i);
        } else {
            const int v0 = stage * 16 + chunk * 2;
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int v = v0 + i;
                if (v < a.nvoxels) {
                    // P = c1·∂T1m + c2·∂T2m + cm·m,  Q' = cq·m
                    const float4 k0 = __ldg(a.jcoef + 2 * int64_t(v)), k1 = __ldg(a.jcoef + 2 * int64_t(v) + 1);
                    const float2 me = __ldg(a.echo + row + v), d1 = __ldg(a.dT1 + row + v), d2 = __ldg(a.dT2 + row + v);
                    e[2 * i] = cadd(cadd(cmul(make_float2(k0.x, k0.y), d1), cmul(make_float2(k0.z, k0.w), d2)),
                                    cmul(make_float2(k1.x, k1.y), me));
                    e[2 * i + 1] = cmul(make_float2(k1.z, k1.w), me);
                }
            }
        }
    }
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; i++) tc::split2(e[i].x, e[i].y, h[i], l[i]);
    // block (readout tile, half for CTA rank, stage): hi plane of nr/2 rows, then the lo plane
    const int half_rows = a.nr / 2;
    const int tile = rp / a.nr, within = rp - tile * a.nr;
    const int half = within / half_rows, hrow = within - half * half_rows;
    unsigned char* blk = const_cast<unsigned char*>(a.apack) +
                         ((int64_t(tile) * 2 + half) * a.apack_stages + stage) * int64_t(half_rows) * 256;
    const uint32_t off = tc::sw128_offset(hrow, chunk);
    *reinterpret_cast<uint4*>(blk + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(blk + half_rows * 128 + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// grid (chunks / 256, padded readout rows)
template<bool JAC>
__global__ void __launch_bounds__(256) tc_pack_a_kernel(TcArgs a) {
    tc_pack_a<JAC>(a, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y);
}

// One output tile (pair tile bx, readout tile by, voxel split bz) of one contraction, computed by
// a CTA pair (cluster of 2, rank 0 / 1): each CTA generates the rows of half the tile's 128 pairs
// (rank·64 .., the MMA's A: M = 256 over the pair) and loads half of the readout tile's streamed
// operand (the MMA's B: N = nr readouts over the pair, any multiple of 16 up to 256, so R needs
// little padding); the leader issues the MMAs, producers of both CTAs arrive on the leader's
// barriers and the leader's commits arrive on both. D per CTA: 128 rows (64 pairs × re/im) × nr
// readout columns. Shared by the one-operation kernel and the batched kernel, so both give
// bit-identical results.
template<bool JAC>
__device__ __forceinline__ void tc_tile(const TcArgs& a, const int bx, const int by, const int bz,
                                        unsigned char* smem_raw) {
    constexpr int TERMS = JAC ? 2 : 1;            // complex terms per voxel along K
    constexpr int VPS = TC_K / (2 * TERMS);       // voxels per stage (32 or 16)
    constexpr int VPH = 2 / TERMS;                // voxels per 8-byte half chunk (2 or 1)
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TC_STAGES * TC_STAGE_BYTES);
    uint64_t* empty = full + TC_STAGES;
    uint64_t* afull = empty + TC_STAGES;  // the stage's A bulk copy has landed
    uint64_t* done = afull + TC_STAGES;
    uint64_t* cdone = done + 1;    // an accumulation chunk's MMAs have completed (both CTAs)
    uint64_t* drained = cdone + 1;  // (leader) both CTAs folded the accumulator into the running sum
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = tc::cluster_ctarank();
    const int n_pair0 = bx * TC_PAIRS;  // first (c,k) pair of this tile
    const int r0 = by * a.nr;
    const int v_begin = bz * a.vchunk;
    const int v_end = min(a.nvoxels, v_begin + a.vchunk);
    const int nstages = max(1, (v_end - v_begin + VPS - 1) / VPS);
    const int npairs = a.C * a.S;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; s++) {
            tc::mbar_init(&full[s], 2 * TC_B_THREADS + 1);  // B of both CTAs + the peer's A landed
            tc::mbar_init(&empty[s], 1);
            tc::mbar_init(&afull[s], 1);
        }
        tc::mbar_init(done, 1);
        tc::mbar_init(cdone, 1);
        tc::mbar_init(drained, 2 * TC_B_THREADS);
        *abort_flag = 0;
        tc::fence_mbarrier_init();
    }
    if (warp == TC_MMA_WARP) tc::tmem_alloc_pair(tmem_slot, TC_TMEM_COLS);
    tc::tc_fence_before();
    __syncthreads();
    tc::cluster_sync();  // both CTAs' barriers exist before either arrives on the other's
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == TC_COPY_WARP) {
        // ---------------- streamed operand: this CTA's half of the readout tile, two bulk copies
        // (hi and lo planes of nr/2 rows) per stage
        if (lane == 0) {
            const uint32_t plane = uint32_t(a.nr / 2) * 128;
            const unsigned char* src =
                a.apack + ((int64_t(by) * 2 + rank) * a.apack_stages + v_begin / VPS) * int64_t(2 * plane);
            int issued[TC_STAGES];
            for (int s = 0; s < TC_STAGES; s++) issued[s] = -1;
            for (int it = 0; it < nstages; it++) {
                const int buf = it % TC_STAGES;
                if (!tc::mbar_wait(&empty[buf], ((it / TC_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::mbar_arrive_expect_tx(&afull[buf], 2 * plane);
                const unsigned char* blk = src + int64_t(it) * 2 * plane;
                tc::bulk_copy_g2s(smem + buf * TC_STAGE_BYTES, blk, plane, &afull[buf]);
                tc::bulk_copy_g2s(smem + buf * TC_STAGE_BYTES + TC_A_BYTES, blk + plane, plane, &afull[buf]);
                issued[buf] = it;
            }
            // copies still in flight land before the CTA can finish (bounded)
            for (int s = 0; s < TC_STAGES; s++)
                if (issued[s] >= 0) tc::mbar_wait(&afull[s], (issued[s] / TC_STAGES) & 1, a.status);
        }
    } else if (warp == TC_MMA_WARP && rank == 0) {
        // ---------------- MMA issuer (leader, one lane): M = 256 over both CTAs
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16_f32(2 * TC_M, a.nr);
            for (int it = 0; it < nstages; it++) {
                const int buf = it % TC_STAGES;
                if (it > 0 && it % TC_CHUNK_STAGES == 0) {
                    // end of an accumulation chunk: once its MMAs complete, the producers of both
                    // CTAs add the accumulator into the running sum; the next chunk starts from 0
                    tc::mma_commit_pair(cdone);
                    if (!tc::mbar_wait(drained, ((it / TC_CHUNK_STAGES) - 1) & 1, a.status)) *abort_flag = 1;
                    if (*(volatile int*)abort_flag) break;
                    tc::tc_fence_after();
                }
                if (!tc::mbar_wait(&full[buf], (it / TC_STAGES) & 1, a.status)) *abort_flag = 1;
                if (!tc::mbar_wait(&afull[buf], (it / TC_STAGES) & 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::tc_fence_after();
                // A (M): the generated rows; B (N): the streamed readouts
                const uint32_t base = tc::smem_u32(smem + buf * TC_STAGE_BYTES);
                const uint32_t bh = base, bl = base + TC_A_BYTES;
                const uint32_t ah = base + 2 * TC_A_BYTES, al = ah + TC_BH_BYTES;
#pragma unroll
                for (int ks = 0; ks < TC_K / 16; ks++) {
                    const uint32_t koff = ks * 32;  // 16 bf16 = 32 bytes along K inside the swizzle atom
                    const uint64_t dah = tc::sw128_kmajor_desc(ah + koff), dal = tc::sw128_kmajor_desc(al + koff);
                    const uint64_t dbh = tc::sw128_kmajor_desc(bh + koff), dbl = tc::sw128_kmajor_desc(bl + koff);
                    tc::mma_bf16_pair(tmem, dah, dbh, idesc, (it % TC_CHUNK_STAGES > 0 || ks > 0) ? 1u : 0u);
                    tc::mma_bf16_pair(tmem, dah, dbl, idesc, 1u);
                    tc::mma_bf16_pair(tmem, dal, dbh, idesc, 1u);
                }
                tc::mma_commit_pair(&empty[buf]);
            }
            tc::mma_commit_pair(done);
            tc::mbar_wait(done, 0, a.status);  // the MMAs finish before the TMEM is released
        }
        __syncwarp();
    } else if (warp == TC_MMA_WARP) {
        // ---------------- peer, warp 16: tell the leader when each stage's A has landed here
        if (lane == 0) {
            for (int it = 0; it < nstages; it++) {
                const int buf = it % TC_STAGES;
                if (!tc::mbar_wait(&afull[buf], (it / TC_STAGES) & 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::mbar_arrive_cluster(&full[buf], 0);
            }
            tc::mbar_wait(done, 0, a.status);
        }
        __syncwarp();
    } else {
        // ---------------- B producers: this CTA's TC_PAIRS / 2 pairs (rank·64 ..) × VPS voxels of
        // F = coil·w·E_k per stage; local B rows 2j, 2j+1 for local pair j.
        // thread → (8-byte half chunk hq = VPH voxels, group pg of TC_PPG consecutive pairs)
        const int t = threadIdx.x;
        const int hq = t & 15, pg = t >> 4;
        const int n_first = n_pair0 + int(rank) * (TC_PAIRS / 2) + pg * TC_PPG;
        const int c_first = n_first / a.S, k_first = n_first - c_first * a.S;
        const bool group_ok = n_first < npairs;
        // the group's start value E_{k_first} (k_first is a multiple of egk), step and coil·w
        // travel one stage ahead of their use
        const float2* e_row = a.estart + int64_t(k_first / a.egk) * a.nvoxels;
        const float2* w_row = a.coilw + int64_t(c_first) * a.nvoxels;
        float2 step[VPH], e0[VPH], cw[VPH], step_n[VPH], e0_n[VPH], cw_n[VPH];
        auto load_gen = [&](int it, float2 (&st)[VPH], float2 (&ee)[VPH], float2 (&ww)[VPH]) {
#pragma unroll
            for (int i = 0; i < VPH; i++) {
                const int v = v_begin + it * VPS + VPH * hq + i;
                st[i] = ee[i] = ww[i] = make_float2(0.f, 0.f);
                if (group_ok && v < v_end) {
                    st[i] = __ldg(a.vstep + v);
                    ee[i] = __ldg(e_row + v);
                    ww[i] = __ldg(w_row + v);
                }
            }
        };
        // TMEM lanes of this warp's quarter; warp w handles the 32-column chunks w/4, w/4 + 4, ...
        const uint32_t tmem_rows = tmem + (uint32_t((warp & 3) * 32) << 16);
        load_gen(0, step, e0, cw);
        for (int it = 0; it < nstages; it++) {
            const int buf = it % TC_STAGES;
            const int vbase = v_begin + it * VPS + VPH * hq;
            if (it > 0 && it % TC_CHUNK_STAGES == 0) {
                // fold the finished chunk into the running sum (FP32, round to nearest): the
                // accumulation error of the tensor core grows with the accumulated K, so no chunk
                // accumulates more than 512 K16 steps
                const int chunk = it / TC_CHUNK_STAGES;
                const bool waited = tc::mbar_wait(cdone, (chunk - 1) & 1, a.status);
                // one decision per warp (tcgen05.ld / st are warp-collective); the warp's lanes stay
                // together because every exit from this loop is decided per warp
                if (__any_sync(0xffffffffu, !waited || *(volatile int*)abort_flag)) {
                    *abort_flag = 1;
                    break;
                }
                tc::tc_fence_after();
#pragma unroll 1
                for (int col = (warp >> 2) * 32; col < a.nr; col += (col & 16) ? 112 : 16) {
                    // 16-column halves of the warp's 32-column chunks (w/4, w/4 + 4, ...)
                    float acc[16];
                    tc::tmem_load16(tmem_rows + uint32_t(col), acc);
                    if (chunk > 1) {
                        float sum[16];
                        tc::tmem_load16(tmem_rows + uint32_t(TC_SUM_COL + col), sum);
#pragma unroll
                        for (int i = 0; i < 16; i++) acc[i] += sum[i];
                    }
                    tc::tmem_store16(tmem_rows + uint32_t(TC_SUM_COL + col), acc);
                }
                tc::tc_fence_before();
                tc::mbar_arrive_cluster(drained, 0);
            }
            if (it + 1 < nstages) load_gen(it + 1, step_n, e0_n, cw_n);
            const bool freed = tc::mbar_wait(&empty[buf], ((it / TC_STAGES) & 1) ^ 1, a.status);
            if (__any_sync(0xffffffffu, !freed || *(volatile int*)abort_flag)) {
                *abort_flag = 1;
                break;
            }
            unsigned char* Bh = smem + buf * TC_STAGE_BYTES + 2 * TC_A_BYTES;
            unsigned char* Bl = Bh + TC_BH_BYTES;
            float2 G[VPH];
#pragma unroll
            for (int i = 0; i < VPH; i++) G[i] = cmul(e0[i], cw[i]);
            int c = c_first, k = k_first;
#pragma unroll
            for (int jj = 0; jj < TC_PPG; jj++) {
                const int j = pg * TC_PPG + jj;
                const bool pok = (n_first + jj) < npairs;
                if (jj > 0) {
                    if (++k == a.S) {
                        // next coil (only when TC_PPG does not divide S): restart at k = 0
                        k = 0;
                        ++c;
#pragma unroll
                        for (int i = 0; i < VPH; i++) {
                            const int v = vbase + i;
                            float2 e = make_float2(0.f, 0.f), w = e;
                            if (pok && v < v_end) {
                                e = __ldg(a.estart + v);
                                w = __ldg(a.coilw + int64_t(c) * a.nvoxels + v);
                            }
                            G[i] = cmul(e, w);
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < VPH; i++) G[i] = cmul(G[i], step[i]);
                    }
                }
                const float ks = float(k) - 0.5f * float(a.S);
                // one hi/lo split per value: BF16 rounding is sign-symmetric, so the split of
                // (x, -y) is the split of (x, y) with the upper sign bit flipped and the split
                // of (y, x) is the same pair with its halves swapped
                uint32_t h0[2], l0[2], h1[2], l1[2];
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    float2 F = pok ? G[JAC ? 0 : i] : make_float2(0.f, 0.f);
                    if (JAC && i == 1) F = make_float2(ks * F.x, ks * F.y);
                    uint32_t h, l;
                    tc::split2(F.x, F.y, h, l);
                    h0[i] = h ^ 0x80000000u;
                    l0[i] = l ^ 0x80000000u;
                    h1[i] = __byte_perm(h, 0, 0x1032);
                    l1[i] = __byte_perm(l, 0, 0x1032);
                }
                const uint32_t o0 = tc::sw128_offset(2 * j, hq >> 1) + (hq & 1) * 8;
                const uint32_t o1 = tc::sw128_offset(2 * j + 1, hq >> 1) + (hq & 1) * 8;
                *reinterpret_cast<uint2*>(Bh + o0) = make_uint2(h0[0], h0[1]);
                *reinterpret_cast<uint2*>(Bl + o0) = make_uint2(l0[0], l0[1]);
                *reinterpret_cast<uint2*>(Bh + o1) = make_uint2(h1[0], h1[1]);
                *reinterpret_cast<uint2*>(Bl + o1) = make_uint2(l1[0], l1[1]);
            }
            tc::fence_async_shared();
            tc::mbar_arrive_cluster(&full[buf], 0);
#pragma unroll
            for (int i = 0; i < VPH; i++) {
                step[i] = step_n[i];
                e0[i] = e0_n[i];
                cw[i] = cw_n[i];
            }
        }

        // ---------------- epilogue: D[row = 2j + re/im of local pair j][col = readout] → shared memory
        // T[j][col] (float2) → rows of out[c][r][k] along k. Warp w reads TMEM lanes 32·(w%4).. (its
        // quarter) and 32-column chunks w/4, w/4 + 4; all 16 warps then write readout rows.
        const bool waited = tc::mbar_wait(done, 0, a.status);
        tc::tc_fence_after();
        // one decision for all 512 producer threads (tcgen05.ld is .sync.aligned, the barriers
        // below need every participant)
        const bool ok = !tc::bar_red_or(1, TC_B_THREADS, !(waited && !*(volatile int*)abort_flag));
        if (ok) {
            float* T = reinterpret_cast<float*>(smem);  // [64][TP]; the stage buffers are free
            const int TP = 2 * a.nr + 2;                // row pitch (floats): conflict-free columns
            const int quarter = warp & 3;
            const int row = quarter * 32 + lane, jr = row >> 1, ri = row & 1;
            const bool chunked = nstages > TC_CHUNK_STAGES;  // earlier chunks are in the running sum
#pragma unroll 1
            for (int ch = warp >> 2; ch * 32 < a.nr; ch += 4) {
                float v[32];
                tc::tmem_load32(tmem_rows + uint32_t(ch * 32), v);
                if (chunked) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        float sum[16];
                        tc::tmem_load16(tmem_rows + uint32_t(TC_SUM_COL + ch * 32 + 16 * h), sum);
#pragma unroll
                        for (int i = 0; i < 16; i++) v[16 * h + i] += sum[i];
                    }
                }
#pragma unroll
                for (int i = 0; i < 32; i++)
                    if (ch * 32 + i < a.nr) T[jr * TP + 2 * (ch * 32 + i) + ri] = v[i];
            }
            tc::bar_sync(1, TC_B_THREADS);
            float2* outp = a.out + int64_t(bz) * npairs * a.R;
            int64_t base[2];
            bool pv[2];
#pragma unroll
            for (int m = 0; m < 2; m++) {
                const int n = n_pair0 + int(rank) * (TC_PAIRS / 2) + lane + 32 * m;
                const int cc = n / a.S, kk = n - cc * a.S;
                pv[m] = n < npairs;
                base[m] = int64_t(cc) * a.R * a.S + kk;
            }
#pragma unroll 1
            for (int col = warp; col < a.nr && r0 + col < a.R; col += TC_B_THREADS / 32) {
                const int64_t roff = int64_t(r0 + col) * a.S;
#pragma unroll
                for (int m = 0; m < 2; m++)
                    if (pv[m]) {
                        const float* t = T + (lane + 32 * m) * TP + 2 * col;
                        outp[base[m] + roff] = make_float2(t[0], t[1]);
                    }
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::cluster_sync();  // neither CTA leaves while the other may still signal it or read TMEM
    if (warp == TC_MMA_WARP) {
        tc::tc_fence_after();
        tc::tmem_dealloc_pair(tmem, TC_TMEM_COLS);
    }
}

// grid (2 × pair tiles, readout tiles, voxel splits); CTAs 2i, 2i + 1 form a cluster
template<bool JAC>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TC_THREADS, 1) tc_contract_kernel(TcArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    tc_tile<JAC>(a, blockIdx.x >> 1, blockIdx.y, blockIdx.z, smem_raw);
}

// tile grid of one contraction: (pair tiles, readout tiles, voxel splits), 2 CTAs per tile
__device__ __forceinline__ int3 tc_grid_of(const TcArgs& a) {
    return make_int3((a.C * a.S + TC_PAIRS - 1) / TC_PAIRS, (a.R + a.nr - 1) / a.nr,
                     (a.nvoxels + a.vchunk - 1) / a.vchunk);
}

// index of the job owning flattened block b: offsets[j] ≤ b < offsets[j + 1] (offsets ascending)
__device__ __forceinline__ int job_of_block(const int* __restrict__ offsets, int njobs, int b) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(offsets + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Batched contraction: one launch for many jobs. Flattened CTA b belongs to job j
// (cta_offsets[j] ≤ b < cta_offsets[j+1], all offsets even) and, with l = b - cta_offsets[j] and
// (nx, ny) the job's pair tiles and readout tiles, takes pair tile (l/2) % nx, readout tile
// (l/2 / nx) % ny and split (l/2) / (nx·ny) as rank l & 1; CTAs 2i, 2i+1 form a cluster. Jobs are
// ordered by decreasing work per CTA, so the block scheduler runs the longest tiles first.
template<bool JAC>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TC_THREADS, 1)
    tc_contract_batch_kernel(const TcArgs* __restrict__ jobs, const int* __restrict__ cta_offsets, int njobs) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ TcArgs job;
    __shared__ int3 tile;
    if (threadIdx.x == 0) {
        const int j = job_of_block(cta_offsets, njobs, blockIdx.x);
        job = jobs[j];
        const int3 g = tc_grid_of(job);
        const int l = blockIdx.x - cta_offsets[j], l2 = l >> 1;
        tile = make_int3(l2 % g.x, (l2 / g.x) % g.y, l2 / (g.x * g.y));
    }
    __syncthreads();
    tc_tile<JAC>(job, tile.x, tile.y, tile.z, smem_raw);
}

// batched tc_prep_kernel: flattened 128-thread block b → job j, voxel (b - offsets[j])·128 + t
template<bool JAC>
__global__ void tc_prep_batch_kernel(const TcArgs* __restrict__ jobs, const int* __restrict__ block_offsets,
                                     int njobs) {
    __shared__ TcArgs job;
    __shared__ int local;
    if (threadIdx.x == 0) {
        const int j = job_of_block(block_offsets, njobs, blockIdx.x);
        job = jobs[j];
        local = blockIdx.x - block_offsets[j];
    }
    __syncthreads();
    tc_prep_voxel<JAC>(job, local * blockDim.x + threadIdx.x);
}

// batched tc_pack_a_kernel: flattened 256-thread block b → job j, local block l = b - offsets[j]
// covering chunks (l % gx)·256 + t of padded readout row l / gx, gx = ⌈8·apack_stages / 256⌉
template<bool JAC>
__global__ void tc_pack_batch_kernel(const TcArgs* __restrict__ jobs, const int* __restrict__ block_offsets,
                                     int njobs) {
    __shared__ TcArgs job;
    __shared__ int local;
    if (threadIdx.x == 0) {
        const int j = job_of_block(block_offsets, njobs, blockIdx.x);
        job = jobs[j];
        local = blockIdx.x - block_offsets[j];
    }
    __syncthreads();
    const int gx = (job.apack_stages * 8 + 255) / 256;
    tc_pack_a<JAC>(job, (local % gx) * 256 + threadIdx.x, local / gx);
}

}  // namespace kernels

// The fewest readout tiles of at most 256, then the least padding at that count: nr = ⌈R / tiles⌉
// rounded up to 16 (224 for 1120 readouts, 256 for 743, 208 for 400). Every readout tile generates
// the (coil, sample) operand over all voxels again, and a narrow tile's MMAs no longer cover that
// generation: the earlier rule (the multiple of 16 that pads R least, ties to the wider tile) took
// 16-readout tiles for 743 readouts (752 rows instead of 768) and ran 10× slower than 256.
int tc_readout_tile(int R) {
    const int r = std::max(R, 1);
    const int tiles = div_ceil(r, 256);
    return div_ceil(div_ceil(r, tiles), 16) * 16;
}

namespace {
TcTuning cartesian_tuning(int nvoxels, int R, int S, int C, bool jac) {
    return tuned_tc(jac ? TcKind::CartesianJacobian : TcKind::CartesianSignal, R, nvoxels, int64_t(C) * S);
}
// the tuned readout tile when it pads R to at most 1/16 more rows than the built-in tile does (a
// tuning table entry covers a class of readout counts), else the built-in tile
int cartesian_tile(int nvoxels, int R, int S, int C, bool jac) {
    const int tile = cartesian_tuning(nvoxels, R, S, C, jac).tile;
    const int builtin = tc_readout_tile(R);
    auto padded = [R](int nr) { return int64_t(div_ceil(std::max(R, 1), nr)) * nr; };
    return tile > 0 && 16 * padded(tile) <= 17 * padded(builtin) ? tile : builtin;
}
}  // namespace

TcPlan tc_plan(int device, int nvoxels, int R, int S, int C, bool jac) {
    TcPlan p;
    const TcTuning tuning = cartesian_tuning(nvoxels, R, S, C, jac);
    p.ntiles = div_ceil(C * S, kernels::TC_PAIRS);
    p.nr = cartesian_tile(nvoxels, R, S, C, jac);
    p.mtiles = div_ceil(std::max(R, 1), p.nr);
    const int tiles = 2 * p.ntiles * p.mtiles;  // CTAs per voxel split
    const int vps = jac ? 16 : 32;
    int splits = 1;
    if (tuning.splits > 0) {
        // tuned: at most 64 splits and at least one voxel stage each
        splits = std::min({tuning.splits, 64, std::max(1, div_ceil(std::max(nvoxels, 1), vps))});
    } else {
        // split the voxel range over CTAs only to fill the GPU: pick the split count (≥ 16 stages
        // per split) whose grid leaves the least idle SM time in the last wave of one CTA per SM,
        // less 0.5 % per split for the partial tiles written and summed. (Accuracy needs no split:
        // the tensor core's FP32 accumulation error grows with the accumulated K, ~2e-4 relative
        // after 3750 K16 steps, measured, so each CTA folds its accumulator into an FP32 running sum
        // every 512 K16 steps.)
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int max_splits = std::max(1, std::min(64, nvoxels / (16 * vps)));
        double best = -1.0;
        for (int sp = 1; sp <= max_splits; sp++) {
            const int64_t ctas = int64_t(tiles) * sp;
            const int64_t waves = (ctas + sms - 1) / sms;
            const double eff = double(ctas) / double(waves * sms) - 0.005 * sp;
            if (eff > best + 1e-9) {
                best = eff;
                splits = sp;
            }
        }
    }
    p.vchunk = std::max(vps, div_ceil(div_ceil(std::max(nvoxels, 1), splits), vps) * vps);
    p.splits = std::max(1, div_ceil(nvoxels, p.vchunk));
    p.ctas = int64_t(tiles) * p.splits;
    return p;
}

TcTables tc_tables(int nvoxels, int R, int S, int C, bool jac) {
    TcTables t;
    const int64_t V = std::max(nvoxels, 0);
    const int vps = jac ? 16 : 32;
    t.egk = (S % kernels::TC_PPG == 0) ? kernels::TC_PPG : 1;
    t.apack_stages = div_ceil(std::max(nvoxels, 1), vps);
    t.nr = cartesian_tile(nvoxels, R, S, C, jac);
    auto align = [](int64_t b) { return (b + 255) / 256 * 256; };
    t.vstep = 0;
    t.estart = t.vstep + align(8 * V);
    t.coilw = t.estart + align(8 * V * (S / t.egk));
    t.jcoef = t.coilw + align(8 * V * C);
    t.apack = t.jcoef + align(jac ? 32 * V : 0);
    t.bytes = t.apack + int64_t(div_ceil(std::max(R, 1), t.nr)) * t.nr * t.apack_stages * 256;
    return t;
}

void tc_assign_tables(kernels::TcArgs& a, const TcTables& t, unsigned char* base) {
    a.vstep = reinterpret_cast<const float2*>(base + t.vstep);
    a.estart = reinterpret_cast<const float2*>(base + t.estart);
    a.egk = t.egk;
    a.coilw = reinterpret_cast<const float2*>(base + t.coilw);
    a.jcoef = reinterpret_cast<const float4*>(base + t.jcoef);
    a.apack = base + t.apack;
    a.apack_stages = t.apack_stages;
    a.nr = t.nr;
}

int tc_pack_blocks(int nr, int R, int apack_stages) {
    return div_ceil(apack_stages * 8, 256) * div_ceil(std::max(R, 1), nr) * nr;
}

namespace {

void set_tc_smem_attribute(bool jac, bool batch) {
    static std::once_flag once[4];
    std::call_once(once[int(jac) + 2 * int(batch)], [&] {
        const void* fn = batch ? (jac ? reinterpret_cast<const void*>(kernels::tc_contract_batch_kernel<true>)
                                      : reinterpret_cast<const void*>(kernels::tc_contract_batch_kernel<false>))
                               : (jac ? reinterpret_cast<const void*>(kernels::tc_contract_kernel<true>)
                                      : reinterpret_cast<const void*>(kernels::tc_contract_kernel<false>));
        COMPAS_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kernels::TC_SMEM));
    });
}

bool run_tc(const CompasContext& ctx, kernels::TcArgs a, bool jac, cfloat* out) {
    if (!tensor_cores_available(ctx.device())) return false;
    DeviceGuard guard(ctx.device());
    const int npairs = a.C * a.S;
    const TcPlan plan = tc_plan(ctx.device(), a.nvoxels, a.R, a.S, a.C, jac);
    const int splits = plan.splits;
    a.vchunk = plan.vchunk;
    const int64_t n = int64_t(npairs) * a.R;
    Array<cfloat, 2> partials({splits > 1 ? splits : 0, n}, ctx.device(), ctx.stream());
    const TcTables tables = tc_tables(a.nvoxels, a.R, a.S, a.C, jac);
    Array<unsigned char> scratch({tables.bytes}, ctx.device(), ctx.stream());
    tc_assign_tables(a, tables, scratch.data());
    a.out = reinterpret_cast<float2*>(splits > 1 ? partials.data() : out);
    a.status = ctx.status_word();
    // per-voxel tables, then A packed once (one pass over the echoes instead of one per pair tile)
    const dim3 pgrid(div_ceil(a.apack_stages * 8, 256), plan.mtiles * plan.nr);
    if (jac) {
        kernels::tc_prep_kernel<true><<<div_ceil(a.nvoxels, 128), 128, 0, ctx.stream()>>>(a);
        kernels::tc_pack_a_kernel<true><<<pgrid, 256, 0, ctx.stream()>>>(a);
    } else {
        kernels::tc_prep_kernel<false><<<div_ceil(a.nvoxels, 128), 128, 0, ctx.stream()>>>(a);
        kernels::tc_pack_a_kernel<false><<<pgrid, 256, 0, ctx.stream()>>>(a);
    }
    check_launch("tc_prep_kernel / tc_pack_a_kernel");
    auto fn = jac ? kernels::tc_contract_kernel<true> : kernels::tc_contract_kernel<false>;
    set_tc_smem_attribute(jac, false);
    dim3 grid(2 * plan.ntiles, plan.mtiles, splits);
    fn<<<grid, kernels::TC_THREADS, kernels::TC_SMEM, ctx.stream()>>>(a);
    check_launch("tc_contract_kernel");
    if (splits > 1) sum_partials(ctx, partials.data(), splits, n, out);
    return true;
}

kernels::TcArgs common_args(const float* params, int64_t pstride, int nvoxels, const cfloat* echos,
                            const cfloat* coils, int ncoils, const CartesianGeom& g) {
    kernels::TcArgs a {};
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
    return a;
}

}  // namespace

bool launch_signal_cartesian_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                const cfloat* echos, const cfloat* coils, int ncoils, const CartesianGeom& g,
                                cfloat* signal) {
    if (int64_t(ncoils) * g.nreadouts * g.ns == 0) return true;
    if (nvoxels == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(signal, 0, sizeof(cfloat) * size_t(ncoils) * g.nreadouts * g.ns, ctx.stream()));
        return true;
    }
    return run_tc(ctx, common_args(params, pstride, nvoxels, echos, coils, ncoils, g), false, signal);
}

bool launch_jacobian_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                        const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils, int ncoils,
                        const cfloat* vec, const CartesianGeom& g, cfloat* Jv) {
    if (int64_t(ncoils) * g.nreadouts * g.ns == 0) return true;
    if (nvoxels == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(Jv, 0, sizeof(cfloat) * size_t(ncoils) * g.nreadouts * g.ns, ctx.stream()));
        return true;
    }
    auto a = common_args(params, pstride, nvoxels, echos, coils, ncoils, g);
    a.dT1 = reinterpret_cast<const float2*>(dT1);
    a.dT2 = reinterpret_cast<const float2*>(dT2);
    a.vec = reinterpret_cast<const float2*>(vec);
    return run_tc(ctx, a, true, Jv);
}

kernels::TcArgs tc_signal_args(const float* params, int64_t pstride, int nvoxels, const cfloat* echos,
                               const cfloat* coils, int ncoils, const CartesianGeom& g) {
    return common_args(params, pstride, nvoxels, echos, coils, ncoils, g);
}

void launch_tc_batch(cudaStream_t stream, int device, bool jac, const kernels::TcArgs* jobs, int njobs,
                     const int* prep_offsets, int prep_blocks, const int* pack_offsets, int pack_blocks,
                     const int* cta_offsets, int ctas) {
    if (njobs <= 0) return;
    DeviceGuard guard(device);
    if (prep_blocks > 0) {
        if (jac) kernels::tc_prep_batch_kernel<true><<<prep_blocks, 128, 0, stream>>>(jobs, prep_offsets, njobs);
        else kernels::tc_prep_batch_kernel<false><<<prep_blocks, 128, 0, stream>>>(jobs, prep_offsets, njobs);
        check_launch("tc_prep_batch_kernel");
    }
    if (pack_blocks > 0) {
        if (jac) kernels::tc_pack_batch_kernel<true><<<pack_blocks, 256, 0, stream>>>(jobs, pack_offsets, njobs);
        else kernels::tc_pack_batch_kernel<false><<<pack_blocks, 256, 0, stream>>>(jobs, pack_offsets, njobs);
        check_launch("tc_pack_batch_kernel");
    }
    if (ctas <= 0) return;
    set_tc_smem_attribute(jac, true);
    if (jac)
        kernels::tc_contract_batch_kernel<true><<<ctas, kernels::TC_THREADS, kernels::TC_SMEM, stream>>>(jobs, cta_offsets, njobs);
    else
        kernels::tc_contract_batch_kernel<false><<<ctas, kernels::TC_THREADS, kernels::TC_SMEM, stream>>>(jobs, cta_offsets, njobs);
    check_launch("tc_contract_batch_kernel");
}

}  // namespace compas
