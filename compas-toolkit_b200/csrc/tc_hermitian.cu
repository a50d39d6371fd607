// tc_hermitian.cu — compute_jacobian_hermitian (Jᴴ·v) on tcgen05 tensor cores, split-BF16.
//
// Reference math: src/jacobian/hermitian_kernels.cuh:30-92 (see hermitian.cu for the
// regrouping). For every voxel v and (readout r, coil c) pair p:
//   Y_p(v) = Σ_k u[c][r][k]·conj(E_k(v)),   Ỹ_p(v) = Σ_k (k - S/2)·u[c][r][k]·conj(E_k(v))
// is a GEMM with M = voxels, N = pairs, K = samples. A CTA owns 128 voxels (the 128 TMEM
// lanes), so the follow-up contraction over readouts with the echoes
//   mHv_c += conj(m[r])·Y,  dmHv0_c += conj(∂T1m[r])·Y,  dmHv1_c += conj(∂T2m[r])·Y + ΔtR2²·conj(m[r])·Ỹ
// happens inside each epilogue thread; the four per-voxel results never leave registers, every
// echo element is read once for all coils, and no [R][V] temporary is written (the reference
// writes two FP32 [2][R][V] arrays per coil and re-reads the echoes per coil).
//
// Real-ified operands (re/im interleaved along K = 2S):
//   A'[v]            = (Re ē_k, Im ē_k) with ē = conj(E_k(v))     — generated, 128 voxels × 32 samples/stage
//   B'[0·64 + p]     = (u_re, -u_im)     → Y_re    B'[1·64 + p] = (u_im, u_re)      → Y_im
//   B'[2·64 + p]     = (k-S/2)(u_re, -u_im) → Ỹ_re B'[3·64 + p] = (k-S/2)(u_im, u_re) → Ỹ_im
// D[128 voxels][256] accumulates in TMEM; two accumulators (512 columns) alternate between
// consecutive pair tiles so the epilogue of tile t overlaps the MMAs of tile t+1.
// Warp roles: 0-7 epilogue (warps w and w+4 share TMEM lanes 32(w%4).. = voxels and split each
// tile's pairs), 8-11 generate A, 12-15 convert u (B), 16 allocates TMEM and issues the MMAs.
// All waits are bounded.
#include <cuda_bf16.h>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {

void sum_partials(const CompasContext& ctx, const cfloat* partials, int nsplit, int64_t n, cfloat* out);

namespace kernels {

constexpr int TH_M = 128, TH_N = 256, TH_K = 64, TH_PAIRS = 64;
constexpr int TH_THREADS = 544;  // 8 epilogue + 4 A + 4 B warps + 1 MMA warp
constexpr int TH_STAGES = 2;
constexpr int TH_A_BYTES = TH_M * TH_K * 2;
constexpr int TH_B_BYTES = TH_N * TH_K * 2;
constexpr int TH_STAGE_BYTES = 2 * TH_A_BYTES + 2 * TH_B_BYTES;
constexpr int TH_SMEM = TH_STAGES * TH_STAGE_BYTES + 1024 + 256;

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
    float2* out;          // [splits][4][V]
    unsigned int* status;
};

__global__ void __launch_bounds__(TH_THREADS, 1) tc_hermitian_kernel(ThArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TH_STAGES * TH_STAGE_BYTES);
    uint64_t* empty = full + TH_STAGES;
    uint64_t* acc_full = empty + TH_STAGES;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int v0 = blockIdx.x * TH_M;
    const int split = blockIdx.y;
    const int npairs = a.R * a.C;
    const int ntiles_total = (npairs + TH_PAIRS - 1) / TH_PAIRS;
    const int tile_begin = split * a.tiles_per_split;
    const int tile_end = min(ntiles_total, tile_begin + a.tiles_per_split);
    const int ntiles = max(0, tile_end - tile_begin);
    const int kstages = (a.S + 31) / 32;  // 32 samples (64 K) per stage

    if (threadIdx.x == 0) {
        for (int s = 0; s < TH_STAGES; s++) {
            tc::mbar_init(&full[s], 256);
            tc::mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < 2; s++) {
            tc::mbar_init(&acc_full[s], 1);
            tc::mbar_init(&acc_empty[s], 256);
        }
        tc::mbar_init(done, 1);
        *abort_flag = 0;
        tc::fence_mbarrier_init();
    }
    if (warp == 16) tc::tmem_alloc(tmem_slot, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const double twopi = 6.283185307179586476925;

    if (warp < 12) {
        // per-voxel constants: warps 0-7 (epilogue) and 8-11 (A producer) own voxel v0 + (tid & 127)
        const int t = threadIdx.x & 127;
        const int v = v0 + t;
        const bool vok = v < a.nvoxels;
        const int vc = vok ? v : (a.nvoxels - 1);
        const float T1 = a.params[vc], T2 = a.params[a.pstride + vc], B0 = a.params[3 * a.pstride + vc];
        const float x = a.params[6 * a.pstride + vc], y = a.params[7 * a.pstride + vc];
        const double theta = double(a.dk_re) * x + double(a.dk_im) * y + double(a.dt) * twopi * B0;
        const float decay = -a.dt / T2;
        if (warp >= 8) {
            // ---------------- A producer: 32 samples of conj(E_k(v)) per stage, row t
            const float2 st = cis_rad(theta);
            const float sm = __expf(decay);
            const float2 step = make_float2(sm * st.x, sm * st.y);
            int g = 0;  // global stage counter (same order as the B producer and the MMA issuer)
            for (int tl = 0; tl < ntiles; tl++) {
                for (int ks = 0; ks < kstages; ks++, g++) {
                    const int buf = g % TH_STAGES;
                    if (!tc::mbar_wait(&empty[buf], ((g / TH_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
                    if (*(volatile int*)abort_flag) break;
                    unsigned char* Ah = smem + buf * TH_STAGE_BYTES;
                    unsigned char* Al = Ah + TH_A_BYTES;
                    // exact restarts at k0 and k0+16 (FP64-reduced phase), recurrence between
#pragma unroll
                    for (int half = 0; half < 2; half++) {
                        const int kb = ks * 32 + half * 16;
                        const float s0 = float(kb) - 0.5f * float(a.S);
                        const float2 ph = cis_rad(double(s0) * theta);
                        const float mg = __expf(s0 * decay);
                        float2 e = make_float2(mg * ph.x, mg * ph.y);
#pragma unroll
                        for (int cq = 0; cq < 4; cq++) {  // 4 chunks of 4 samples
                            uint32_t h[4], l[4];
#pragma unroll
                            for (int i = 0; i < 4; i++) {
                                const bool kok = vok && (kb + 4 * cq + i) < a.S;
                                tc::split2(kok ? e.x : 0.0f, kok ? -e.y : 0.0f, h[i], l[i]);
                                e = cmul(e, step);
                            }
                            const uint32_t off = tc::sw128_offset(t, half * 4 + cq);
                            *reinterpret_cast<uint4*>(Ah + off) = make_uint4(h[0], h[1], h[2], h[3]);
                            *reinterpret_cast<uint4*>(Al + off) = make_uint4(l[0], l[1], l[2], l[3]);
                        }
                    }
                    tc::fence_async_shared();
                    tc::mbar_arrive(&full[buf]);
                }
                if (*(volatile int*)abort_flag) break;
            }
        } else {
            // ---------------- epilogue: thread = voxel = TMEM lane 32·(warp%4) + lane; warps w and
            // w+4 take alternate 8-pair chunks of every tile
            const float2 rho = make_float2(a.params[4 * a.pstride + vc], a.params[5 * a.pstride + vc]);
            const float R2 = 1.0f / T2;
            const float dscale = a.dt * R2 * R2;
            const int quarter = warp & 3, parity = warp >> 2;
            float2 acc[4];
#pragma unroll
            for (int f = 0; f < 4; f++) acc[f] = make_float2(0.f, 0.f);
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
                    // loads first (echo, ∂echo, coil of the 8 pairs), then the TMEM reads and math
                    float2 m[8], m1[8], m2[8], cc[8];
                    {
                        int r = pb / a.C, c = pb - r * a.C;
#pragma unroll
                        for (int i = 0; i < 8; i++) {
                            if (vok && pb + i < npairs) {
                                const int64_t idx = int64_t(r) * a.nvoxels + v;
                                m[i] = __ldg(a.echo + idx);
                                m1[i] = __ldg(a.dT1 + idx);
                                m2[i] = __ldg(a.dT2 + idx);
                                cc[i] = __ldg(a.coils + int64_t(c) * a.nvoxels + v);
                            } else {
                                m[i] = m1[i] = m2[i] = cc[i] = make_float2(0.f, 0.f);
                            }
                            if (++c == a.C) {
                                c = 0;
                                ++r;
                            }
                        }
                    }
                    float yr[8], yi[8], tr[8], ti[8];
                    tc::tmem_load8(tbase + 0 * 64 + ch * 8, yr);
                    tc::tmem_load8(tbase + 1 * 64 + ch * 8, yi);
                    tc::tmem_load8(tbase + 2 * 64 + ch * 8, tr);
                    tc::tmem_load8(tbase + 3 * 64 + ch * 8, ti);
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const float2 Y = make_float2(yr[i], yi[i]), Yt = make_float2(tr[i], ti[i]);
                        const float2 mH = cmulc(Y, m[i]);
                        const float2 d0 = cmulc(Y, m1[i]);
                        const float2 dd1 = cadd(cmulc(Y, m2[i]), cscale(dscale, cmulc(Yt, m[i])));
                        const float2 rc = cmul(rho, cc[i]);
                        acc[0] = cadd(acc[0], cmulc(d0, cscale(T1, rc)));
                        acc[1] = cadd(acc[1], cmulc(dd1, cscale(T2, rc)));
                        const float2 cm = cmulc(mH, cc[i]);
                        acc[2] = cadd(acc[2], cm);
                        acc[3] = cadd(acc[3], make_float2(cm.y, -cm.x));
                    }
                }
                tc::tc_fence_before();
                tc::mbar_arrive(&acc_empty[abuf]);
            }
            // combine the two warps of each lane quarter through shared memory (stage buffer 0,
            // free once every tile has been consumed) and write the four results
            float2* red = reinterpret_cast<float2*>(smem);
            asm volatile("bar.sync 2, 256;" ::: "memory");  // epilogue warps only: all MMAs consumed
            if (parity == 1) {
#pragma unroll
                for (int f = 0; f < 4; f++) red[f * 128 + t] = acc[f];
            }
            asm volatile("bar.sync 2, 256;" ::: "memory");
            if (parity == 0 && ok && vok && !*(volatile int*)abort_flag) {
                float2* o = a.out + int64_t(split) * 4 * a.nvoxels;
#pragma unroll
                for (int f = 0; f < 4; f++) o[int64_t(f) * a.nvoxels + v] = cadd(acc[f], red[f * 128 + t]);
            }
        }
    } else if (warp < 16) {
        // ---------------- B producer: u → rows (u_re,-u_im), (u_im,u_re) and their (k-S/2)-scaled copies
        const int t = threadIdx.x - 384;
        const int pl = t & 63, half = t >> 6;  // pair within tile, 16-sample half of the stage
        int g = 0;
        for (int tl = 0; tl < ntiles; tl++) {
            const int p = (tile_begin + tl) * TH_PAIRS + pl;
            const bool pok = p < npairs;
            const int r = pok ? p / a.C : 0, c = pok ? p - r * a.C : 0;
            const float2* urow = a.u + (int64_t(c) * a.R + r) * a.S;
            for (int ks = 0; ks < kstages; ks++, g++) {
                const int buf = g % TH_STAGES;
                const int kb = ks * 32 + half * 16;
                float2 uv[16];
#pragma unroll
                for (int i = 0; i < 16; i++)
                    uv[i] = (pok && kb + i < a.S) ? __ldg(urow + kb + i) : make_float2(0.f, 0.f);
                if (!tc::mbar_wait(&empty[buf], ((g / TH_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                unsigned char* Bh = smem + buf * TH_STAGE_BYTES + 2 * TH_A_BYTES;
                unsigned char* Bl = Bh + TH_B_BYTES;
#pragma unroll
                for (int cq = 0; cq < 4; cq++) {  // 4 samples per 16-byte chunk
                    uint32_t h0[4], l0[4], h1[4], l1[4], h2[4], l2[4], h3[4], l3[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float2 w = uv[4 * cq + i];
                        const float ksf = float(kb + 4 * cq + i) - 0.5f * float(a.S);
                        tc::split2(w.x, -w.y, h0[i], l0[i]);
                        tc::split2(w.y, w.x, h1[i], l1[i]);
                        tc::split2(ksf * w.x, -ksf * w.y, h2[i], l2[i]);
                        tc::split2(ksf * w.y, ksf * w.x, h3[i], l3[i]);
                    }
                    const int chunk = half * 4 + cq;
                    const uint32_t o0 = tc::sw128_offset(0 * 64 + pl, chunk), o1 = tc::sw128_offset(1 * 64 + pl, chunk);
                    const uint32_t o2 = tc::sw128_offset(2 * 64 + pl, chunk), o3 = tc::sw128_offset(3 * 64 + pl, chunk);
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
            }
            if (*(volatile int*)abort_flag) break;
        }
    } else {
        // ---------------- MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(TH_M, TH_N);
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
                    if (*(volatile int*)abort_flag) break;
                    tc::tc_fence_after();
                    const uint32_t base = tc::smem_u32(smem + buf * TH_STAGE_BYTES);
                    const uint32_t ah = base, al = base + TH_A_BYTES;
                    const uint32_t bh = base + 2 * TH_A_BYTES, bl = bh + TH_B_BYTES;
#pragma unroll
                    for (int k16 = 0; k16 < TH_K / 16; k16++) {
                        const uint32_t koff = k16 * 32;
                        const uint64_t dah = tc::sw128_kmajor_desc(ah + koff), dal = tc::sw128_kmajor_desc(al + koff);
                        const uint64_t dbh = tc::sw128_kmajor_desc(bh + koff), dbl = tc::sw128_kmajor_desc(bl + koff);
                        tc::mma_bf16(d, dah, dbh, idesc, (ks > 0 || k16 > 0) ? 1u : 0u);
                        tc::mma_bf16(d, dah, dbl, idesc, 1u);
                        tc::mma_bf16(d, dal, dbh, idesc, 1u);
                    }
                    tc::mma_commit(&empty[buf]);
                }
                tc::mma_commit(&acc_full[abuf]);
            }
            tc::mma_commit(done);
            tc::mbar_wait(done, 0, a.status);  // all MMAs complete before TMEM is released
        }
        __syncwarp();
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 16) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

}  // namespace kernels

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
    a.status = detail::device_status_word(ctx.device());
    const int vtiles = div_ceil(nvoxels, kernels::TH_M);
    const int ptiles = div_ceil(ncoils * g.nreadouts, kernels::TH_PAIRS);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device());
    // split the pair tiles over CTAs (≥ 4 tiles each) to minimise the idle part of the last wave
    int splits = 1;
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
    a.tiles_per_split = div_ceil(ptiles, splits);
    splits = div_ceil(ptiles, a.tiles_per_split);
    const int64_t n = 4 * int64_t(nvoxels);
    Array<cfloat, 2> partials({splits > 1 ? splits : 0, n}, ctx.device(), ctx.stream());
    a.out = reinterpret_cast<float2*>(splits > 1 ? partials.data() : JHv);
    static bool attr_set = false;
    if (!attr_set) {
        COMPAS_CUDA_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(kernels::tc_hermitian_kernel),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, kernels::TH_SMEM));
        attr_set = true;
    }
    dim3 grid(vtiles, splits);
    kernels::tc_hermitian_kernel<<<grid, kernels::TH_THREADS, kernels::TH_SMEM, ctx.stream()>>>(a);
    check_launch("tc_hermitian_kernel");
    if (splits > 1) sum_partials(ctx, partials.data(), splits, n, JHv);
    return true;
}

}  // namespace compas
