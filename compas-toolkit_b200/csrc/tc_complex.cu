// tc_complex.cu — split-BF16 tcgen05 tensor-core kernels for the Cartesian signal and J·v.
//
// Both operations are voxel contractions of a streamed operand A with a generated operand B
// (see signal.cu for the algebra, reference src/trajectories/signal_kernels.cuh:137-167 and
// src/jacobian/product_kernels.cuh:7-67):
//   signal: out[c][r][k] = Σ_v echo[r][v] · F_{c,k}(v),        F = coil·ρ·E_k·e^{i(S/2)Δk_im y}
//   J·v:    out[c][r][k] = Σ_v P[r][v]·F_{c,k}(v) + Q'[r][v]·(k-S/2)·F_{c,k}(v),  F = coil·E_k
// The complex contraction is real-ified by interleaving re/im along K: A'[r] = (A_re, A_im) per
// complex term, B'[2j] = (F_re, -F_im), B'[2j+1] = (F_im, F_re) per output pair j = (c, k), so
// one real GEMM D[128 readouts][256 = 128 pairs × re/im] = A'·B'ᵀ yields the complex tile.
//
// Precision: every operand x is split as x = hi + lo (two BF16s, |x - hi - lo| ≤ 2⁻¹⁸|x|) and the
// product is accumulated in FP32 TMEM as hi·hi + hi·lo + lo·hi (three tcgen05.mma per K step);
// the dropped lo·lo term is ≤ 2⁻¹⁶ relative, giving ~1e-5 relative L2 against FP64.
//
// CTA organisation (288 threads, 1 CTA/SM, 192 KB shared memory in 2 pipeline stages):
//   warps 0-3  convert the A tile (128 readouts × 64 K) from the FP32 echoes into BF16 hi/lo,
//              128-byte swizzled K-major, and afterwards drain the TMEM accumulator;
//   warps 4-7  generate the B tile (256 rows × 64 K): E_k by an exact FP64-reduced start and a
//              complex recurrence along k, times the per-voxel coil (and ρ) factor;
//   warp 8     allocates 256 TMEM columns and one lane issues the 12 MMAs per stage.
// Stages hand over through mbarriers (full: producers → MMA, empty: tcgen05.commit → producers).
// The voxel range is split over CTAs (split-K); partial tiles are summed in a fixed order.
#include <cuda_bf16.h>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {

void sum_partials(const CompasContext& ctx, const cfloat* partials, int nsplit, int64_t n, cfloat* out);

namespace kernels {

constexpr int TC_M = 128, TC_N = 256, TC_K = 64;  // real-ified tile; TC_N/2 = 128 complex pairs
constexpr int TC_THREADS = 288;
constexpr int TC_STAGES = 2;
constexpr int TC_A_BYTES = TC_M * TC_K * 2;  // 16 KB per hi/lo plane
constexpr int TC_B_BYTES = TC_N * TC_K * 2;  // 32 KB per hi/lo plane
constexpr int TC_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TC_B_BYTES;
constexpr int TC_SMEM = TC_STAGES * TC_STAGE_BYTES + 1024 /*align*/ + 128 /*barriers*/;

struct TcArgs {
    const float* params;
    int64_t pstride;
    int nvoxels;
    const float2* echo;   // [R][V]
    const float2* dT1;    // J·v only
    const float2* dT2;
    const float2* vec;    // J·v only: [4][V]
    const float2* coils;  // [C][V]
    int R, S, C;
    float dt, dk_re, dk_im;
    int vchunk;           // voxels per split
    float2* out;          // [splits][C][R][S]
    unsigned int* status;
};

template<bool JAC>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_contract_kernel(TcArgs a) {
    constexpr int TERMS = JAC ? 2 : 1;            // complex terms per voxel along K
    constexpr int VPS = TC_K / (2 * TERMS);       // voxels per stage (32 or 16)
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TC_STAGES * TC_STAGE_BYTES);
    uint64_t* empty = full + TC_STAGES;
    uint64_t* done = empty + TC_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_pair0 = blockIdx.x * (TC_N / 2);          // first (c,k) pair of this tile
    const int r0 = blockIdx.y * TC_M;
    const int split = blockIdx.z;
    const int v_begin = split * a.vchunk;
    const int v_end = min(a.nvoxels, v_begin + a.vchunk);
    const int nstages = max(1, (v_end - v_begin + VPS - 1) / VPS);
    const int npairs = a.C * a.S;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; s++) {
            tc::mbar_init(&full[s], 256);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(done, 1);
        *abort_flag = 0;
        tc::fence_mbarrier_init();
    }
    if (warp == 8) tc::tmem_alloc(tmem_slot, 256);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < 4) {
        // ---------------- A producer: 128 readouts × VPS voxels → BF16 hi/lo, swizzled
        const int t = threadIdx.x;          // 0..127
        const int chunk = t & 7, rsub = t >> 3;  // 8 chunks per row, 16 rows per pass
        for (int it = 0; it < nstages; it++) {
            const int buf = it % TC_STAGES;
            if (!tc::mbar_wait(&empty[buf], ((it / TC_STAGES) & 1) ^ 1, a.status)) {
                *abort_flag = 1;
            }
            if (*(volatile int*)abort_flag) break;
            unsigned char* Ah = smem + buf * TC_STAGE_BYTES;
            unsigned char* Al = Ah + TC_A_BYTES;
            const int v0 = v_begin + it * VPS;
#pragma unroll 2
            for (int pass = 0; pass < TC_M / 16; pass++) {
                const int rl = rsub + 16 * pass;
                const int r = r0 + rl;
                float x[8];
                if constexpr (!JAC) {
                    // chunk covers voxels 4·chunk .. 4·chunk+3 (re, im interleaved)
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int v = v0 + 4 * chunk + q;
                        float2 e = make_float2(0.f, 0.f);
                        if (r < a.R && v < v_end) e = __ldg(a.echo + int64_t(r) * a.nvoxels + v);
                        x[2 * q] = e.x;
                        x[2 * q + 1] = e.y;
                    }
                } else {
                    // chunk covers voxels 2·chunk, 2·chunk+1, each (P_re, P_im, Q'_re, Q'_im)
#pragma unroll
                    for (int q = 0; q < 2; q++) {
                        const int v = v0 + 2 * chunk + q;
                        float2 P = make_float2(0.f, 0.f), Q = P;
                        if (r < a.R && v < v_end) {
                            const int64_t idx = int64_t(r) * a.nvoxels + v;
                            const float T1 = a.params[v], T2 = a.params[a.pstride + v];
                            const float2 rho = make_float2(a.params[4 * a.pstride + v], a.params[5 * a.pstride + v]);
                            const float2 me = __ldg(a.echo + idx), d1 = __ldg(a.dT1 + idx), d2 = __ldg(a.dT2 + idx);
                            const float2 w0 = a.vec[v], w1 = a.vec[a.nvoxels + v];
                            const float2 w2 = a.vec[2 * int64_t(a.nvoxels) + v], w3 = a.vec[3 * int64_t(a.nvoxels) + v];
                            const float2 t1r = cscale(T1, rho), t2r = cscale(T2, rho);
                            P = cmul(cmul(w0, t1r), d1);
                            P = cadd(P, cmul(cmul(w1, t2r), d2));
                            P = cadd(P, cmul(w2, me));
                            P = cadd(P, cmul(make_float2(-w3.y, w3.x), me));
                            const float R2 = 1.0f / T2;
                            Q = cscale(a.dt * R2 * R2, cmul(cmul(w1, t2r), me));
                        }
                        x[4 * q] = P.x;
                        x[4 * q + 1] = P.y;
                        x[4 * q + 2] = Q.x;
                        x[4 * q + 3] = Q.y;
                    }
                }
                uint32_t h[4], l[4];
#pragma unroll
                for (int q = 0; q < 4; q++) tc::split2(x[2 * q], x[2 * q + 1], h[q], l[q]);
                const uint32_t off = tc::sw128_offset(rl, chunk);
                *reinterpret_cast<uint4*>(Ah + off) = make_uint4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<uint4*>(Al + off) = make_uint4(l[0], l[1], l[2], l[3]);
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
        }
    } else if (warp < 8) {
        // ---------------- B producer: 128 pairs × VPS voxels of F = factor·E_k
        const int t = threadIdx.x - 128;          // 0..127
        const double twopi = 6.283185307179586476925;
        // thread → (voxel slot vs, pair group pg): VPS voxels × (128/VPS) groups of pairs
        constexpr int GROUPS = 128 / VPS;         // 4 (signal) or 8 (J·v)
        constexpr int PPG = (TC_N / 2) / GROUPS;  // pairs per group: 32 or 16
        const int vs = t % VPS, pg = t / VPS;
        for (int it = 0; it < nstages; it++) {
            const int buf = it % TC_STAGES;
            if (!tc::mbar_wait(&empty[buf], ((it / TC_STAGES) & 1) ^ 1, a.status)) {
                *abort_flag = 1;
            }
            if (*(volatile int*)abort_flag) break;
            unsigned char* Bh = smem + buf * TC_STAGE_BYTES + 2 * TC_A_BYTES;
            unsigned char* Bl = Bh + TC_B_BYTES;
            const int v = v_begin + it * VPS + vs;
            const bool vok = v < v_end;
            const int vc = vok ? v : 0;
            const float T2 = a.params[a.pstride + vc], B0 = a.params[3 * a.pstride + vc];
            const float x = a.params[6 * a.pstride + vc], y = a.params[7 * a.pstride + vc];
            const double theta = double(a.dk_re) * x + double(a.dk_im) * y + double(a.dt) * twopi * B0;
            const float decay = -a.dt / T2;
            float2 wv = make_float2(1.f, 0.f);
            if constexpr (!JAC) {
                wv = make_float2(a.params[4 * a.pstride + vc], a.params[5 * a.pstride + vc]);
                if (a.dk_im != 0.0f) wv = cmul(wv, cis_rad(0.5 * double(a.S) * double(a.dk_im) * y));
            }
            const float2 st = cis_rad(theta);
            const float sm = __expf(decay);
            const float2 step = make_float2(sm * st.x, sm * st.y);
            int cur_c = -1;
            float2 e = make_float2(0.f, 0.f), wc = e;
            for (int jj = 0; jj < PPG; jj++) {
                const int j = pg * PPG + jj;       // pair within tile
                const int n = n_pair0 + j;         // global pair
                float2 F = make_float2(0.f, 0.f);
                float ks = 0.0f;
                if (vok && n < npairs) {
                    const int c = n / a.S, k = n - c * a.S;
                    ks = float(k) - 0.5f * float(a.S);
                    if (c != cur_c || jj % 16 == 0) {  // exact restart (new coil, or every 16 samples)
                        const float2 ph = cis_rad(double(ks) * theta);
                        const float mg = __expf(ks * decay);
                        e = make_float2(mg * ph.x, mg * ph.y);
                        if (c != cur_c) {
                            wc = cmul(a.coils[int64_t(c) * a.nvoxels + v], wv);
                            cur_c = c;
                        }
                    } else {
                        e = cmul(e, step);
                    }
                    F = cmul(e, wc);
                }
                // rows 2j: (F_re, -F_im), 2j+1: (F_im, F_re) at K' = TERMS·2·vs (+2 for the Q' term)
                uint32_t h0, l0, h1, l1;
                tc::split2(F.x, -F.y, h0, l0);
                tc::split2(F.y, F.x, h1, l1);
                const int kk = TERMS * 2 * vs;                     // bf16 index along K
                const int chunk = kk >> 3, within = (kk & 7) * 2;  // byte offset inside the chunk
                const uint32_t o0 = tc::sw128_offset(2 * j, chunk) + within;
                const uint32_t o1 = tc::sw128_offset(2 * j + 1, chunk) + within;
                if constexpr (!JAC) {
                    *reinterpret_cast<uint32_t*>(Bh + o0) = h0;
                    *reinterpret_cast<uint32_t*>(Bl + o0) = l0;
                    *reinterpret_cast<uint32_t*>(Bh + o1) = h1;
                    *reinterpret_cast<uint32_t*>(Bl + o1) = l1;
                } else {
                    uint32_t h2, l2, h3, l3;
                    tc::split2(ks * F.x, -ks * F.y, h2, l2);
                    tc::split2(ks * F.y, ks * F.x, h3, l3);
                    *reinterpret_cast<uint2*>(Bh + o0) = make_uint2(h0, h2);
                    *reinterpret_cast<uint2*>(Bl + o0) = make_uint2(l0, l2);
                    *reinterpret_cast<uint2*>(Bh + o1) = make_uint2(h1, h3);
                    *reinterpret_cast<uint2*>(Bl + o1) = make_uint2(l1, l3);
                }
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
        }
    } else {
        // ---------------- MMA issuer (warp 8, lane 0)
        if (lane == 0) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(TC_M, TC_N);
            for (int it = 0; it < nstages; it++) {
                const int buf = it % TC_STAGES;
                if (!tc::mbar_wait(&full[buf], (it / TC_STAGES) & 1, a.status)) {
                    *abort_flag = 1;
                }
                if (*(volatile int*)abort_flag) break;
                tc::tc_fence_after();
                const uint32_t base = tc::smem_u32(smem + buf * TC_STAGE_BYTES);
                const uint32_t ah = base, al = base + TC_A_BYTES;
                const uint32_t bh = base + 2 * TC_A_BYTES, bl = bh + TC_B_BYTES;
#pragma unroll
                for (int ks = 0; ks < TC_K / 16; ks++) {
                    const uint32_t koff = ks * 32;  // 16 bf16 = 32 bytes along K inside the swizzle atom
                    const uint64_t dah = tc::sw128_kmajor_desc(ah + koff), dal = tc::sw128_kmajor_desc(al + koff);
                    const uint64_t dbh = tc::sw128_kmajor_desc(bh + koff), dbl = tc::sw128_kmajor_desc(bl + koff);
                    tc::mma_bf16(tmem, dah, dbh, idesc, (it > 0 || ks > 0) ? 1u : 0u);
                    tc::mma_bf16(tmem, dah, dbl, idesc, 1u);
                    tc::mma_bf16(tmem, dal, dbh, idesc, 1u);
                }
                tc::mma_commit(&empty[buf]);
            }
            tc::mma_commit(done);
        }
        __syncwarp();
    }

    // ---------------- epilogue: warps 0-3 drain TMEM rows 32w..32w+31
    if (warp < 4) {
        const bool waited = tc::mbar_wait(done, 0, a.status);
        tc::tc_fence_after();
        // tcgen05.ld is .sync.aligned: the whole warp takes the same branch
        const bool ok = __all_sync(0xffffffffu, waited && !*(volatile int*)abort_flag);
        if (ok) {
            const int r = r0 + warp * 32 + lane;
            float2* outp = a.out + int64_t(split) * npairs * a.R;
#pragma unroll 1
            for (int q = 0; q < TC_N / 32; q++) {
                float v[32];
                tc::tmem_load32(tmem + (uint32_t(warp * 32) << 16) + uint32_t(q * 32), v);
                if (r < a.R) {
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        const int n = n_pair0 + q * 16 + i;
                        if (n < npairs) {
                            const int c = n / a.S, k = n - c * a.S;
                            outp[(int64_t(c) * a.R + r) * a.S + k] = make_float2(v[2 * i], v[2 * i + 1]);
                        }
                    }
                }
            }
        }
    } else if (warp == 8) {
        // the MMA lane waited for nothing after its last commit: make sure the MMAs finished
        // before the TMEM is released (bounded)
        if (lane == 0) tc::mbar_wait(done, 0, a.status);
        __syncwarp();
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 8) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 256);
    }
}

}  // namespace kernels

namespace {

bool run_tc(const CompasContext& ctx, kernels::TcArgs a, bool jac, cfloat* out) {
    if (!tensor_cores_available(ctx.device())) return false;
    DeviceGuard guard(ctx.device());
    const int npairs = a.C * a.S;
    const int ntiles = div_ceil(npairs, kernels::TC_N / 2), mtiles = div_ceil(a.R, kernels::TC_M);
    const int tiles = ntiles * mtiles;
    const int vps = jac ? 16 : 32;
    // split the voxel range so that the grid fills ~3 waves of 148 SMs, ≥ 8 stages per split
    int splits = std::max(1, (148 * 3 + tiles - 1) / tiles);
    splits = std::min(splits, std::max(1, a.nvoxels / (8 * vps)));
    a.vchunk = div_ceil(div_ceil(a.nvoxels, splits), vps) * vps;
    splits = std::max(1, div_ceil(a.nvoxels, a.vchunk));
    const int64_t n = int64_t(npairs) * a.R;
    Array<cfloat, 2> partials({splits > 1 ? splits : 0, n}, ctx.device());
    a.out = reinterpret_cast<float2*>(splits > 1 ? partials.data() : out);
    a.status = detail::device_status_word(ctx.device());
    auto fn = jac ? kernels::tc_contract_kernel<true> : kernels::tc_contract_kernel<false>;
    static bool attr_set[2] = {false, false};
    if (!attr_set[jac]) {
        COMPAS_CUDA_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, kernels::TC_SMEM));
        attr_set[jac] = true;
    }
    dim3 grid(ntiles, mtiles, splits);
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

bool launch_jacobian_hermitian_tc(const CompasContext&, const float*, int64_t, int, const cfloat*, const cfloat*,
                                  const cfloat*, const cfloat*, int, const cfloat*, const CartesianGeom&, cfloat*) {
    return false;
}

}  // namespace compas
