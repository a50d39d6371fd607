// tc_spiral.cu — split-BF16 tcgen05 kernels for the spiral signal and the spiral J·v.
//
// Spiral signal (reference: src/trajectories/signal_kernels.cuh:274-345, spiral_view.cuh:352-412):
//   s[c][r][k] = Σ_v C[c][v]·A_rv·z_rv^k,  A_rv = ρ_v·m[r][v]·rewind_rv,  z_rv = e^{-Δt R2 + iΘ_rv}.
// For one readout r this is a complex GEMM D_r[k][c] = Σ_v Z_r[k][v]·W_r[v][c] whose operands both
// depend on r: Z_r[k][v] = z_rv^k (generated) and W_r[v][c] = A_rv·C[c][v]. A CTA owns one readout,
// 128 samples (TMEM lanes) and CT ∈ {8, 16} coils (N = 2·CT real columns), and streams the voxels:
//   warps 0-15  generate Z for 128 samples × 32 complex columns per stage (8 consecutive samples per
//               thread: an exact FP64-reduced start, then the complex step z), split FP32 → BF16
//               hi + lo, 128-byte-swizzled K-major; warps 0-3 afterwards drain the TMEM tile;
//   warps 16-17 form W (the readout's source times each coil) for the 32 columns, real-ified as the
//               rows (W_re, -W_im), (W_im, W_re) per coil;
//   warp 18     allocates 32 TMEM columns and one lane issues 3 tcgen05.mma per K16 step
//               (hi·hi + hi·lo + lo·hi, FP32 accumulation).
// J·v on a spiral (no counterpart in the reference) uses two columns per voxel: z^k with source
// readout·P and (k - S/2)·z^k with source readout·Q (P, Q as in the FP32 spiral J·v).
// The SIMT kernel spends 4·C FMAs per (sample, voxel); this one spends ~15 producer instructions
// per (sample, voxel) whatever C is, and the tensor cores do the coil contraction.
#include <cuda_bf16.h>

#include <mutex>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {
namespace kernels {

constexpr int TS_M = 128, TS_K = 64;  // 64 bf16 per row per stage = 32 complex columns
constexpr int TS_STAGES = 4;
constexpr int TS_A_WARPS = 16, TS_B_WARPS = 2;
constexpr int TS_THREADS = (TS_A_WARPS + TS_B_WARPS + 1) * 32;  // 608
constexpr int TS_A_BYTES = TS_M * TS_K * 2;                      // 16 KB per plane

template<int CT>
struct TsLayout {
    static constexpr int N = 2 * CT;
    static constexpr int B_BYTES = N * TS_K * 2;
    static constexpr int STAGE = 2 * TS_A_BYTES + 2 * B_BYTES;
    static constexpr int SMEM = TS_STAGES * STAGE + 1024 + 128;
};

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
    float2* out;  // [C][R][S]
    unsigned int* status;
};

template<bool JAC, int CT>
__global__ void __launch_bounds__(TS_THREADS, 1) tc_spiral_kernel(TsArgs a) {
    using L = TsLayout<CT>;
    constexpr int TERMS = JAC ? 2 : 1;
    constexpr int VPS = 32 / TERMS;  // voxels per stage
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TS_STAGES * L::STAGE);
    uint64_t* empty = full + TS_STAGES;
    uint64_t* done = empty + TS_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k_base = blockIdx.x * TS_M;
    const int r = blockIdx.y;
    const int c0 = blockIdx.z * CT;
    const int nstages = max(1, (a.nvoxels + VPS - 1) / VPS);
    const double twopi = 6.283185307179586476925, inv_2pi = 0.15915494309189533577;
    const float2 ks = a.k_start[r], dkr = a.delta_k[r];

    if (threadIdx.x == 0) {
        for (int s = 0; s < TS_STAGES; s++) {
            tc::mbar_init(&full[s], (TS_A_WARPS + TS_B_WARPS) * 32);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(done, 1);
        *abort_flag = 0;
        tc::fence_mbarrier_init();
    }
    if (warp == TS_A_WARPS + TS_B_WARPS) tc::tmem_alloc(tmem_slot, 32);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < TS_A_WARPS) {
        // ---------------- Z producer: column `col`, samples k_base + 8·kg .. +7
        const int col = threadIdx.x & 31, kg = threadIdx.x >> 5;
        const int term = col % TERMS;
        const int k_first = k_base + kg * 8;
        for (int it = 0; it < nstages; it++) {
            const int buf = it % TS_STAGES;
            const int v = it * VPS + col / TERMS;
            float2 z = make_float2(0.f, 0.f), step = make_float2(0.f, 0.f);
            if (v < a.nvoxels) {
                const float T2 = a.params[a.pstride + v], B0 = a.params[3 * a.pstride + v];
                const float x = a.params[6 * a.pstride + v], y = a.params[7 * a.pstride + v];
                const float dec = -a.dt / T2;
                const double turns = (double(dkr.x) * x + double(dkr.y) * y + double(a.dt) * twopi * B0) * inv_2pi;
                const float2 ph = cis_turns(double(k_first) * turns);
                const float m0 = __expf(float(k_first) * dec);
                z = make_float2(m0 * ph.x, m0 * ph.y);
                step = cscale(__expf(dec), cis_turns(turns));
            }
            if (!tc::mbar_wait(&empty[buf], ((it / TS_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
            if (*(volatile int*)abort_flag) break;
            unsigned char* Ah = smem + buf * L::STAGE;
            unsigned char* Al = Ah + TS_A_BYTES;
            const uint32_t cbyte = uint32_t(col & 3) * 4;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                float2 e = z;
                if constexpr (JAC) {
                    if (term == 1) {
                        const float w = float(k_first + i) - 0.5f * float(a.S);
                        e = make_float2(w * z.x, w * z.y);
                    }
                }
                uint32_t h, l;
                tc::split2(e.x, e.y, h, l);
                const uint32_t off = tc::sw128_offset(kg * 8 + i, col >> 2) + cbyte;
                *reinterpret_cast<uint32_t*>(Ah + off) = h;
                *reinterpret_cast<uint32_t*>(Al + off) = l;
                z = cmul(z, step);
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
        }
    } else if (warp < TS_A_WARPS + TS_B_WARPS) {
        // ---------------- W producer: column `lane`, coils half·CT/2 .. +CT/2
        constexpr int HALF = CT / 2;
        const int half = warp - TS_A_WARPS;
        const int term = lane % TERMS;
        const double hdt = 0.5 * double(a.S) * double(a.dt);
        for (int it = 0; it < nstages; it++) {
            const int buf = it % TS_STAGES;
            const int v = it * VPS + lane / TERMS;
            float2 src = make_float2(0.f, 0.f);
            float2 cv[HALF];
            if (v < a.nvoxels) {
                const float T2 = a.params[a.pstride + v], B0 = a.params[3 * a.pstride + v];
                const float x = a.params[6 * a.pstride + v];
                const float2 rho = make_float2(a.params[4 * a.pstride + v], a.params[5 * a.pstride + v]);
                const float R2 = 1.0f / T2;
                // rewind by (S/2)Δt and prephase with Re k0·x   (spiral_view.cuh:352-398)
                const float2 rw = cis_rad(-hdt * twopi * double(B0) + double(ks.x) * double(x));
                const float2 rd = cscale(expf(float(hdt) * R2), rw);
                const int64_t idx = int64_t(r) * a.nvoxels + v;
                if constexpr (!JAC) {
                    src = cmul(cmul(a.echo[idx], rd), rho);
                } else {
                    const float T1 = a.params[v];
                    const float2 me = a.echo[idx];
                    const float2 w1 = a.vec[a.nvoxels + v];
                    const float2 c2 = cmul(w1, cscale(T2, rho));
                    if (term == 0) {
                        const float2 w0 = a.vec[v];
                        const float2 w2 = a.vec[2 * int64_t(a.nvoxels) + v], w3 = a.vec[3 * int64_t(a.nvoxels) + v];
                        const float2 c1 = cmul(w0, cscale(T1, rho));
                        const float2 cm = make_float2(w2.x - w3.y, w2.y + w3.x);
                        const float2 P = cadd(cadd(cmul(c1, a.dT1[idx]), cmul(c2, a.dT2[idx])), cmul(cm, me));
                        src = cmul(rd, P);
                    } else {
                        src = cmul(rd, cmul(cscale(a.dt * R2 * R2, c2), me));
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < HALF; c++) {
                const int cc = c0 + half * HALF + c;
                cv[c] = (v < a.nvoxels && cc < a.C) ? cmul(a.coils[int64_t(cc) * a.nvoxels + v], src)
                                                     : make_float2(0.f, 0.f);
            }
            if (!tc::mbar_wait(&empty[buf], ((it / TS_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
            if (*(volatile int*)abort_flag) break;
            unsigned char* Bh = smem + buf * L::STAGE + 2 * TS_A_BYTES;
            unsigned char* Bl = Bh + L::B_BYTES;
            const uint32_t cbyte = uint32_t(lane & 3) * 4;
#pragma unroll
            for (int c = 0; c < HALF; c++) {
                const int row = 2 * (half * HALF + c);
                uint32_t h0, l0, h1, l1;
                tc::split2(cv[c].x, -cv[c].y, h0, l0);
                tc::split2(cv[c].y, cv[c].x, h1, l1);
                const uint32_t o0 = tc::sw128_offset(row, lane >> 2) + cbyte;
                const uint32_t o1 = tc::sw128_offset(row + 1, lane >> 2) + cbyte;
                *reinterpret_cast<uint32_t*>(Bh + o0) = h0;
                *reinterpret_cast<uint32_t*>(Bl + o0) = l0;
                *reinterpret_cast<uint32_t*>(Bh + o1) = h1;
                *reinterpret_cast<uint32_t*>(Bl + o1) = l1;
            }
            tc::fence_async_shared();
            tc::mbar_arrive(&full[buf]);
        }
    } else {
        // ---------------- MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(TS_M, L::N);
            for (int it = 0; it < nstages; it++) {
                const int buf = it % TS_STAGES;
                if (!tc::mbar_wait(&full[buf], (it / TS_STAGES) & 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::tc_fence_after();
                const uint32_t base = tc::smem_u32(smem + buf * L::STAGE);
                const uint32_t ah = base, al = base + TS_A_BYTES;
                const uint32_t bh = base + 2 * TS_A_BYTES, bl = bh + L::B_BYTES;
#pragma unroll
                for (int kstep = 0; kstep < TS_K / 16; kstep++) {
                    const uint32_t koff = kstep * 32;
                    const uint64_t dah = tc::sw128_kmajor_desc(ah + koff), dal = tc::sw128_kmajor_desc(al + koff);
                    const uint64_t dbh = tc::sw128_kmajor_desc(bh + koff), dbl = tc::sw128_kmajor_desc(bl + koff);
                    tc::mma_bf16(tmem, dah, dbh, idesc, (it > 0 || kstep > 0) ? 1u : 0u);
                    tc::mma_bf16(tmem, dah, dbl, idesc, 1u);
                    tc::mma_bf16(tmem, dal, dbh, idesc, 1u);
                }
                tc::mma_commit(&empty[buf]);
            }
            tc::mma_commit(done);
        }
        __syncwarp();
    }

    // ---------------- epilogue: warps 0-3 drain TMEM lanes (samples) 32w..32w+31
    if (warp < 4) {
        const bool waited = tc::mbar_wait(done, 0, a.status);
        tc::tc_fence_after();
        const bool ok = __all_sync(0xffffffffu, waited && !*(volatile int*)abort_flag);
        if (ok) {
            float vals[L::N];
            if constexpr (L::N == 16) {
                tc::tmem_load16(tmem + (uint32_t(warp * 32) << 16), vals);
            } else {
                tc::tmem_load32(tmem + (uint32_t(warp * 32) << 16), vals);
            }
            const int k = k_base + warp * 32 + lane;
            if (k < a.S) {
#pragma unroll
                for (int c = 0; c < CT; c++) {
                    if (c0 + c < a.C)
                        a.out[(int64_t(c0 + c) * a.R + r) * a.S + k] = make_float2(vals[2 * c], vals[2 * c + 1]);
                }
            }
        }
    } else if (warp == TS_A_WARPS + TS_B_WARPS) {
        if (lane == 0) tc::mbar_wait(done, 0, a.status);
        __syncwarp();
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == TS_A_WARPS + TS_B_WARPS) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 32);
    }
}

}  // namespace kernels

namespace {

template<bool JAC, int CT>
void run_tc_spiral(const CompasContext& ctx, const kernels::TsArgs& a) {
    using L = kernels::TsLayout<CT>;
    auto fn = kernels::tc_spiral_kernel<JAC, CT>;
    static std::once_flag once;
    std::call_once(once, [&] {
        COMPAS_CUDA_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM));
    });
    dim3 grid(div_ceil(a.S, kernels::TS_M), a.R, div_ceil(a.C, CT));
    fn<<<grid, kernels::TS_THREADS, L::SMEM, ctx.stream()>>>(a);
    check_launch("tc_spiral_kernel");
}

bool launch_tc_spiral(const CompasContext& ctx, kernels::TsArgs a, bool jac) {
    if (!tensor_cores_available(ctx.device())) return false;
    DeviceGuard guard(ctx.device());
    if (int64_t(a.C) * a.R * a.S == 0) return true;
    if (a.nvoxels == 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(a.out, 0, sizeof(float2) * size_t(a.C) * a.R * a.S, ctx.stream()));
        return true;
    }
    a.status = detail::device_status_word(ctx.device());
    if (a.C <= 8) {
        if (jac) run_tc_spiral<true, 8>(ctx, a);
        else run_tc_spiral<false, 8>(ctx, a);
    } else {
        if (jac) run_tc_spiral<true, 16>(ctx, a);
        else run_tc_spiral<false, 16>(ctx, a);
    }
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
