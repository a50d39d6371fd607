// tc_gemm.cu — the GEMM utility API: compute_gemm, compute_complex_gemm, convert_complex_to_planar,
// convert_planar_to_complex (include/compas/utils/gemm.h:7-70, src/utils/gemm.cu:8-254).
//
// result = α·lhs·rhsᵀ + β·result with lhs [m][k], rhs [n][k], result [m][n] (row-major; the complex
// forms take planar [2][rows][cols] arrays: plane 0 real, plane 1 imaginary). The reference calls
// cuBLAS, four real GEMMs per complex product. Here:
//  * GemmComputeMethod::Fast, FP32 inputs: split-BF16 on tcgen05 tensor cores. Every operand
//    x = hi + lo (two BF16) and hi·hi + hi·lo + lo·hi accumulate in FP32 TMEM, ~1e-5 relative
//    error — at least as accurate as the reference's TF32 "Fast". The complex product is one real
//    GEMM on real-ified operands: A' = (Re a, Im a) interleaved along K and, per output column j,
//    the rows (Re b, -Im b) and (Im b, Re b) of B', so that the columns of A'·B'ᵀ alternate Re c
//    and Im c (the same construction as the signal kernels).
//  * Regular and Pedantic, FP32 inputs: a plain FP32 kernel on the CUDA cores (FFMA, FP32
//    accumulation), the arithmetic of the reference's CUBLAS_COMPUTE_32F(_PEDANTIC).
//  * BF16 inputs (any method): the inputs are exact in BF16, so one BF16 MMA per product with FP32
//    accumulation is exact up to the accumulation.
// Tensor-core accumulation: the FP32 accumulate of the tensor cores loses a little per MMA and the
// loss grows with the number of K16 steps summed in one accumulator, so two TMEM accumulators
// alternate every 64 K16 steps (K = 1024) and the epilogue warps add each finished one into FP32
// registers (K = 50176: 1e-5 instead of 2e-4).
#include <cuda_bf16.h>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {
namespace kernels {

constexpr int TG_M = 128, TG_N = 128, TG_K = 64;  // tile rows, columns, BF16 elements of K per stage
constexpr int TG_PLANE = TG_M * TG_K * 2;         // 16 KB: one BF16 plane of a 128-row stage tile
constexpr int TG_STAGES = 3;
constexpr int TG_CHUNK = 16;                      // stages (64 K16 steps) per accumulator
constexpr int TG_THREADS = 192;                   // copy warp, MMA warp, 4 epilogue warps
constexpr int TG_COPY_WARP = 0, TG_MMA_WARP = 1;
constexpr int TG_PITCH = TG_N + 1;                // epilogue staging tile pitch (floats)

// Logical real operand: element (row, kk) of a [rows][kp] matrix built from the caller's arrays.
//  kind 0: real [rows][k], kind 1: A' of a planar complex [2][rows][k] (kk even Re, odd Im),
//  kind 2: B' of a planar complex [2][n][k] (row 2j: (Re, -Im), row 2j+1: (Im, Re)).
template<typename T>
struct GemmOperand {
    const T* data;
    int64_t rows, k;  // the caller's array: [rows][k] per plane (rows = n for kind 2)
    int kind;
};

__device__ __forceinline__ float as_float(float x) {
    return x;
}
__device__ __forceinline__ float as_float(__nv_bfloat16 x) {
    return __bfloat162float(x);
}

template<typename T>
__device__ __forceinline__ float operand_at(const GemmOperand<T>& o, int64_t row, int64_t kk) {
    if (o.kind == 0) return (row < o.rows && kk < o.k) ? as_float(o.data[row * o.k + kk]) : 0.0f;
    const int64_t k = kk >> 1, part = kk & 1;
    if (k >= o.k) return 0.0f;
    if (o.kind == 1) return row < o.rows ? as_float(o.data[(part * o.rows + row) * o.k + k]) : 0.0f;
    const int64_t j = row >> 1, rp = row & 1;
    if (j >= o.rows) return 0.0f;
    const float re = as_float(o.data[j * o.k + k]), im = as_float(o.data[(o.rows + j) * o.k + k]);
    return rp == 0 ? (part == 0 ? re : -im) : (part == 0 ? im : re);
}

// The operand as the shared-memory images of every (128-row tile, 64-wide K stage): `planes` BF16
// planes (hi, and lo = x - hi when planes == 2), 128-byte swizzled K-major. One thread writes one
// 16-byte chunk (8 elements) of one row of one plane pair. grid = (chunks / 128, stages, tiles).
template<typename T>
__global__ void __launch_bounds__(128) tc_gemm_pack_kernel(GemmOperand<T> o, int planes, int kstages,
                                                           unsigned char* __restrict__ images) {
    const int tile = blockIdx.z, stage = blockIdx.y;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // (row, chunk) of the tile
    const int r = idx >> 3, c = idx & 7;
    const int64_t row = int64_t(tile) * TG_M + r;
    const int64_t kk0 = int64_t(stage) * TG_K + c * 8;
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float a = operand_at(o, row, kk0 + 2 * i), b = operand_at(o, row, kk0 + 2 * i + 1);
        tc::split2(a, b, h[i], l[i]);
    }
    unsigned char* blk = images + (int64_t(tile) * kstages + stage) * int64_t(planes) * TG_PLANE;
    const uint32_t off = tc::sw128_offset(r, c);
    *reinterpret_cast<uint4*>(blk + off) = make_uint4(h[0], h[1], h[2], h[3]);
    if (planes == 2) *reinterpret_cast<uint4*>(blk + TG_PLANE + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

struct TgArgs {
    const unsigned char* aimg;  // [tiles_m][kstages][planes][128][64] bf16
    const unsigned char* bimg;  // [tiles_n][kstages][planes][128][64] bf16
    int kstages;
    int64_t M, N;  // real-ified result rows / columns
    float* out;    // real: [M][N]; complex: planar [2][M][N/2]
    int complex_out;
    float alpha, beta;
    unsigned int* status;
};

// One 128 x 128 tile of the real-ified result per CTA. TERMS 3: split-BF16 (hi·hi + hi·lo +
// lo·hi), 1: BF16 inputs.
template<int TERMS>
__global__ void __launch_bounds__(TG_THREADS, 1) tc_gemm_kernel(TgArgs a) {
    constexpr int PLANES = TERMS == 3 ? 2 : 1;
    constexpr int STAGE = 2 * PLANES * TG_PLANE;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TG_STAGES * STAGE);
    uint64_t* empty = full + TG_STAGES;
    uint64_t* acc_full = empty + TG_STAGES;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tm = blockIdx.x, tn = blockIdx.y;
    const int nst = a.kstages;
    const int nchunks = (nst + TG_CHUNK - 1) / TG_CHUNK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TG_STAGES; s++) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < 2; s++) {
            tc::mbar_init(&acc_full[s], 1);
            tc::mbar_init(&acc_empty[s], 4);  // one arrival per epilogue warp
        }
        tc::mbar_init(done, 1);
        *abort_flag = 0;
        tc::fence_mbarrier_init();
    }
    if (warp == TG_MMA_WARP) tc::tmem_alloc(tmem_slot, 2 * TG_N);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == TG_COPY_WARP) {
        // ---------------- stage images: A and B of this tile, one bulk copy each (no multicast)
        if (lane == 0) {
            const unsigned char* asrc = a.aimg + int64_t(tm) * nst * PLANES * TG_PLANE;
            const unsigned char* bsrc = a.bimg + int64_t(tn) * nst * PLANES * TG_PLANE;
            int issued[TG_STAGES];
            for (int s = 0; s < TG_STAGES; s++) issued[s] = -1;
            for (int g = 0; g < nst; g++) {
                const int buf = g % TG_STAGES;
                if (!tc::mbar_wait(&empty[buf], ((g / TG_STAGES) & 1) ^ 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::mbar_arrive_expect_tx(&full[buf], STAGE);
                unsigned char* dst = smem + buf * STAGE;
                tc::bulk_copy_g2s(dst, asrc + int64_t(g) * PLANES * TG_PLANE, PLANES * TG_PLANE, &full[buf]);
                tc::bulk_copy_g2s(dst + PLANES * TG_PLANE, bsrc + int64_t(g) * PLANES * TG_PLANE, PLANES * TG_PLANE,
                                  &full[buf]);
                issued[buf] = g;
            }
            // copies still in flight land before the CTA can finish (bounded)
            for (int s = 0; s < TG_STAGES; s++)
                if (issued[s] >= 0) tc::mbar_wait(&full[s], (issued[s] / TG_STAGES) & 1, a.status);
        }
    } else if (warp == TG_MMA_WARP) {
        // ---------------- MMA issuer: accumulator (chunk & 1), 16 stages per chunk
        if (lane == 0) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(TG_M, TG_N);
            for (int g = 0; g < nst && !*(volatile int*)abort_flag; g++) {
                const int chunk = g / TG_CHUNK, acc = chunk & 1;
                if (g % TG_CHUNK == 0 && chunk >= 2 &&
                    !tc::mbar_wait(&acc_empty[acc], ((chunk >> 1) - 1) & 1, a.status)) {
                    *abort_flag = 1;
                    break;
                }
                const int buf = g % TG_STAGES;
                if (!tc::mbar_wait(&full[buf], (g / TG_STAGES) & 1, a.status)) *abort_flag = 1;
                if (*(volatile int*)abort_flag) break;
                tc::tc_fence_after();
                const uint32_t base = tc::smem_u32(smem + buf * STAGE);
                const uint32_t ah = base, al = base + TG_PLANE;
                const uint32_t bh = base + PLANES * TG_PLANE, bl = bh + TG_PLANE;
                const uint32_t d = tmem + uint32_t(acc * TG_N);
#pragma unroll
                for (int k16 = 0; k16 < TG_K / 16; k16++) {
                    const uint32_t koff = k16 * 32;
                    const uint32_t first = (g % TG_CHUNK > 0 || k16 > 0) ? 1u : 0u;
                    tc::mma_bf16(d, tc::sw128_kmajor_desc(ah + koff), tc::sw128_kmajor_desc(bh + koff), idesc, first);
                    if constexpr (TERMS == 3) {
                        tc::mma_bf16(d, tc::sw128_kmajor_desc(ah + koff), tc::sw128_kmajor_desc(bl + koff), idesc, 1u);
                        tc::mma_bf16(d, tc::sw128_kmajor_desc(al + koff), tc::sw128_kmajor_desc(bh + koff), idesc, 1u);
                    }
                }
                tc::mma_commit(&empty[buf]);
                if (g % TG_CHUNK == TG_CHUNK - 1 || g == nst - 1) tc::mma_commit(&acc_full[acc]);
            }
            tc::mma_commit(done);
            tc::mbar_wait(done, 0, a.status);  // every MMA has completed before the TMEM is released
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: thread = row (TMEM lane) of this tile; sums the chunks in FP32
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane;
        float sum[TG_N];
#pragma unroll
        for (int i = 0; i < TG_N; i++) sum[i] = 0.0f;
        bool ok = true;
        for (int chunk = 0; chunk < nchunks; chunk++) {
            const int acc = chunk & 1;
            ok = ok && tc::mbar_wait(&acc_full[acc], (chunk >> 1) & 1, a.status) && !*(volatile int*)abort_flag;
            ok = !tc::bar_red_or(1, 128, !ok);
            if (!ok) break;
            tc::tc_fence_after();
#pragma unroll
            for (int q = 0; q < TG_N / 32; q++) {
                float v[32];
                tc::tmem_load32(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(acc * TG_N + 32 * q), v);
#pragma unroll
                for (int i = 0; i < 32; i++) sum[32 * q + i] += v[i];
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&acc_empty[acc]);
        }
        if (ok) {
            // stage the tile through shared memory (the pipeline buffers are free once the last
            // chunk is complete) and write it row by row, coalesced
            float* tile = reinterpret_cast<float*>(smem);
#pragma unroll
            for (int i = 0; i < TG_N; i++) tile[row * TG_PITCH + i] = sum[i];
            tc::bar_sync(1, 128);
            const int t = threadIdx.x - 64;
            const int64_t row0 = int64_t(tm) * TG_M, col0 = int64_t(tn) * TG_N;
            if (!a.complex_out) {
                for (int e = t; e < TG_M * TG_N; e += 128) {
                    const int r = e / TG_N, c = e % TG_N;
                    const int64_t gr = row0 + r, gc = col0 + c;
                    if (gr >= a.M || gc >= a.N) continue;
                    float* dst = a.out + gr * a.N + gc;
                    const float v = a.alpha * tile[r * TG_PITCH + c];
                    *dst = a.beta == 0.0f ? v : fmaf(a.beta, *dst, v);
                }
            } else {
                const int64_t nc = a.N / 2;  // complex columns of the result
                for (int e = t; e < TG_M * (TG_N / 2); e += 128) {
                    const int r = e / (TG_N / 2), j = e % (TG_N / 2);
                    const int64_t gr = row0 + r, gj = col0 / 2 + j;
                    if (gr >= a.M || gj >= nc) continue;
                    float* re = a.out + gr * nc + gj;
                    float* im = re + a.M * nc;
                    const float vr = a.alpha * tile[r * TG_PITCH + 2 * j];
                    const float vi = a.alpha * tile[r * TG_PITCH + 2 * j + 1];
                    *re = a.beta == 0.0f ? vr : fmaf(a.beta, *re, vr);
                    *im = a.beta == 0.0f ? vi : fmaf(a.beta, *im, vi);
                }
            }
        }
    }
    // the MMA lane waited on `done` for every MMA it issued, so the TMEM is free to release
    tc::tc_fence_before();
    __syncthreads();
    if (warp == TG_MMA_WARP) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 2 * TG_N);
    }
}

// FP32 result = α·A·Bᵀ + β·C on the CUDA cores (real, or planar complex): 64 x 64 output tiles,
// 16-wide K slices staged in shared memory, 4 x 4 outputs per thread.
template<bool COMPLEX>
__global__ void __launch_bounds__(256) sgemm_nt_kernel(const float* __restrict__ A, const float* __restrict__ B,
                                                       float* __restrict__ C, int64_t m, int64_t n, int64_t k,
                                                       float alpha, float beta) {
    constexpr int T = 64, KS = 16, P = COMPLEX ? 2 : 1;
    __shared__ float As[P][KS][T + 4], Bs[P][KS][T + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int64_t i0 = int64_t(blockIdx.y) * T, j0 = int64_t(blockIdx.x) * T;
    float acc[P][4][4] = {};
    for (int64_t k0 = 0; k0 < k; k0 += KS) {
        for (int e = threadIdx.x; e < T * KS; e += 256) {
            const int r = e / KS, kk = e % KS;
#pragma unroll
            for (int p = 0; p < P; p++) {
                const int64_t ia = i0 + r, jb = j0 + r, kg = k0 + kk;
                As[p][kk][r] = (ia < m && kg < k) ? A[(p * m + ia) * k + kg] : 0.0f;
                Bs[p][kk][r] = (jb < n && kg < k) ? B[(p * n + jb) * k + kg] : 0.0f;
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KS; kk++) {
            float a[P][4], b[P][4];
#pragma unroll
            for (int p = 0; p < P; p++)
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    a[p][u] = As[p][kk][ty * 4 + u];
                    b[p][u] = Bs[p][kk][tx * 4 + u];
                }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    if constexpr (COMPLEX) {
                        acc[0][u][w] = fmaf(a[0][u], b[0][w], fmaf(-a[1][u], b[1][w], acc[0][u][w]));
                        acc[1][u][w] = fmaf(a[0][u], b[1][w], fmaf(a[1][u], b[0][w], acc[1][u][w]));
                    } else {
                        acc[0][u][w] = fmaf(a[0][u], b[0][w], acc[0][u][w]);
                    }
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int w = 0; w < 4; w++) {
                const int64_t i = i0 + ty * 4 + u, j = j0 + tx * 4 + w;
                if (i >= m || j >= n) continue;
                float* dst = C + (p * m + i) * n + j;
                const float v = alpha * acc[p][u][w];
                *dst = beta == 0.0f ? v : fmaf(beta, *dst, v);
            }
}

// result = β·result (k = 0), or zero when β = 0
__global__ void gemm_scale_kernel(float* __restrict__ c, int64_t n, float beta) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        c[i] = beta == 0.0f ? 0.0f : beta * c[i];
}

template<typename T>
__global__ void complex_to_planar_kernel(const float2* __restrict__ in, T* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float2 v = in[i];
        if constexpr (std::is_same_v<T, float>) {
            out[i] = v.x;
            out[n + i] = v.y;
        } else {
            out[i] = __float2bfloat16_rn(v.x);
            out[n + i] = __float2bfloat16_rn(v.y);
        }
    }
}

__global__ void planar_to_complex_kernel(const float* __restrict__ in, float2* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = make_float2(in[i], in[n + i]);
}

}  // namespace kernels

namespace {

int grid_for(int64_t n) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)));
}

// result (real [M][N], or planar complex [2][m][n]) of the tensor-core path
template<typename T>
void tc_gemm(const CompasContext& ctx, float* out, int64_t M, int64_t Nr, int64_t Kr, bool complex_out,
             kernels::GemmOperand<T> A, kernels::GemmOperand<T> B, float alpha, float beta, int terms) {
    const int planes = terms == 3 ? 2 : 1;
    const int64_t tiles_m = (M + kernels::TG_M - 1) / kernels::TG_M;
    const int64_t tiles_n = (Nr + kernels::TG_N - 1) / kernels::TG_N;
    const int64_t kstages = (Kr + kernels::TG_K - 1) / kernels::TG_K;
    if (tiles_m > 65535 || tiles_n > 65535 || kstages > 65535) COMPAS_ERROR("GEMM too large (65535 tiles per axis)");
    const int64_t tile_bytes = kstages * planes * kernels::TG_PLANE;
    Array<unsigned char> aimg({tiles_m * tile_bytes}, ctx.device(), ctx.stream());
    Array<unsigned char> bimg({tiles_n * tile_bytes}, ctx.device(), ctx.stream());
    const dim3 pb(kernels::TG_M * 8 / 128, unsigned(kstages));
    kernels::tc_gemm_pack_kernel<T><<<dim3(pb.x, pb.y, unsigned(tiles_m)), 128, 0, ctx.stream()>>>(
        A, planes, int(kstages), aimg.data());
    check_launch("tc_gemm_pack_kernel (A)");
    kernels::tc_gemm_pack_kernel<T><<<dim3(pb.x, pb.y, unsigned(tiles_n)), 128, 0, ctx.stream()>>>(
        B, planes, int(kstages), bimg.data());
    check_launch("tc_gemm_pack_kernel (B)");
    kernels::TgArgs a {};
    a.aimg = aimg.data();
    a.bimg = bimg.data();
    a.kstages = int(kstages);
    a.M = M;
    a.N = Nr;
    a.out = out;
    a.complex_out = complex_out ? 1 : 0;
    a.alpha = alpha;
    a.beta = beta;
    a.status = ctx.status_word();
    const int stage = 2 * planes * kernels::TG_PLANE;
    const size_t smem = size_t(kernels::TG_STAGES) * stage + 1024 + 256;
    static_assert(kernels::TG_M * kernels::TG_PITCH * 4 <= kernels::TG_STAGES * 2 * kernels::TG_PLANE,
                  "the epilogue's staging tile fits in the pipeline buffers");
    auto fn = terms == 3 ? kernels::tc_gemm_kernel<3> : kernels::tc_gemm_kernel<1>;
    COMPAS_CUDA_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    fn<<<dim3(unsigned(tiles_m), unsigned(tiles_n)), kernels::TG_THREADS, smem, ctx.stream()>>>(a);
    check_launch("tc_gemm_kernel");
}

template<typename T, size_t R>
void check_gemm_shapes(const Array<float, R>& result, const Array<T, R>& lhs, const Array<T, R>& rhs) {
    constexpr int o = R == 3 ? 1 : 0;  // leading plane axis of the complex forms
    if (R == 3) COMPAS_CHECK(result.size(0) == 2 && lhs.size(0) == 2 && rhs.size(0) == 2);
    COMPAS_CHECK(lhs.size(o) == result.size(o));
    COMPAS_CHECK(rhs.size(o) == result.size(o + 1));
    COMPAS_CHECK(lhs.size(o + 1) == rhs.size(o + 1));
    COMPAS_CHECK(lhs.device() == result.device() && rhs.device() == result.device());
}

}  // namespace

void compute_gemm(const CompasContext& ctx, Array<float, 2>& result, const Array<float, 2>& lhs,
                  const Array<float, 2>& rhs, float alpha, float beta, GemmComputeMethod kind) {
    check_gemm_shapes(result, lhs, rhs);
    const int64_t m = result.size(0), n = result.size(1), k = lhs.size(1);
    if (m * n == 0) return;
    DeviceGuard guard(ctx.device());
    if (k == 0) {
        kernels::gemm_scale_kernel<<<grid_for(m * n), 256, 0, ctx.stream()>>>(result.data(), m * n, beta);
        check_launch("gemm_scale_kernel");
    } else if (kind == GemmComputeMethod::Fast && tensor_cores_available(ctx.device())) {
        tc_gemm<float>(ctx, result.data(), m, n, k, false, {lhs.data(), m, k, 0}, {rhs.data(), n, k, 0}, alpha, beta, 3);
    } else {
        kernels::sgemm_nt_kernel<false><<<dim3(unsigned((n + 63) / 64), unsigned((m + 63) / 64)), 256, 0, ctx.stream()>>>(
            lhs.data(), rhs.data(), result.data(), m, n, k, alpha, beta);
        check_launch("sgemm_nt_kernel");
    }
}

void compute_gemm(const CompasContext& ctx, Array<float, 2>& result, const Array<bfloat16, 2>& lhs,
                  const Array<bfloat16, 2>& rhs, float alpha, float beta, GemmComputeMethod) {
    check_gemm_shapes(result, lhs, rhs);
    const int64_t m = result.size(0), n = result.size(1), k = lhs.size(1);
    if (m * n == 0) return;
    DeviceGuard guard(ctx.device());
    if (k == 0) {
        kernels::gemm_scale_kernel<<<grid_for(m * n), 256, 0, ctx.stream()>>>(result.data(), m * n, beta);
        check_launch("gemm_scale_kernel");
        return;
    }
    if (!tensor_cores_available(ctx.device())) COMPAS_ERROR("BF16 GEMM needs the sm_100 tensor cores");
    tc_gemm<bfloat16>(ctx, result.data(), m, n, k, false, {lhs.data(), m, k, 0}, {rhs.data(), n, k, 0}, alpha, beta,
                      1);
}

void compute_complex_gemm(const CompasContext& ctx, Array<float, 3>& result, const Array<float, 3>& lhs,
                          const Array<float, 3>& rhs, float alpha, float beta, GemmComputeMethod kind) {
    check_gemm_shapes(result, lhs, rhs);
    const int64_t m = result.size(1), n = result.size(2), k = lhs.size(2);
    if (m * n == 0) return;
    DeviceGuard guard(ctx.device());
    if (k == 0) {
        kernels::gemm_scale_kernel<<<grid_for(2 * m * n), 256, 0, ctx.stream()>>>(result.data(), 2 * m * n, beta);
        check_launch("gemm_scale_kernel");
    } else if (kind == GemmComputeMethod::Fast && tensor_cores_available(ctx.device())) {
        tc_gemm<float>(ctx, result.data(), m, 2 * n, 2 * k, true, {lhs.data(), m, k, 1}, {rhs.data(), n, k, 2}, alpha,
                       beta, 3);
    } else {
        kernels::sgemm_nt_kernel<true><<<dim3(unsigned((n + 63) / 64), unsigned((m + 63) / 64)), 256, 0, ctx.stream()>>>(
            lhs.data(), rhs.data(), result.data(), m, n, k, alpha, beta);
        check_launch("sgemm_nt_kernel");
    }
}

void compute_complex_gemm(const CompasContext& ctx, Array<float, 3>& result, const Array<bfloat16, 3>& lhs,
                          const Array<bfloat16, 3>& rhs, float alpha, float beta, GemmComputeMethod) {
    check_gemm_shapes(result, lhs, rhs);
    const int64_t m = result.size(1), n = result.size(2), k = lhs.size(2);
    if (m * n == 0) return;
    DeviceGuard guard(ctx.device());
    if (k == 0) {
        kernels::gemm_scale_kernel<<<grid_for(2 * m * n), 256, 0, ctx.stream()>>>(result.data(), 2 * m * n, beta);
        check_launch("gemm_scale_kernel");
        return;
    }
    if (!tensor_cores_available(ctx.device())) COMPAS_ERROR("BF16 GEMM needs the sm_100 tensor cores");
    tc_gemm<bfloat16>(ctx, result.data(), m, 2 * n, 2 * k, true, {lhs.data(), m, k, 1}, {rhs.data(), n, k, 2}, alpha,
                      beta, 1);
}

template<typename T>
static void complex_to_planar(const CompasContext& ctx, Array<T, 3>& output, const Array<cfloat, 2>& input) {
    COMPAS_CHECK(output.size(0) == 2 && output.size(1) == input.size(0) && output.size(2) == input.size(1));
    const int64_t n = input.numel();
    if (n == 0) return;
    DeviceGuard guard(ctx.device());
    kernels::complex_to_planar_kernel<T><<<grid_for(n), 256, 0, ctx.stream()>>>(
        reinterpret_cast<const float2*>(input.data()), output.data(), n);
    check_launch("complex_to_planar_kernel");
}

void convert_complex_to_planar(const CompasContext& ctx, Array<float, 3>& output, const Array<cfloat, 2>& input) {
    complex_to_planar(ctx, output, input);
}

void convert_complex_to_planar(const CompasContext& ctx, Array<bfloat16, 3>& output, const Array<cfloat, 2>& input) {
    complex_to_planar(ctx, output, input);
}

void convert_planar_to_complex(const CompasContext& ctx, Array<cfloat, 2>& output, const Array<float, 3>& input) {
    COMPAS_CHECK(input.size(0) == 2 && input.size(1) == output.size(0) && input.size(2) == output.size(1));
    const int64_t n = output.numel();
    if (n == 0) return;
    DeviceGuard guard(ctx.device());
    kernels::planar_to_complex_kernel<<<grid_for(n), 256, 0, ctx.stream()>>>(input.data(),
                                                                            reinterpret_cast<float2*>(output.data()), n);
    check_launch("planar_to_complex_kernel");
}

}  // namespace compas
