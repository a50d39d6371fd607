// ref_gpu_gemm.cuh — the reference's cuBLAS GEMM calls, restated for the re-hosted products.
//
// TEST INFRASTRUCTURE / BASELINE ONLY. src/utils/gemm.cu:8-82 multiplies `lhs` [m][k] by
// transpose(`rhs` [n][k]) into `result` [m][n] with one cublasGemmEx_64 (op(A) = rhsᵀ, B = lhs,
// FP32 storage; the Fast method computes in TF32), and src/utils/gemm.cu:146-172 forms a planar
// complex product from four of them. The reference reaches cuBLAS through its kmm context; here a
// handle of our own is bound to the caller's stream. Device scratch buffers are cached per name and
// grown on demand (the first call allocates, later calls reuse).
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <map>
#include <string>

namespace ref_gpu {

inline cublasHandle_t blas(cudaStream_t stream) {
    static cublasHandle_t handle = nullptr;
    if (!handle) cublasCreate(&handle);
    cublasSetStream(handle, stream);
    return handle;
}

inline float* scratch(const std::string& name, size_t floats) {
    static std::map<std::string, std::pair<float*, size_t>> buffers;
    auto& b = buffers[name];
    if (b.second < floats) {
        if (b.first) cudaFree(b.first);
        cudaMalloc(&b.first, floats * sizeof(float));
        b.second = floats;
    }
    return b.first;
}

// result [m][n] = alpha · lhs [m][k] · rhs [n][k]ᵀ + beta · result (row-major, contiguous)
inline void gemm(cudaStream_t stream, float* result, const float* lhs, const float* rhs, int64_t m, int64_t n,
                 int64_t k, float alpha, float beta, cublasComputeType_t compute) {
    cublasGemmEx_64(blas(stream), CUBLAS_OP_T, CUBLAS_OP_N, n, m, k, &alpha, rhs, CUDA_R_32F, k, lhs, CUDA_R_32F, k,
                    &beta, result, CUDA_R_32F, n, compute, CUBLAS_GEMM_DEFAULT);
}

// planar complex [2][m][n] = lhs [2][m][k] · rhs [2][n][k]ᵀ (alpha, beta real)
inline void complex_gemm(cudaStream_t stream, float* result, const float* lhs, const float* rhs, int64_t m,
                         int64_t n, int64_t k, float alpha, float beta, cublasComputeType_t compute) {
    float* re = result;
    float* im = result + m * n;
    const float *lre = lhs, *lim = lhs + m * k, *rre = rhs, *rim = rhs + n * k;
    gemm(stream, re, lre, rre, m, n, k, alpha, beta, compute);
    gemm(stream, re, lim, rim, m, n, k, -alpha, 1.0f, compute);
    gemm(stream, im, lre, rim, m, n, k, alpha, beta, compute);
    gemm(stream, im, lim, rre, m, n, k, alpha, 1.0f, compute);
}

}  // namespace ref_gpu
