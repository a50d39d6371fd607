// job_args.cuh — argument blocks of the simulation and signal kernels.
//
// One block describes one operation (a simulation, a signal or J·v contraction) on one set of
// device arrays. The one-operation kernels take it as a kernel parameter; the batched work-queue
// kernels (batch.cu) take an array of them, one per job, in device memory.
#pragma once

#include <cstdint>

#include <vector_types.h>

namespace compas {
namespace kernels {

struct FispArgs {
    const float* params;   // [9][param_stride]
    int64_t param_stride;
    int voxel_begin;       // first voxel of this launch
    int nvoxels;           // voxels in this launch
    const float4* table;   // [P][nTR]
    int nTR, P, N, uf, reps, inversion, wait_spoil;
    float TR, TE, TW, TI;
    float2* echo;          // [nTR*uf][echo_stride], column = voxel_begin + local voxel
    int64_t echo_stride;
    float2* dT1;           // ∂echo/∂T1, ∂echo/∂T2 (same layout); used by the tangent kernels only
    float2* dT2;
    const int* skip;       // one-simulation kernel: returns at once when *skip != 0 (null: never)
};

// Voxel tiles per item of the FISP work-queue kernels, for a job of P slice positions on CTAs of W
// warps: an item's (tile, position) pairs run in rounds of W warps, and one tile of 35 positions on
// 8 warps leaves the last of 5 rounds with 3 warps busy (35 of 40 warp slots), two tiles fill 70 of
// 72. The count up to 4 with the fullest rounds, the fewest on ties. The batch builds its items and
// the kernel reads them with this same count; the summation order, and so every bit, does not
// depend on it.
__host__ __device__ inline int fisp_queue_tiles_per_item(int P, int W) {
    int best = 1, best_pairs = P, best_slots = ((P + W - 1) / W) * W;
    for (int n = 2; n <= 4; n++) {
        const int pairs = n * P, slots = ((pairs + W - 1) / W) * W;
        if (int64_t(pairs) * best_slots > int64_t(best_pairs) * slots) {
            best = n;
            best_pairs = pairs;
            best_slots = slots;
        }
    }
    return best;
}

struct PssfpArgs {
    const float* params;
    int64_t param_stride;
    int voxel_begin, nvoxels;
    const float2* zap;  // [nTR+1][nRF]
    const float* z;     // [nz]
    int nTR, nRF, nz;
    float dt_ex, dt_inv, dt_pr, gz_ex, gz_pr;
    float2* echo;  // [nTR][echo_stride]
    int64_t echo_stride;
    float2* dT1;   // ∂echo/∂T1, ∂echo/∂T2 (same layout); used by the tangent kernels only
    float2* dT2;
    const int* skip;  // one-simulation kernel: returns at once when *skip != 0 (null: never)
};

struct SpiralArgs {
    const float* params;
    int64_t pstride;
    int nvoxels;
    const float2* echo;
    const float2* coils;
    int R, S, C;
    float dt;
    const float2* k_start;
    const float2* delta_k;
    float2* signal;  // [C][R][S]
    // J·v only (the spiral kernel's JAC form): derivative echoes and the direction [4][V]
    const float2* dT1;
    const float2* dT2;
    const float2* vec;
};

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
    // tables written by the prep kernel:
    const float2* vstep;   // [V] e^{-Δt/T2 + iΘ_v}, the per-sample step of E_k
    const float2* estart;  // [S / egk][V] E_k exactly (FP64-reduced phase) at k = 0, egk, 2·egk, …
    int egk;               // restart granularity: TC_PPG when it divides S, else 1
    const float2* coilw;   // [C][V] coil·w
    const float4* jcoef;   // J·v only: [V][2] {T1ρv0, T2ρv1}, {v2 + i v3, ΔtR2²·T2ρv1}
    // A operand split and laid out as shared-memory stage images (tc_pack_a): block (readout
    // tile, voxel stage) = hi then lo plane, 16 KB each
    const unsigned char* apack;
    int apack_stages;      // voxel stages per readout tile in apack
    int nr;                // readouts per tile (a multiple of 16, ≤ 256; each CTA of a pair holds nr/2)
};

// one split-K reduction: out[i] = Σ_q partials[q·n + i], q = 0..nsplit-1 in order
struct PartialSum {
    const float2* partials;
    float2* out;
    int64_t n;
    int nsplit;
};

}  // namespace kernels
}  // namespace compas
