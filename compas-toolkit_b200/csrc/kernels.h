// kernels.h — internal launch interfaces between the host operations, the batch /
// graph / serving layers and the autotuner. Not part of the public API.
#pragma once

#include <cstdint>

#include "compas/compas.h"
#include "job_args.cuh"

namespace compas {

// ---- FISP EPG -------------------------------------------------------------------------
struct FispLaunch {
    int config;  // index into the instantiated (K, G) layouts, -1 = default choice
    int warps;   // warps per CTA (slice positions in flight per voxel tile)
};
int fisp_config_count();
bool fisp_config_info(int index, int* K, int* G);
bool fisp_config_packed(int index);  // EPGPacked layout (two states per FFMA2)
FispLaunch fisp_default_launch(int N, int64_t nvoxels, int P);
FispLaunch tuned_fisp_launch(int N, int64_t nvoxels, int P);
const Array<float, 3>& fisp_excite_table(const CompasContext& ctx, const FISPSequence& seq);
// whether every RF and slice-profile phase of the sequence is real (sin φ = 0), read back from its
// excitation table: synchronises the context's stream the first time (not while it is captured)
bool fisp_sequence_real_phases(const CompasContext& ctx, const FISPSequence& seq);
// simulates voxels [voxel_begin, voxel_begin + nvoxels) of `params` into echo columns
// voxel_begin.. of a [nTR*uf][echo_stride] complex array
// `skip` (device int, may be null): when it holds a nonzero value at run time the kernel returns
// without writing (a step of a captured graph that is not needed this time)
// `balance`: split the (tile, position) items evenly over the CTAs, neighbours handing over the
// partial sums of the tile they share (the echoes are the same bits either way); its per-CTA flags
// live in `handoff` (`handoff_capacity` ints, owned by the caller, zeroed here on the stream) or,
// without, in a small stream-ordered allocation per call. Off: whole tiles per CTA.
void launch_fisp(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                 const FISPSequence& seq, cfloat* echo, int64_t echo_stride, FispLaunch L,
                 const int* skip = nullptr, bool balance = false, int* handoff = nullptr, int handoff_capacity = 0);
// argument block of one FISP simulation (validates the sequence, builds its table on first use)
kernels::FispArgs fisp_args(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                            const FISPSequence& seq, cfloat* echo, int64_t echo_stride);
int fisp_tile_voxels(FispLaunch L);  // voxels per work item (tile) of layout L
// persistent work-queue launch over (job, tile) items of FISP jobs that all use layout L;
// *head must be 0 when the kernel starts. `real`: every job's phases are real
// (fisp_sequence_real_phases), which a packed layout runs in its real-phase form.
void launch_fisp_queue(cudaStream_t stream, int device, FispLaunch L, int max_state, const kernels::FispArgs* jobs,
                       const int2* items, int nitems, int* head, bool real = false);

// value and T1/T2 tangents (forward mode) in one launch; L.config indexes the tangent layouts
int fisp_tangent_config_count();
bool fisp_tangent_config_info(int index, int* K, int* G);
bool fisp_tangent_config_packed(int index);  // EPGPackedTangent layout
FispLaunch fisp_tangent_default_launch(int N, int64_t nvoxels, int P);
FispLaunch tuned_fisp_tangent_launch(int N, int64_t nvoxels, int P);  // honours the test override
void launch_fisp_tangent(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                         const FISPSequence& seq, cfloat* echo, cfloat* dT1, cfloat* dT2, int64_t echo_stride,
                         FispLaunch L);
int fisp_tangent_tile_voxels(FispLaunch L);  // voxels per work item of tangent layout L
// work-queue launch over (job, tile) items of FISP tangent jobs (args with dT1 / dT2 set), every
// job with max_state states; `real`: every job's phases are real, which a packed layout runs in its
// real-phase form
void launch_fisp_tangent_queue(cudaStream_t stream, int device, FispLaunch L, int max_state,
                               const kernels::FispArgs* jobs, const int2* items, int nitems, int* head,
                               bool real = false);

// ---- pSSFP ------------------------------------------------------------------------------
struct PssfpLaunch {
    int config;  // index into the instantiated (ZT, GZ) layouts, -1 = default
};
int pssfp_config_count();
bool pssfp_config_info(int index, int* ZT, int* GZ);
bool pssfp_config_packed(int index);  // two-wide layout: ZT/2 pairs of isochromats per lane
PssfpLaunch pssfp_default_launch(int nz, int64_t nvoxels);
PssfpLaunch tuned_pssfp_launch(int nz, int64_t nvoxels);
void launch_pssfp(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                  const pSSFPSequence& seq, cfloat* echo, int64_t echo_stride, PssfpLaunch L,
                  const int* skip = nullptr);
kernels::PssfpArgs pssfp_args(const CompasContext& ctx, const TissueParameters& params, int voxel_begin,
                              int nvoxels, const pSSFPSequence& seq, cfloat* echo, int64_t echo_stride);
int pssfp_tile_voxels(PssfpLaunch L);
// value and T1/T2 tangents (forward mode) in one launch of layout L
void launch_pssfp_tangent(const CompasContext& ctx, const TissueParameters& params, int voxel_begin, int nvoxels,
                          const pSSFPSequence& seq, cfloat* echo, cfloat* dT1, cfloat* dT2, int64_t echo_stride,
                          PssfpLaunch L);
// work-queue launches over (job, tile) items of pSSFP jobs that all use layout L; `real`: every job's
// RF is real (pssfp_sequence_real_rf), which a packed layout runs in its real-RF form
void launch_pssfp_tangent_queue(cudaStream_t stream, int device, PssfpLaunch L, int nz,
                                const kernels::PssfpArgs* jobs, const int2* items, int nitems, int* head,
                                bool real = false);
void launch_pssfp_queue(cudaStream_t stream, int device, PssfpLaunch L, int nz, const kernels::PssfpArgs* jobs,
                        const int2* items, int nitems, int* head, bool real = false);
// whether every RF sample of the sequence (RF train × waveform) is real, read back from its rotation
// table: synchronises the context's stream the first time (not while it is captured)
bool pssfp_sequence_real_rf(const CompasContext& ctx, const pSSFPSequence& seq);

// ---- signal / Jacobian products ----------------------------------------------------------
enum class Precision { FP32, SplitBF16 };

struct CartesianGeom {
    int nreadouts, ns;
    float dt;
    float dk_re, dk_im;
};
CartesianGeom cartesian_geom(const CartesianTrajectory& t);
Precision signal_precision(SimulateSignalMethod m);

// s[c][r][k] = Σ_v coil[c][v]·ρ_v·m[r][v]·w_v·z_v^k  (Cartesian, signal_kernels.cuh:137-167)
void launch_signal_cartesian(const CompasContext& ctx, const float* params, int64_t param_stride, int nvoxels,
                             const cfloat* echos, const cfloat* coils, int ncoils, const CartesianGeom& g,
                             cfloat* signal, Precision prec);
void launch_signal_spiral(const CompasContext& ctx, const float* params, int64_t param_stride, int nvoxels,
                          const cfloat* echos, const cfloat* coils, int ncoils, int nreadouts, int ns, float dt,
                          const cfloat* k_start, const cfloat* delta_k, cfloat* signal, Precision prec);
void launch_jacobian_spiral(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                            const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils, int ncoils,
                            const cfloat* vec, int nreadouts, int ns, float dt, const cfloat* k_start,
                            const cfloat* delta_k, cfloat* Jv, Precision prec);
void launch_jacobian_hermitian_spiral(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                      const cfloat* echos, const cfloat* dT1, const cfloat* dT2,
                                      const cfloat* coils, int ncoils, const cfloat* vec, int nreadouts, int ns,
                                      float dt, const cfloat* k_start, const cfloat* delta_k, cfloat* JHv,
                                      Precision prec);
// split-BF16 tensor-core form; false when it does not apply (no tensor cores, readouts > 1024 samples)
bool launch_jacobian_hermitian_spiral_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                         const cfloat* echos, const cfloat* dT1, const cfloat* dT2,
                                         const cfloat* coils, int ncoils, const cfloat* vec, int nreadouts, int ns,
                                         float dt, const cfloat* k_start, const cfloat* delta_k, cfloat* JHv);
void launch_jacobian(const CompasContext& ctx, const float* params, int64_t param_stride, int nvoxels,
                     const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils, int ncoils,
                     const cfloat* vec, const CartesianGeom& g, cfloat* Jv, Precision prec);
void launch_jacobian_hermitian(const CompasContext& ctx, const float* params, int64_t param_stride, int nvoxels,
                               const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                               int ncoils, const cfloat* vec, const CartesianGeom& g, cfloat* JHv, Precision prec);

// ---- elementwise -------------------------------------------------------------------------
void launch_phase_encoding(const CompasContext& ctx, const cfloat* echos, const float* params, int64_t param_stride,
                           int nvoxels, int nreadouts, const cfloat* k_start, cfloat* out);
void launch_residual(const CompasContext& ctx, const cfloat* lhs, const cfloat* rhs, int64_t n, cfloat* out,
                     float* partials, int npartials, float* objective);
int residual_partial_count(int64_t n);  // partial sums launch_residual uses for n values

// ---- tcgen05 tensor-core complex GEMM support ---------------------------------------------
bool tensor_cores_available(int device);

// tile grid and voxel split of one split-BF16 contraction (a function of its shape only, so a
// job gives the same partial sums alone and inside a batch)
struct TcPlan {
    int ntiles, mtiles, splits, vchunk;  // pair tiles, readout tiles, voxel splits, voxels per split
    int nr;                              // readouts per tile
    int64_t ctas;                        // CTAs of the contraction (CTA pairs × 2)
};
// readouts per tile of the Cartesian contraction: a multiple of 16 up to 256, the fewest tiles,
// then the least padding
int tc_readout_tile(int R);

// ---- tensor-core launch knobs searched by the autotuner -----------------------------------
// Per contraction kind: the readout tile of the Cartesian signal / J·v kernel (a multiple of 16 in
// [16, 256]) and the split count of every kind (voxel splits of the signal and J·v kernels, pair-tile
// splits of the Cartesian Jᴴ·v kernel, readout splits of the spiral Jᴴ·v kernel); 0 = the built-in
// choice. The accuracy bound of the signal and J·v kernels (≤ 512 K16 steps per split) still applies
// to a tuned split count. Chosen, in order, from an explicit override (compas_b200_set_tc_launch),
// the tuning table's "tc" lines, and the built-in heuristics.
enum class TcKind : int {
    CartesianSignal = 0,
    CartesianJacobian = 1,
    CartesianHermitian = 2,
    SpiralSignal = 3,
    SpiralJacobian = 4,
    SpiralHermitian = 5,
    Count = 6,
};
struct TcTuning {
    int tile = 0, splits = 0;
};
// shape class: the kind and the log2 classes of the readout count R, the voxel count and C·S (coils ×
// samples per readout)
TcTuning tuned_tc(TcKind kind, int R, int64_t nvoxels, int64_t coil_samples);
void set_tc_override(int kind, int tile, int splits);
// the launch a call of this shape gets: tile (Cartesian signal / J·v, else 0) and split count
TcTuning tc_launch_choice(int device, TcKind kind, int nvoxels, int R, int S, int C);
// split counts the launches run (tuned or built-in), per kind
int tc_hermitian_splits(int device, int nvoxels, int R, int S, int C);
int tc_spiral_splits(int device, int nvoxels, int R, int S, int C, bool jac);
int tc_spiral_hermitian_splits(int device, int nvoxels, int R, int S, int C);
// readouts per chunk of a spiral contraction whose per-readout table takes `per_readout_bytes`
int spiral_table_chunk(int64_t per_readout_bytes, int R);
TcPlan tc_plan(int device, int nvoxels, int R, int S, int C, bool jac);
// argument block of a Cartesian signal contraction; out / vchunk / status / tables set by the caller
kernels::TcArgs tc_signal_args(const float* params, int64_t pstride, int nvoxels, const cfloat* echos,
                               const cfloat* coils, int ncoils, const CartesianGeom& g);
// device scratch of one contraction, carved from one allocation (byte offsets, 256-aligned):
// per-voxel E_k step and restart values, coil·w, J·v coefficients and the packed A images
struct TcTables {
    int64_t vstep, estart, coilw, jcoef, apack, bytes;
    int egk, apack_stages, nr;
};
TcTables tc_tables(int nvoxels, int R, int S, int C, bool jac);
void tc_assign_tables(kernels::TcArgs& a, const TcTables& t, unsigned char* base);
int tc_pack_blocks(int nr, int R, int apack_stages);  // 256-thread blocks of one job's echo packing
// batched prep (prep_blocks flattened 128-thread blocks), A packing (pack_blocks flattened
// 256-thread blocks) and contraction (ctas flattened CTAs)
void launch_tc_batch(cudaStream_t stream, int device, bool jac, const kernels::TcArgs* jobs, int njobs,
                     const int* prep_offsets, int prep_blocks, const int* pack_offsets, int pack_blocks,
                     const int* cta_offsets, int ctas);

// ---- batched spiral signal and split-K sums -----------------------------------------------
int spiral_coil_group(int ncoils);  // coils per block (1, 2, 4 or 8) of the spiral kernel
int spiral_block_count(int ncoils, int nreadouts, int ns);
void launch_signal_spiral_batch(cudaStream_t stream, int device, int coil_group, const kernels::SpiralArgs* jobs,
                                const int* cta_offsets, int njobs, int ctas);
void launch_sum_partials_batch(cudaStream_t stream, int device, const kernels::PartialSum* jobs,
                               const int* block_offsets, int njobs, int blocks);

// a one-thread kernel whose bounded wait on a barrier nobody completes gives up after
// `limit_cycles` SM cycles and records STATUS_WAIT_TIMEOUT in ctx's status word (diag.cu)
void launch_wait_probe(const CompasContext& ctx, long long limit_cycles);

}  // namespace compas
