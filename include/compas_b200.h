/* compas_b200.h — C ABI of the B200 implementation of the compas-toolkit simulation hot path.
 *
 * Binary drop-in for the reference's Julia binding library (libcompas-julia.so): the first
 * block declares the same 26 `extern "C"` symbols with the same parameter lists, in the
 * order of compas-toolkit julia-bindings/src/bindings.cpp (file:line cited per symbol).
 * Handles are opaque heap objects owned by the caller and released with
 * compas_destroy_object / compas_destroy_array / compas_destroy_context.
 * Complex arrays are interleaved {float re, im}; dimensions are given slowest first
 * (C row-major), i.e. reversed with respect to Julia.
 *
 * Errors: inside a Julia process (symbol `jl_errorf` resolvable) a failing call raises a
 * Julia error exactly like the reference (julia-bindings/src/common.h:48-62). Elsewhere the
 * call returns NULL (or leaves outputs untouched) and compas_last_error() describes the
 * failure; it returns NULL when the last call on this thread succeeded.
 */
#ifndef COMPAS_B200_H
#define COMPAS_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define COMPAS_API __attribute__((visibility("default")))
#else
#define COMPAS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct compas_context compas_context; /* compas::CompasContext */
typedef struct compas_object compas_object;   /* tissue parameters, sequences, trajectories */
typedef struct compas_array compas_array;     /* compas::Array<T, N> */
typedef struct {
    float re, im;
} compas_cfloat;

/* ---- identical to the reference's C ABI ------------------------------------------------ */

/* bindings.cpp:19-21 */
COMPAS_API const char* compas_version(void);
/* bindings.cpp:23-28 */
COMPAS_API const compas_context* compas_make_context(void);
/* bindings.cpp:30-36 */
COMPAS_API const compas_context* compas_copy_context_for_device(compas_context* ctx, int device);
/* bindings.cpp:38-40 */
COMPAS_API void compas_destroy_context(const compas_context* ctx);
/* bindings.cpp:42-44 */
COMPAS_API void compas_destroy_object(const compas_object* obj);
/* bindings.cpp:46-48 */
COMPAS_API void compas_synchronize(const compas_context* ctx);
/* bindings.cpp:50-67: rank 1..3, sizes slowest first */
COMPAS_API const compas_array* compas_make_array_float(const compas_context* ctx, const float* data, int rank, int64_t* sizes);
/* bindings.cpp:69-78: blocking copy of `length` elements */
COMPAS_API void compas_read_array_float(const compas_context* ctx, const compas_array* array, float* dest, int64_t length);
/* bindings.cpp:80-96 */
COMPAS_API const compas_array* compas_make_array_complex(const compas_context* ctx, const compas_cfloat* data, int rank,
                                              int64_t* sizes);
/* bindings.cpp:98-107 */
COMPAS_API void compas_read_array_complex(const compas_context* ctx, const compas_array* array, compas_cfloat* dest,
                               int64_t length);
/* bindings.cpp:109-111 */
COMPAS_API void compas_destroy_array(const compas_array* array);
/* bindings.cpp:117-149: nine host arrays of nvoxels floats (T1,T2,B1,B0,rho_x,rho_y,x,y,z) */
COMPAS_API const compas_object* compas_make_tissue_parameters(const compas_context* ctx, int nvoxels, const float* T1,
                                                   const float* T2, const float* B1, const float* B0,
                                                   const float* rho_x, const float* rho_y, const float* x,
                                                   const float* y, const float* z);
/* bindings.cpp:151-174: RF_train [nTR] complex array, sliceprofiles [npos][nTR] complex array */
COMPAS_API compas_object* compas_make_fisp_sequence(const compas_array* RF_train, const compas_array* sliceprofiles, float TR,
                                         float TE, float TW, int max_state, float TI, int undersampling_factor,
                                         int repetitions);
/* bindings.cpp:176-196: z is a float array */
COMPAS_API compas_object* compas_make_pssfp_sequence(const compas_array* RF_train, float TR, const compas_array* gamma_dt_RF,
                                          float dt_ex, float dt_inv, float dt_pr, float gamma_dt_GRz_ex,
                                          float gamma_dt_GRz_inv, float gamma_dt_GRz_pr, const compas_array* z);
/* bindings.cpp:198-212 */
COMPAS_API compas_object* compas_make_cartesian_trajectory(int nreadouts, int samples_per_readout, float delta_t,
                                                compas_array* k_start, float delta_k);
/* bindings.cpp:214-228 */
COMPAS_API compas_object* compas_make_spiral_trajectory(int nreadouts, int samples_per_readout, float delta_t,
                                             compas_array* k_start, compas_array* delta_k);
/* bindings.cpp:230-241: echos [nreadouts][nvoxels] */
COMPAS_API compas_array* compas_simulate_magnetization_fisp(const compas_context* ctx, const compas_object* parameters,
                                                 const compas_object* sequence);
/* bindings.cpp:243-254 */
COMPAS_API compas_array* compas_simulate_magnetization_pssfp(const compas_context* ctx, const compas_object* parameters,
                                                  const compas_object* sequence);
/* bindings.cpp:256-276: signal [ncoils][nreadouts][ns]; low_precision selects MatmulLow instead
 * of MatmulFast — both run the split-BF16 tensor-core kernels here */
COMPAS_API compas_array* compas_magnetization_to_signal_cartesian(const compas_context* ctx, int ncoils,
                                                       const compas_array* echos, const compas_object* parameters,
                                                       const compas_array* coils, const compas_object* trajectory,
                                                       int32_t low_precision);
/* bindings.cpp:278-294 */
COMPAS_API compas_array* compas_magnetization_to_signal_spiral(const compas_context* ctx, int ncoils, const compas_array* echos,
                                                    const compas_object* parameters, const compas_array* coils,
                                                    const compas_object* trajectory);
/* bindings.cpp:296-322: vector [4][nvoxels] -> [ncoils][nreadouts][ns] */
COMPAS_API compas_array* compas_compute_jacobian(const compas_context* ctx, int ncoils, const compas_array* echos,
                                      const compas_array* delta_echos_T1, const compas_array* delta_echos_T2,
                                      const compas_object* parameters, const compas_array* coils,
                                      const compas_object* trajectory, const compas_array* vector,
                                      const int32_t low_precision);
/* bindings.cpp:324-350: note trajectory before coils; vector [ncoils][nreadouts][ns] -> [4][nvoxels] */
COMPAS_API compas_array* compas_compute_jacobian_hermitian(const compas_context* ctx, int ncoils, const compas_array* echos,
                                                const compas_array* delta_echos_T1,
                                                const compas_array* delta_echos_T2, const compas_object* parameters,
                                                const compas_object* trajectory, const compas_array* coils,
                                                const compas_array* vector, const int32_t low_precision);
/* bindings.cpp:352-365 (no compas_ prefix in the reference) */
COMPAS_API compas_array* phase_encoding(const compas_context* ctx, const compas_array* echos, const compas_object* parameters,
                             const compas_object* trajectory);
/* bindings.cpp:367-374: returns lhs - rhs; *sum = Σ|lhs - rhs|² when sum != NULL */
COMPAS_API compas_array* compas_compute_residual(const compas_context* ctx, const compas_array* lhs, const compas_array* rhs,
                                      float* sum);
/* bindings.cpp:376-393 */
COMPAS_API compas_array* compas_simulate_magnetization_derivative_pssfp(const compas_context* ctx, int field,
                                                             const compas_array* echos,
                                                             const compas_object* parameters, float delta,
                                                             const compas_object* sequence);
/* bindings.cpp:395-411 */
COMPAS_API compas_array* compas_simulate_magnetization_derivative_fisp(const compas_context* ctx, int field,
                                                            const compas_array* echos, const compas_object* parameters,
                                                            float delta, const compas_object* sequence);

/* ---- additions (no counterpart in the reference) ----------------------------------------- */

/* Message of the last failed call on this thread, or NULL. Needed outside Julia, where the
 * reference's jl_errorf path is not available. */
COMPAS_API const char* compas_last_error(void);

/* m, ∂m/∂T1 and ∂m/∂T2 of a FISP or pSSFP sequence in one pass (forward-mode tangents carried
 * with the state). Replaces the pair compas_simulate_magnetization_derivative_{fisp,pssfp}
 * (bindings.cpp:376-411; compas/simulate/derivative.h:7-47) for the fields T1 and T2 by their
 * Δ → 0 limit, and compas_simulate_magnetization_{fisp,pssfp} (bindings.cpp:230-254) for the
 * value (the same recurrence, equal to FP32 rounding). Writes three new [nreadouts][nvoxels] arrays; returns 0, or -1
 * with compas_last_error() set. */
COMPAS_API int compas_b200_simulate_magnetization_tangents(const compas_context* ctx, const compas_object* parameters,
                                                const compas_object* sequence, compas_array** echos,
                                                compas_array** delta_echos_T1, compas_array** delta_echos_T2);

/* compas_make_fisp_sequence with the two flags of the C++ FISPSequence that the reference's C ABI
 * leaves at their defaults (compas/sequences/fisp.h:37-41; bindings.cpp:151-174 always builds the
 * sequence with both true): the inversion prepulse at the start of every repetition and the spoiling
 * before the wait TW. Nonzero = on. Same ownership and errors as compas_make_fisp_sequence. */
COMPAS_API compas_object* compas_b200_make_fisp_sequence_ex(const compas_array* RF_train,
                                                  const compas_array* sliceprofiles, float TR, float TE, float TW,
                                                  int max_state, float TI, int undersampling_factor,
                                                  int repetitions, int inversion_prepulse, int wait_spoiling);

/* Explicit-method variants of the signal and Jacobian entry points: `method` takes the
 * reference's enum values SimulateSignalMethod {Naive=0, Direct, MatmulPedantic, Matmul,
 * MatmulFast, MatmulLow} (compas/trajectories/signal.h:14-44) and JacobianComputeMethod
 * {Naive=0, Direct, Gemm, GemmFast, GemmLow} (compas/jacobian/product.h:10). */
COMPAS_API compas_array* compas_b200_magnetization_to_signal(const compas_context* ctx, const compas_array* echos,
                                                  const compas_object* parameters, const compas_object* trajectory,
                                                  const compas_array* coils, int method);
COMPAS_API compas_array* compas_b200_compute_jacobian(const compas_context* ctx, const compas_array* echos,
                                           const compas_array* delta_echos_T1, const compas_array* delta_echos_T2,
                                           const compas_object* parameters, const compas_object* trajectory,
                                           const compas_array* coils, const compas_array* vector, int method);
COMPAS_API compas_array* compas_b200_compute_jacobian_hermitian(const compas_context* ctx, const compas_array* echos,
                                                     const compas_array* delta_echos_T1,
                                                     const compas_array* delta_echos_T2,
                                                     const compas_object* parameters,
                                                     const compas_object* trajectory, const compas_array* coils,
                                                     const compas_array* vector, int method);

/* The CUDA stream (cudaStream_t) all work of `ctx` is ordered on, and the device pointer,
 * rank and extents of an array — for callers that time or chain work on the device. */
COMPAS_API void* compas_b200_context_stream(const compas_context* ctx);
COMPAS_API void* compas_b200_array_device_ptr(const compas_array* array);
COMPAS_API int compas_b200_array_rank(const compas_array* array);
COMPAS_API int64_t compas_b200_array_extent(const compas_array* array, int axis);

/* Residual without any device allocation (no counterpart in the reference): diff = lhs - rhs
 * over n complex values and *objective = Σ|lhs - rhs|², where lhs, rhs, diff and objective are
 * device pointers on `device` supplied by the caller and the work is ordered on `stream`
 * (a cudaStream_t; NULL is the legacy default stream). For callers that cannot let a library
 * allocate device memory (a fixed, caller-owned memory budget, or a loop that must not trigger
 * allocations). Its scratch is a fixed 256 KB device array inside the library, shared by all calls
 * on a device: n is limited to 16,777,216 (larger n returns an error), and calls whose work
 * overlaps on the GPU race on the scratch. The first call on a device resolves the scratch's
 * address; make it before any stream capture. Returns 0, or -1 with compas_last_error() set. */
COMPAS_API int compas_b200_compute_residual_noalloc(int device, const compas_cfloat* lhs, const compas_cfloat* rhs,
                                                    compas_cfloat* diff, float* objective, int64_t n, void* stream);

/* Failure-channel self-test: enqueue on the context's stream a one-thread kernel whose bounded wait
 * on a barrier that nothing completes gives up after `limit_cycles` SM cycles and records
 * STATUS_WAIT_TIMEOUT; the next compas_synchronize / read of the context then reports "a bounded
 * device-side wait gave up" through compas_last_error() (the device status word is cleared by
 * that report). Returns 0, or -1 on a launch error. */
COMPAS_API int compas_b200_wait_probe(const compas_context* ctx, int64_t limit_cycles);

/* Number of kernels this library has launched in this process (all devices). */
COMPAS_API uint64_t compas_b200_launch_count(void);

/* Launch-layout overrides used by the autotuner: FISP (config index, warps per CTA) and
 * pSSFP (config index); -1 restores the built-in choice. Number/description of layouts. */
COMPAS_API void compas_b200_set_fisp_launch(int config, int warps);
COMPAS_API void compas_b200_set_pssfp_launch(int config);
COMPAS_API int compas_b200_fisp_config_count(void);
COMPAS_API int compas_b200_fisp_config_info(int index, int* states_per_lane, int* lanes);
/* 1 when FISP layout `index` is a packed one-lane layout (two states per two-wide FP32
 * instruction, states_per_lane = 2 x pairs), else 0. */
COMPAS_API int compas_b200_fisp_config_packed(int index);
COMPAS_API int compas_b200_pssfp_config_count(void);
COMPAS_API int compas_b200_pssfp_config_info(int index, int* iso_per_lane, int* lanes);
/* 1 when pSSFP layout `index` is a two-wide layout (iso_per_lane / 2 pairs of isochromats per
 * lane, one two-wide FP32 instruction per pair; the same bits as the scalar layout of that size),
 * else 0. */
COMPAS_API int compas_b200_pssfp_config_packed(int index);
/* Layouts of the FISP tangent kernel (compas_b200_simulate_magnetization_tangents); the
 * override (-1 = built-in choice) applies when it covers the state count. */
COMPAS_API void compas_b200_set_fisp_tangent_launch(int config);
COMPAS_API int compas_b200_fisp_tangent_config_count(void);
COMPAS_API int compas_b200_fisp_tangent_config_info(int index, int* states_per_lane, int* lanes);
/* 1 when FISP tangent layout `index` is a two-wide layout (value, ∂/∂T1 and ∂/∂T2 of states_per_lane
 * states as pairs; the same bits as the scalar tangent layout of that shape), else 0. */
COMPAS_API int compas_b200_fisp_tangent_config_packed(int index);
/* The layout a simulation of this shape gets (override, tuning table, or built-in choice). */
COMPAS_API void compas_b200_fisp_launch_choice(int max_state, int64_t nvoxels, int npositions, int* config,
                                               int* warps);
COMPAS_API int compas_b200_pssfp_launch_choice(int nz, int64_t nvoxels);

/* Tensor-core contraction launches (split-BF16 methods): per kind, the readout tile of the
 * Cartesian signal / J·v kernel (a multiple of 16 in [16, 256]) and the split count (voxel splits
 * of the signal and J·v kernels, pair-tile splits of the Cartesian Jᴴ·v kernel, readout splits of
 * the spiral Jᴴ·v kernel). 0 keeps the tuning table's or the built-in choice. A tile that pads the
 * readout count to more than 17/16 of the rows the built-in tile pads it to is not used (the
 * built-in tile is the multiple of 16 up to 256 that pads least), and the signal and J·v kernels still
 * split so that one split accumulates at most 512 K16 steps. Overrides are process-wide and used by
 * the autotuner while it times candidates. */
#define COMPAS_B200_TC_CARTESIAN_SIGNAL 0
#define COMPAS_B200_TC_CARTESIAN_JACOBIAN 1
#define COMPAS_B200_TC_CARTESIAN_HERMITIAN 2
#define COMPAS_B200_TC_SPIRAL_SIGNAL 3
#define COMPAS_B200_TC_SPIRAL_JACOBIAN 4
#define COMPAS_B200_TC_SPIRAL_HERMITIAN 5
COMPAS_API void compas_b200_set_tc_launch(int kind, int tile, int splits);
/* The tile (0 where the kind has none) and split count a call of this shape runs with on `device`
 * (override, tuning table, or built-in choice). Returns 0, or -1 on a bad kind. */
COMPAS_API int compas_b200_tc_launch_choice(int kind, int device, int nvoxels, int nreadouts,
                                            int samples_per_readout, int ncoils, int* tile, int* splits);

/* Batched jobs (no counterpart in the reference): njobs independent simulate -> signal jobs,
 * job i = (parameters[i], sequences[i] (FISP or pSSFP), trajectories[i] (Cartesian, spiral, or
 * NULL for simulate only), coils[i] ([ncoils][nvoxels] complex; NULL without trajectory)),
 * planned once into a few persistent work-queue / batched launches. `method` is a
 * SimulateSignalMethod value as in compas_b200_magnetization_to_signal. The handle is released
 * with compas_destroy_object. Each job's echoes and signal equal, bit for bit, those of the
 * one-job calls (compas_simulate_magnetization_* then compas_b200_magnetization_to_signal). */
COMPAS_API compas_object* compas_b200_make_batch(const compas_context* ctx, int njobs,
                                                 const compas_object* const* parameters,
                                                 const compas_object* const* sequences,
                                                 const compas_object* const* trajectories,
                                                 const compas_array* const* coils, int method);
/* Enqueue every job of the batch on the context's stream; 0 on success, -1 on error. */
COMPAS_API int compas_b200_batch_run(const compas_object* batch);
/* New array handles sharing the batch's result storage (valid while the batch exists or
 * until released with compas_destroy_array; the next run overwrites them). */
/* As compas_b200_make_batch; tangents[i] != 0 (or tangents == NULL for none) also computes job
 * i's exact derivatives ∂echos/∂T1, ∂echos/∂T2 in the same pass (forward-mode tangents, the bits of
 * compas_b200_simulate_magnetization_tangents for it alone), read with compas_b200_batch_derivative. */
COMPAS_API compas_object* compas_b200_make_batch_tangents(const compas_context* ctx, int njobs,
                                                          const compas_object* const* parameters,
                                                          const compas_object* const* sequences,
                                                          const compas_object* const* trajectories,
                                                          const compas_array* const* coils, int method,
                                                          const int32_t* tangents);
/* field 0: ∂echos/∂T1, 1: ∂echos/∂T2 of a job made with tangents ([nreadouts][nvoxels]) */
COMPAS_API compas_array* compas_b200_batch_derivative(const compas_object* batch, int job, int field);
COMPAS_API compas_array* compas_b200_batch_echos(const compas_object* batch, int job);
COMPAS_API compas_array* compas_b200_batch_signal(const compas_object* batch, int job);

/* One Gauss-Newton iteration of parameter fitting on the device (no counterpart in the
 * reference): simulate, dm/dT1 and dm/dT2 (forward differences with step `delta`, or, for
 * delta = 0, exact forward-mode tangents in the simulation pass), signal, residual against `data`
 * ([ncoils][nreadouts][ns] complex), `cg_iterations` CGLS steps of J.v / J^H.v, then a line search
 * on the objective |y - s(p)|^2 (src/utils/residual.cu:8-46): the first of the steps t = 1, 1/2
 * that does not raise it is taken, else none, so the objective never rises between iterations.
 * Captured as a CUDA graph on the first graph run. `method` is a JacobianComputeMethod value.
 * The estimate starts as a copy of `parameters`. Released with compas_destroy_object. */
COMPAS_API compas_object* compas_b200_make_gauss_newton(const compas_context* ctx, const compas_object* parameters,
                                                        const compas_object* sequence,
                                                        const compas_object* trajectory, const compas_array* coils,
                                                        const compas_array* data, int cg_iterations, float delta,
                                                        int method);
/* Enqueue one iteration (graph replay when use_graph != 0); 0 on success, -1 on error. */
COMPAS_API int compas_b200_gauss_newton_run(const compas_object* gn, int use_graph);
/* New array handle sharing the iteration's device storage: 0 parameters [9][nvoxels] float,
 * 1 echoes, 2 dm/dT1, 3 dm/dT2 ([nreadouts][nvoxels] complex), 4 signal [ncoils][nreadouts][ns],
 * 5 J^H.b [4][nvoxels] complex, 6 step [4][nvoxels] float, 7 scalars [8] float
 * (objective before the update, gamma, gamma', |q|^2, alpha, beta, objective of the last
 * line-search trial, step length taken: 1, 0.5 or 0). */
COMPAS_API compas_array* compas_b200_gauss_newton_array(const compas_object* gn, int which);
/* Line search on (1, the default) or off (0: the full CGLS step is always applied). Changing it
 * drops the captured graph. 0 on success, -1 on error. */
COMPAS_API int compas_b200_gauss_newton_set_line_search(const compas_object* gn, int on);
/* Kernel nodes of the captured graph, -1 before the first graph run. */
COMPAS_API int compas_b200_gauss_newton_graph_kernels(const compas_object* gn);

/* GEMM utilities (compas/utils/gemm.h:7-70; the reference's C ABI does not export them).
 * result = alpha * lhs * rhs^T + beta * result with lhs [m][k], rhs [n][k], result [m][n] float
 * arrays (result is not read when beta == 0); the complex form takes planar [2][rows][cols] arrays
 * (plane 0 real, plane 1 imaginary). `method` is a GemmComputeMethod value: 0 Pedantic and
 * 1 Regular compute in FP32 on the CUDA cores, 2 Fast in split-BF16 on the tensor cores (~1e-5
 * relative). BF16 arrays (compas_b200_make_array_bfloat16) run on the tensor cores for every method.
 * 0, or -1 on error. */
COMPAS_API int compas_b200_compute_gemm(const compas_context* ctx, compas_array* result, const compas_array* lhs,
                                        const compas_array* rhs, float alpha, float beta, int method);
COMPAS_API int compas_b200_compute_complex_gemm(const compas_context* ctx, compas_array* result,
                                                const compas_array* lhs, const compas_array* rhs, float alpha,
                                                float beta, int method);
/* interleaved complex [n][m] -> planar [2][n][m] (float, or bfloat16 rounded to nearest) and back */
COMPAS_API int compas_b200_convert_complex_to_planar(const compas_context* ctx, compas_array* output,
                                                     const compas_array* input);
COMPAS_API int compas_b200_convert_planar_to_complex(const compas_context* ctx, compas_array* output,
                                                     const compas_array* input);
/* bfloat16 arrays (raw 16-bit patterns), as compas_make_array_float / compas_read_array_float */
COMPAS_API const compas_array* compas_b200_make_array_bfloat16(const compas_context* ctx, const uint16_t* data,
                                                               int rank, int64_t* sizes);
COMPAS_API void compas_b200_read_array_bfloat16(const compas_context* ctx, const compas_array* array, uint16_t* dest,
                                                int64_t length);

/* One slice sharded over processes, one GPU each (no counterpart in the reference's C ABI; its
 * kmm runtime chunks voxels over the devices of one process, include/compas/core/context.h:51-68,
 * and sums the chunks' signals, src/trajectories/signal.cu:289-300).
 * compas_b200_voxel_shard: voxels [begin, end) of `rank` among `world` ranks, contiguous, sizes
 * differing by at most one (host-only; needs no device). 0, or -1 on invalid arguments. */
COMPAS_API int compas_b200_voxel_shard(int64_t nvoxels, int rank, int world, int64_t* begin, int64_t* end);
/* A new NCCL unique id (128 bytes) into `out` (nbytes >= 128): one rank makes it and the caller
 * sends it to the others. Returns the bytes written, or -1. */
COMPAS_API int compas_b200_comm_unique_id(char* out, int nbytes);
/* NCCL communicator over `world` processes on the context's device; every rank passes the same
 * unique id and the call blocks until all have joined. NCCL (libnccl.so.2) is loaded at run time.
 * Released with compas_destroy_object. */
COMPAS_API compas_object* compas_b200_make_communicator(const compas_context* ctx, int rank, int world,
                                                        const char* unique_id);
/* In-place sum over the ranks of a float or complex array, ordered on the context's stream.
 * 0, or -1 on error. */
COMPAS_API int compas_b200_allreduce_sum(const compas_context* ctx, const compas_object* comm, compas_array* array);
/* Signal / J.v of a slice whose voxels are sharded over the communicator's ranks: each rank passes
 * its own voxels (echoes [nreadouts][nvoxels_rank], parameters, coils [ncoils][nvoxels_rank], for
 * J.v also the derivative echoes and the direction [4][nvoxels_rank]) and every rank receives the
 * full [ncoils][nreadouts][ns] sum. `method` as in compas_b200_magnetization_to_signal /
 * compas_b200_compute_jacobian. J^H.v needs no such variant: each rank computes its own voxels'
 * gradient from the full residual with compas_b200_compute_jacobian_hermitian. */
COMPAS_API compas_array* compas_b200_magnetization_to_signal_sharded(const compas_context* ctx,
                                                                     const compas_object* comm,
                                                                     const compas_array* echos,
                                                                     const compas_object* parameters,
                                                                     const compas_object* trajectory,
                                                                     const compas_array* coils, int method);
COMPAS_API compas_array* compas_b200_compute_jacobian_sharded(const compas_context* ctx, const compas_object* comm,
                                                              const compas_array* echos,
                                                              const compas_array* delta_echos_T1,
                                                              const compas_array* delta_echos_T2,
                                                              const compas_object* parameters,
                                                              const compas_object* trajectory,
                                                              const compas_array* coils, const compas_array* vector,
                                                              int method);

/* Continuous-batching serving engine (no counterpart in the reference). Requests (parameters,
 * FISP or pSSFP sequence, Cartesian or spiral trajectory, coils [ncoils][nvoxels], measured data
 * [ncoils][nreadouts][ns]) are admitted by estimated device footprint against
 * `memory_budget_gb`, grouped into batches (at most `max_batch_requests` each, at most
 * `max_inflight_batches` on the device at once) and give residual, objective and gradient J^H.r.
 * Each batch slot reports kernel errors in a status word of its own, so a failing batch fails only
 * its own requests. A nonzero echo_key lets requests with equal parameters and sequence share
 * resident echoes (`echo_cache_gb`). `method` is a SimulateSignalMethod value. `delta` is the
 * forward-difference step of the derivatives; 0 takes exact forward-mode tangents from the
 * simulation pass. Released with compas_destroy_object, which finishes queued requests first. */
COMPAS_API compas_object* compas_b200_make_server(const compas_context* ctx, double memory_budget_gb,
                                                  int max_inflight_batches, int max_batch_requests,
                                                  double echo_cache_gb, int method, float delta);
/* Queue a request; returns its ticket (> 0) or -1 on error. */
COMPAS_API int64_t compas_b200_server_submit(const compas_object* server, const compas_object* parameters,
                                             const compas_object* sequence, const compas_object* trajectory,
                                             const compas_array* coils, const compas_array* data,
                                             uint64_t echo_key);
/* compas_b200_server_submit with request flags. COMPAS_B200_REQUEST_INJECT_WAIT_TIMEOUT (a test hook
 * of the failure path): the batch that runs the request also runs a kernel whose bounded wait
 * gives up, so that batch's requests fail with "a bounded device-side wait gave up" while other
 * batches, on other slots, complete. */
#define COMPAS_B200_REQUEST_INJECT_WAIT_TIMEOUT 1
COMPAS_API int64_t compas_b200_server_submit_flags(const compas_object* server, const compas_object* parameters,
                                                   const compas_object* sequence, const compas_object* trajectory,
                                                   const compas_array* coils, const compas_array* data,
                                                   uint64_t echo_key, int flags);
/* Block until the request completed: objective, times[3] = queued, device, latency (ms), batch
 * id; 0 on success, -1 if it failed (message in compas_last_error). */
COMPAS_API int compas_b200_server_wait(const compas_object* server, int64_t ticket, float* objective,
                                       double* times, int* batch);
/* Result arrays of a completed request: 0 residual [ncoils][nreadouts][ns], 1 gradient J^H.r
 * [4][nvoxels] (Cartesian and spiral trajectories). New handles, valid after release. */
COMPAS_API compas_array* compas_b200_server_result(const compas_object* server, int64_t ticket, int which);
COMPAS_API int compas_b200_server_release(const compas_object* server, int64_t ticket);
COMPAS_API int compas_b200_server_drain(const compas_object* server);
/* Statistics: out[0..9] = completed, failed, batches, echo cache hits, p50, p99, mean, max latency
 * (ms), peak footprint (bytes), most batches in flight at once. Returns the count written. */
COMPAS_API int compas_b200_server_stats(const compas_object* server, double* out, int n);
COMPAS_API void compas_b200_server_reset_stats(const compas_object* server);

#ifdef __cplusplus
}
#endif

#endif /* COMPAS_B200_H */
