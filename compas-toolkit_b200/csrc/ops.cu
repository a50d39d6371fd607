// ops.cu — host entry points of the compas API that are not simulation kernels:
// phase encoding, residual, finite-difference derivatives, and the dispatch of
// magnetization_to_signal / compute_jacobian / compute_jacobian_hermitian to the plain
// FP32 SIMT kernels or the split-BF16 tcgen05 kernels.
#include <mutex>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"

namespace compas {

// implemented in signal.cu / hermitian.cu / tc_complex.cu
void launch_signal_cartesian_simt(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                  const cfloat* echos, const cfloat* coils, int ncoils, const CartesianGeom& g,
                                  cfloat* signal);
void launch_jacobian_simt(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                          const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils, int ncoils,
                          const cfloat* vec, const CartesianGeom& g, cfloat* Jv);
void launch_jacobian_hermitian_simt(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                    const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                                    int ncoils, const cfloat* vec, const CartesianGeom& g, cfloat* JHv);
bool launch_signal_cartesian_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                const cfloat* echos, const cfloat* coils, int ncoils, const CartesianGeom& g,
                                cfloat* signal);
bool launch_jacobian_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                        const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils, int ncoils,
                        const cfloat* vec, const CartesianGeom& g, cfloat* Jv);
bool launch_jacobian_hermitian_tc(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                                  const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                                  int ncoils, const cfloat* vec, const CartesianGeom& g, cfloat* JHv);

namespace kernels {

__global__ void fill_kernel(float* p, int64_t n, float value) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        p[i] = value;
}

// echo[r][v]·exp(i y_v Im k_start[r])   (src/trajectories/phase_encoding_kernels.cuh:10-25)
// One voxel per thread; the CTA rows stride over the readouts, so y is read once per voxel and a
// few thousand CTAs cover the array.
__global__ void phase_encoding_kernel(const float2* __restrict__ echo, const float* __restrict__ params,
                                      int64_t pstride, int nvoxels, int nreadouts, const float2* __restrict__ k_start,
                                      float2* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvoxels) return;
    const double y = double(params[7 * pstride + v]);
    for (int r = blockIdx.y; r < nreadouts; r += gridDim.y) {
        const float2 f = cis_rad(y * double(k_start[r].y));
        const int64_t i = int64_t(r) * nvoxels + v;
        out[i] = cmul(echo[i], f);
    }
}

// d = lhs - rhs, per-block Σ|d|² (fixed-order tree)   (src/utils/residual_kernels.cuh:26-64)
__global__ void residual_kernel(const float2* __restrict__ lhs, const float2* __restrict__ rhs, int64_t n,
                                float2* __restrict__ out, float* __restrict__ partials) {
    __shared__ float red[256];
    float acc = 0.0f;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float2 d = csub(lhs[i], rhs[i]);
        out[i] = d;
        acc = fmaf(d.x, d.x, fmaf(d.y, d.y, acc));
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void sum_kernel(const float* __restrict__ partials, int n, float* __restrict__ result) {
    __shared__ float red[256];
    float acc = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *result = red[0];
}

// copy parameters and add Δ to one field   (src/simulate/derivative_kernels.cuh:6-21)
__global__ void add_difference_kernel(const float* __restrict__ src, float* __restrict__ dst, int64_t nvoxels,
                                      int field, float delta) {
    const int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (v >= nvoxels) return;
    for (int f = 0; f < TissueParameterField::NUM_FIELDS; f++) dst[f * nvoxels + v] = src[f * nvoxels + v];
    dst[field * nvoxels + v] += delta;
}

// (echos1 - echos0) / Δ   (src/simulate/derivative_kernels.cuh:23-35)
__global__ void finite_difference_kernel(const float2* __restrict__ e0, float2* __restrict__ e1, int64_t n,
                                         float inv_delta) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        e1[i] = cscale(inv_delta, csub(e1[i], e0[i]));
}

}  // namespace kernels

void fill_float(float* ptr, int64_t n, float value, cudaStream_t stream) {
    if (n <= 0) return;
    int blocks = int(std::min<int64_t>((n + 255) / 256, 148 * 16));
    kernels::fill_kernel<<<blocks, 256, 0, stream>>>(ptr, n, value);
    check_launch("fill_kernel");
}

void launch_phase_encoding(const CompasContext& ctx, const cfloat* echos, const float* params, int64_t pstride,
                           int nvoxels, int nreadouts, const cfloat* k_start, cfloat* out) {
    if (int64_t(nvoxels) * nreadouts == 0) return;
    DeviceGuard guard(ctx.device());
    const int cols = div_ceil(nvoxels, 256);
    const int rows = std::max(1, std::min(nreadouts, div_ceil(148 * 16, cols)));  // ~16 CTAs per SM
    dim3 block(256), grid(cols, rows);
    kernels::phase_encoding_kernel<<<grid, block, 0, ctx.stream()>>>(
        reinterpret_cast<const float2*>(echos), params, pstride, nvoxels, nreadouts,
        reinterpret_cast<const float2*>(k_start), reinterpret_cast<float2*>(out));
    check_launch("phase_encoding_kernel");
}

Array<cfloat, 2> phase_encoding(const CompasContext& ctx, const Array<cfloat, 2>& echos,
                                const TissueParameters& parameters, const CartesianTrajectory& trajectory) {
    const int nreadouts = trajectory.nreadouts, nvoxels = parameters.nvoxels;
    COMPAS_CHECK(echos.size(0) == nreadouts && echos.size(1) == nvoxels);
    COMPAS_CHECK(trajectory.k_start.size() == nreadouts);
    Array<cfloat, 2> out({nreadouts, nvoxels}, ctx.device(), ctx.stream());
    launch_phase_encoding(ctx, echos.data(), parameters.data.data(), parameters.data.size(1), nvoxels, nreadouts,
                          trajectory.k_start.data(), out.data());
    return out;
}

void launch_residual(const CompasContext& ctx, const cfloat* lhs, const cfloat* rhs, int64_t n, cfloat* out,
                     float* partials, int npartials, float* objective) {
    DeviceGuard guard(ctx.device());
    kernels::residual_kernel<<<npartials, 256, 0, ctx.stream()>>>(reinterpret_cast<const float2*>(lhs),
                                                                  reinterpret_cast<const float2*>(rhs), n,
                                                                  reinterpret_cast<float2*>(out), partials);
    check_launch("residual_kernel");
    kernels::sum_kernel<<<1, 256, 0, ctx.stream()>>>(partials, npartials, objective);
    check_launch("sum_kernel");
}

int residual_partial_count(int64_t n) {
    return int(std::max<int64_t>(1, std::min<int64_t>(1024, (n + 255) / 256)));
}

Array<cfloat, 3> compute_residual(CompasContext ctx, Array<cfloat, 3> lhs, Array<cfloat, 3> rhs, float* objective_out) {
    COMPAS_CHECK(lhs.sizes() == rhs.sizes());
    const int64_t n = lhs.numel();
    Array<cfloat, 3> out(lhs.sizes(), ctx.device());
    const int np = residual_partial_count(n);
    Array<float> partials({np}, ctx.device(), ctx.stream());
    Array<float> objective({1}, ctx.device(), ctx.stream());
    launch_residual(ctx, lhs.data(), rhs.data(), n, out.data(), partials.data(), np, objective.data());
    if (objective_out != nullptr) objective.copy_to(objective_out);
    return out;
}

namespace {
template<typename Sequence>
Array<cfloat, 2> derivative_impl(const CompasContext& ctx, int field, Array<cfloat, 2> echos,
                                 TissueParameters parameters, Sequence sequence, float delta) {
    const int nvoxels = parameters.nvoxels;
    COMPAS_CHECK(echos.size(1) == nvoxels);
    COMPAS_CHECK(field >= 0 && field < TissueParameterField::NUM_FIELDS);
    COMPAS_CHECK(delta != 0.0f);
    Array<float, 2> data({TissueParameterField::NUM_FIELDS, nvoxels}, ctx.device(), ctx.stream());
    DeviceGuard guard(ctx.device());
    if (nvoxels > 0) {
        kernels::add_difference_kernel<<<div_ceil(nvoxels, 256), 256, 0, ctx.stream()>>>(
            parameters.data.data(), data.data(), nvoxels, field, delta);
        check_launch("add_difference_kernel");
    }
    TissueParameters shifted(data, parameters.has_z, parameters.has_b0, parameters.has_b1);
    Array<cfloat, 2> next = simulate_magnetization(ctx, shifted, sequence);
    COMPAS_CHECK(next.sizes() == echos.sizes());
    const int64_t n = next.numel();
    if (n > 0) {
        kernels::finite_difference_kernel<<<int(std::min<int64_t>((n + 255) / 256, 148 * 16)), 256, 0, ctx.stream()>>>(
            reinterpret_cast<const float2*>(echos.data()), reinterpret_cast<float2*>(next.data()), n, 1.0f / delta);
        check_launch("finite_difference_kernel");
    }
    return next;
}
}  // namespace

Array<cfloat, 2> simulate_magnetization_derivative(const CompasContext& context, int field, Array<cfloat, 2> echos,
                                                   TissueParameters parameters, pSSFPSequence sequence, float delta) {
    return derivative_impl(context, field, echos, parameters, sequence, delta);
}

Array<cfloat, 2> simulate_magnetization_derivative(const CompasContext& context, int field, Array<cfloat, 2> echos,
                                                   TissueParameters parameters, FISPSequence sequence, float delta) {
    return derivative_impl(context, field, echos, parameters, sequence, delta);
}

// ---------------------------------------------------------------------------------------
// signal / Jacobian dispatch
// ---------------------------------------------------------------------------------------

bool tensor_cores_available(int device) {
    static int cache[64];
    static std::once_flag flags[64];
    if (device < 0 || device >= 64) return false;
    std::call_once(flags[device], [&] {
        int major = 0, minor = 0;
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device);
        cache[device] = (major == 10 && minor == 0) ? 1 : 0;
    });
    return cache[device] == 1;
}

CartesianGeom cartesian_geom(const CartesianTrajectory& t) {
    return CartesianGeom {t.nreadouts, t.samples_per_readout, t.delta_t, t.delta_k.re, t.delta_k.im};
}

void launch_signal_cartesian(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                             const cfloat* echos, const cfloat* coils, int ncoils, const CartesianGeom& g,
                             cfloat* signal, Precision prec) {
    if (prec == Precision::SplitBF16 &&
        launch_signal_cartesian_tc(ctx, params, pstride, nvoxels, echos, coils, ncoils, g, signal))
        return;
    launch_signal_cartesian_simt(ctx, params, pstride, nvoxels, echos, coils, ncoils, g, signal);
}

void launch_jacobian(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels, const cfloat* echos,
                     const cfloat* dT1, const cfloat* dT2, const cfloat* coils, int ncoils, const cfloat* vec,
                     const CartesianGeom& g, cfloat* Jv, Precision prec) {
    if (prec == Precision::SplitBF16 &&
        launch_jacobian_tc(ctx, params, pstride, nvoxels, echos, dT1, dT2, coils, ncoils, vec, g, Jv))
        return;
    launch_jacobian_simt(ctx, params, pstride, nvoxels, echos, dT1, dT2, coils, ncoils, vec, g, Jv);
}

void launch_jacobian_hermitian(const CompasContext& ctx, const float* params, int64_t pstride, int nvoxels,
                               const cfloat* echos, const cfloat* dT1, const cfloat* dT2, const cfloat* coils,
                               int ncoils, const cfloat* vec, const CartesianGeom& g, cfloat* JHv, Precision prec) {
    if (prec == Precision::SplitBF16 &&
        launch_jacobian_hermitian_tc(ctx, params, pstride, nvoxels, echos, dT1, dT2, coils, ncoils, vec, g, JHv))
        return;
    launch_jacobian_hermitian_simt(ctx, params, pstride, nvoxels, echos, dT1, dT2, coils, ncoils, vec, g, JHv);
}

Precision signal_precision(SimulateSignalMethod m) {
    return (m == SimulateSignalMethod::MatmulFast || m == SimulateSignalMethod::MatmulLow) ? Precision::SplitBF16
                                                                                             : Precision::FP32;
}

static Precision jacobian_precision(JacobianComputeMethod m) {
    return (m == JacobianComputeMethod::GemmFast || m == JacobianComputeMethod::GemmLow) ? Precision::SplitBF16
                                                                                           : Precision::FP32;
}

Array<cfloat, 3> magnetization_to_signal(const CompasContext& context, Array<cfloat, 2> echos,
                                         TissueParameters parameters, const Trajectory& trajectory,
                                         Array<cfloat, 2> coil_sensitivities, SimulateSignalMethod method) {
    const int ncoils = int(coil_sensitivities.size(0));
    const int nvoxels = parameters.nvoxels;
    const int nreadouts = trajectory.nreadouts, ns = trajectory.samples_per_readout;
    COMPAS_CHECK(nreadouts >= 0 && ns >= 0);
    COMPAS_CHECK(coil_sensitivities.size(1) == nvoxels);
    COMPAS_CHECK(echos.size(0) == nreadouts && echos.size(1) == nvoxels);
    Array<cfloat, 3> signal({ncoils, nreadouts, ns}, context.device(), context.stream());
    if (const auto* cart = dynamic_cast<const CartesianTrajectory*>(&trajectory)) {
        launch_signal_cartesian(context, parameters.data.data(), parameters.data.size(1), nvoxels, echos.data(),
                                coil_sensitivities.data(), ncoils, cartesian_geom(*cart), signal.data(),
                                signal_precision(method));
    } else if (const auto* sp = dynamic_cast<const SpiralTrajectory*>(&trajectory)) {
        COMPAS_CHECK(sp->k_start.size() == nreadouts && sp->delta_k.size() == nreadouts);
        launch_signal_spiral(context, parameters.data.data(), parameters.data.size(1), nvoxels, echos.data(),
                             coil_sensitivities.data(), ncoils, nreadouts, ns, sp->delta_t, sp->k_start.data(),
                             sp->delta_k.data(), signal.data(), signal_precision(method));
    } else {
        COMPAS_ERROR("invalid trajectory type");
    }
    return signal;
}

static void check_jacobian_shapes(int nreadouts, int nvoxels, const Array<cfloat, 2>& echos,
                                  const Array<cfloat, 2>& d1, const Array<cfloat, 2>& d2,
                                  const Array<cfloat, 2>& coils) {
    COMPAS_CHECK(echos.size(0) == nreadouts && echos.size(1) == nvoxels);
    COMPAS_CHECK(d1.size(0) == nreadouts && d1.size(1) == nvoxels);
    COMPAS_CHECK(d2.size(0) == nreadouts && d2.size(1) == nvoxels);
    COMPAS_CHECK(coils.size(1) == nvoxels);
}

Array<cfloat, 3> compute_jacobian(const CompasContext& ctx, Array<cfloat, 2> echos, Array<cfloat, 2> delta_echos_T1,
                                  Array<cfloat, 2> delta_echos_T2, TissueParameters parameters,
                                  CartesianTrajectory trajectory, Array<cfloat, 2> coil_sensitivities,
                                  Array<cfloat, 2> vector, JacobianComputeMethod kind) {
    const int ns = trajectory.samples_per_readout, nreadouts = trajectory.nreadouts;
    const int nvoxels = parameters.nvoxels, ncoils = int(coil_sensitivities.size(0));
    check_jacobian_shapes(nreadouts, nvoxels, echos, delta_echos_T1, delta_echos_T2, coil_sensitivities);
    COMPAS_CHECK(vector.size(0) == 4 && vector.size(1) == nvoxels);  // product.cu:304-313
    Array<cfloat, 3> Jv({ncoils, nreadouts, ns}, ctx.device(), ctx.stream());
    launch_jacobian(ctx, parameters.data.data(), parameters.data.size(1), nvoxels, echos.data(), delta_echos_T1.data(),
                    delta_echos_T2.data(), coil_sensitivities.data(), ncoils, vector.data(), cartesian_geom(trajectory),
                    Jv.data(), jacobian_precision(kind));
    return Jv;
}

Array<cfloat, 2> compute_jacobian_hermitian(const CompasContext& ctx, Array<cfloat, 2> echos,
                                            Array<cfloat, 2> delta_echos_T1, Array<cfloat, 2> delta_echos_T2,
                                            TissueParameters parameters, CartesianTrajectory trajectory,
                                            Array<cfloat, 2> coil_sensitivities, Array<cfloat, 3> vector,
                                            JacobianComputeMethod kind) {
    const int ns = trajectory.samples_per_readout, nreadouts = trajectory.nreadouts;
    const int nvoxels = parameters.nvoxels, ncoils = int(coil_sensitivities.size(0));
    check_jacobian_shapes(nreadouts, nvoxels, echos, delta_echos_T1, delta_echos_T2, coil_sensitivities);
    COMPAS_CHECK(vector.size(0) == ncoils && vector.size(1) == nreadouts && vector.size(2) == ns);  // hermitian.cu:265-275
    Array<cfloat, 2> JHv({4, nvoxels}, ctx.device(), ctx.stream());
    launch_jacobian_hermitian(ctx, parameters.data.data(), parameters.data.size(1), nvoxels, echos.data(),
                              delta_echos_T1.data(), delta_echos_T2.data(), coil_sensitivities.data(), ncoils,
                              vector.data(), cartesian_geom(trajectory), JHv.data(), jacobian_precision(kind));
    return JHv;
}

// Spiral trajectories (no counterpart in the reference, whose Jacobians take CartesianTrajectory
// only): derived from the spiral signal model. J·v and Jᴴ·v: split-BF16 tensor cores for
// GemmFast/GemmLow, FP32 otherwise.
Array<cfloat, 3> compute_jacobian(const CompasContext& ctx, Array<cfloat, 2> echos, Array<cfloat, 2> delta_echos_T1,
                                  Array<cfloat, 2> delta_echos_T2, TissueParameters parameters,
                                  SpiralTrajectory trajectory, Array<cfloat, 2> coil_sensitivities,
                                  Array<cfloat, 2> vector, JacobianComputeMethod kind) {
    const int ns = trajectory.samples_per_readout, nreadouts = trajectory.nreadouts;
    const int nvoxels = parameters.nvoxels, ncoils = int(coil_sensitivities.size(0));
    check_jacobian_shapes(nreadouts, nvoxels, echos, delta_echos_T1, delta_echos_T2, coil_sensitivities);
    COMPAS_CHECK(vector.size(0) == 4 && vector.size(1) == nvoxels);
    COMPAS_CHECK(trajectory.k_start.size() == nreadouts && trajectory.delta_k.size() == nreadouts);
    Array<cfloat, 3> Jv({ncoils, nreadouts, ns}, ctx.device(), ctx.stream());
    launch_jacobian_spiral(ctx, parameters.data.data(), parameters.data.size(1), nvoxels, echos.data(),
                           delta_echos_T1.data(), delta_echos_T2.data(), coil_sensitivities.data(), ncoils,
                           vector.data(), nreadouts, ns, trajectory.delta_t, trajectory.k_start.data(),
                           trajectory.delta_k.data(), Jv.data(), jacobian_precision(kind));
    return Jv;
}

Array<cfloat, 2> compute_jacobian_hermitian(const CompasContext& ctx, Array<cfloat, 2> echos,
                                            Array<cfloat, 2> delta_echos_T1, Array<cfloat, 2> delta_echos_T2,
                                            TissueParameters parameters, SpiralTrajectory trajectory,
                                            Array<cfloat, 2> coil_sensitivities, Array<cfloat, 3> vector,
                                            JacobianComputeMethod kind) {
    const int ns = trajectory.samples_per_readout, nreadouts = trajectory.nreadouts;
    const int nvoxels = parameters.nvoxels, ncoils = int(coil_sensitivities.size(0));
    check_jacobian_shapes(nreadouts, nvoxels, echos, delta_echos_T1, delta_echos_T2, coil_sensitivities);
    COMPAS_CHECK(vector.size(0) == ncoils && vector.size(1) == nreadouts && vector.size(2) == ns);
    COMPAS_CHECK(trajectory.k_start.size() == nreadouts && trajectory.delta_k.size() == nreadouts);
    Array<cfloat, 2> JHv({4, nvoxels}, ctx.device(), ctx.stream());
    launch_jacobian_hermitian_spiral(ctx, parameters.data.data(), parameters.data.size(1), nvoxels, echos.data(),
                                     delta_echos_T1.data(), delta_echos_T2.data(), coil_sensitivities.data(), ncoils,
                                     vector.data(), nreadouts, ns, trajectory.delta_t, trajectory.k_start.data(),
                                     trajectory.delta_k.data(), JHv.data(), jacobian_precision(kind));
    return JHv;
}

}  // namespace compas
