// gn.cu — one Gauss–Newton iteration of MR-STAT parameter fitting, captured as a CUDA graph.
//
// MR-STAT fits tissue parameters p (T1, T2, ρ per voxel) to measured k-space data y by
// minimising ½‖s(p) - y‖². The reference provides the operations and leaves the iteration to
// the caller (its Julia examples chain simulate_magnetization, the finite-difference
// derivatives, magnetization_to_signal, compute_residual, compute_jacobian and
// compute_jacobian_hermitian: src/simulate/derivative.cu:11-94, src/utils/residual.cu:8-46,
// src/jacobian/product.cu, src/jacobian/hermitian.cu). Here the whole iteration is enqueued
// on the context's stream with every buffer allocated once, and is captured into a CUDA graph
// on first use, so one replay issues the ~20 kernels of an iteration with one launch:
//
//   m = simulate(p);  ∂m/∂T1, ∂m/∂T2 by forward differences (absolute step Δ, as the reference),
//   or, with Δ = 0, m and its exact derivatives in one forward-mode tangent pass;
//   s = signal(m);  b = y - s;  objective = ‖b‖²;
//   CGLS on the linearised problem  min_δ ‖J δ - b‖²  over real δ in the scaled coordinates
//   of the Jacobian (δT1/T1, δT2/T2, δRe ρ, δIm ρ), starting from δ = 0:
//       g = Re(Jᴴ b), d = g, γ = ‖g‖²;  repeat k times:
//       q = J d;  α = γ/‖q‖²;  δ += α d;  b -= α q;  g = Re(Jᴴ b);  γ' = ‖g‖²;  d = g + (γ'/γ) d
//   p ← (T1·c(δ0), T2·c(δ1), Re ρ + δ2, Im ρ + δ3) with c(x) = min(max(1 + x, ½), 2), which
//   keeps T1, T2 positive for large steps.
// With the line search (the default), the step is tried on the objective first: the trial
// p(t) (δ scaled by t) is simulated, its signal and ‖y - s(p(t))‖² computed, and the first of
// t = 1, ½ whose objective is not above ‖y - s(p)‖² is taken; if neither is, p stays, so the
// objective never rises from one iteration to the next (the reference's objective:
// src/utils/residual.cu:8-46). A graph cannot branch, so the kernels of the t = ½ trial read a
// device flag and return at once when t = 1 was taken; and an accepted trial's echoes are m of
// the next iteration's estimate, so that iteration copies them instead of simulating again.
//
// Scalars (γ, α, β, norms) stay on the device; every reduction uses a fixed grid and a fixed
// summation order, so a replayed graph reproduces the eager iteration bit for bit.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"

namespace compas {
namespace kernels {
// ops.cu
__global__ void residual_kernel(const float2* __restrict__ lhs, const float2* __restrict__ rhs, int64_t n,
                                float2* __restrict__ out, float* __restrict__ partials);
__global__ void sum_kernel(const float* __restrict__ partials, int n, float* __restrict__ result);
__global__ void add_difference_kernel(const float* __restrict__ src, float* __restrict__ dst, int64_t nvoxels,
                                      int field, float delta);
__global__ void finite_difference_kernel(const float2* __restrict__ e0, float2* __restrict__ e1, int64_t n,
                                         float inv_delta);

namespace {

constexpr int kRedBlocks = 296;  // fixed grid of every reduction: 2 CTAs per SM on 148 SMs
constexpr int kRedThreads = 256;

// scalar slots in the device scalar array
enum Scalar {
    kObjective = 0, kGamma = 1, kGammaNew = 2, kQQ = 3, kAlpha = 4, kBeta = 5,
    kTrial = 6,       // ‖y - s(p(t))‖² of the last trial of the line search
    kStepLength = 7,  // t taken by the line search: 1, ½, or 0 (no step)
    kNumScalars = 8
};
// device flags of the line search
enum Flag { kAccepted = 0, kHaveEchoes = 1, kNumFlags = 2 };

__device__ __forceinline__ float block_sum(float v, float* red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    return red[0];
}

// partials[b] = Σ over the grid-stride share of block b of |z|² (complex) or, when real_part,
// of (Re z)²
__global__ void norm2_partials_kernel(const float2* __restrict__ z, int64_t n, bool real_part,
                                      float* __restrict__ partials) {
    __shared__ float red[kRedThreads];
    float acc = 0.0f;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float2 v = z[i];
        acc = fmaf(v.x, v.x, acc);
        if (!real_part) acc = fmaf(v.y, v.y, acc);
    }
    const float s = block_sum(acc, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// scalars[slot] = Σ partials (one block, fixed order); then the CG scalar updates that depend on it
__global__ void finish_norm_kernel(const float* __restrict__ partials, int n, float* __restrict__ scalars, int slot,
                                   int mode) {
    __shared__ float red[kRedThreads];
    float acc = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
    const float s = block_sum(acc, red);
    if (threadIdx.x == 0) {
        scalars[slot] = s;
        if (mode == 1) {  // after ‖q‖²: α = γ / ‖q‖²
            scalars[kAlpha] = s > 0.0f ? scalars[kGamma] / s : 0.0f;
        } else if (mode == 2) {  // after γ' = ‖g‖²: β = γ'/γ, γ = γ'
            const float g = scalars[kGamma];
            scalars[kBeta] = g > 0.0f ? s / g : 0.0f;
            scalars[kGamma] = s;
        }
    }
}

// δ = 0, d = Re g (imaginary part 0)
__global__ void cg_start_kernel(const float2* __restrict__ g, int64_t n, float* __restrict__ x,
                                float2* __restrict__ d) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        x[i] = 0.0f;
        d[i] = make_float2(g[i].x, 0.0f);
    }
}

// δ += α d (real, n4 entries)
__global__ void cg_step_x_kernel(float* __restrict__ x, const float2* __restrict__ d, int64_t n,
                                 const float* __restrict__ scalars) {
    const float alpha = scalars[kAlpha];
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        x[i] = fmaf(alpha, d[i].x, x[i]);
}

// b -= α q (complex data-space residual)
__global__ void cg_step_b_kernel(float2* __restrict__ b, const float2* __restrict__ q, int64_t n,
                                 const float* __restrict__ scalars) {
    const float alpha = scalars[kAlpha];
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        b[i] = make_float2(fmaf(-alpha, q[i].x, b[i].x), fmaf(-alpha, q[i].y, b[i].y));
}

// d = Re g + β d
__global__ void cg_direction_kernel(const float2* __restrict__ g, float2* __restrict__ d, int64_t n,
                                    const float* __restrict__ scalars) {
    const float beta = scalars[kBeta];
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        d[i] = make_float2(fmaf(beta, d[i].x, g[i].x), 0.0f);
}

// parameter update from δ [4][V] in the scaled coordinates of the Jacobian columns
__global__ void gn_update_kernel(float* __restrict__ params, int64_t pstride, int nvoxels,
                                 const float* __restrict__ x) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvoxels) return;
    const float c1 = fminf(fmaxf(1.0f + x[v], 0.5f), 2.0f);
    const float c2 = fminf(fmaxf(1.0f + x[nvoxels + v], 0.5f), 2.0f);
    params[0 * pstride + v] *= c1;
    params[1 * pstride + v] *= c2;
    params[4 * pstride + v] += x[2 * int64_t(nvoxels) + v];
    params[5 * pstride + v] += x[3 * int64_t(nvoxels) + v];
}

// trial parameters p(t): T1·c(t·δ0), T2·c(t·δ1), ρ + t·(δ2 + iδ3), the other fields as in p (the
// trial array holds them from construction). The first trial resets the accepted flag and the
// step length; a later trial returns at once when an earlier one was taken.
__global__ void gn_trial_kernel(const float* __restrict__ params, float* __restrict__ trial, int64_t pstride,
                                int nvoxels, const float* __restrict__ x, float t, bool first, int* __restrict__ flags,
                                float* __restrict__ scalars) {
    if (first) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            flags[kAccepted] = 0;
            scalars[kStepLength] = 0.0f;
        }
    } else if (flags[kAccepted] != 0) {
        return;
    }
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvoxels) return;
    const float c1 = fminf(fmaxf(fmaf(t, x[v], 1.0f), 0.5f), 2.0f);
    const float c2 = fminf(fmaxf(fmaf(t, x[nvoxels + v], 1.0f), 0.5f), 2.0f);
    trial[0 * pstride + v] = params[0 * pstride + v] * c1;
    trial[1 * pstride + v] = params[1 * pstride + v] * c2;
    trial[4 * pstride + v] = fmaf(t, x[2 * int64_t(nvoxels) + v], params[4 * pstride + v]);
    trial[5 * pstride + v] = fmaf(t, x[3 * int64_t(nvoxels) + v], params[5 * pstride + v]);
}

// take step length t when no earlier trial was taken and this trial's objective is not above the
// estimate's (a NaN objective is never taken)
__global__ void gn_decide_kernel(float* __restrict__ scalars, int* __restrict__ flags, float t) {
    if (flags[kAccepted] != 0) return;
    if (scalars[kTrial] <= scalars[kObjective]) {
        flags[kAccepted] = 1;
        scalars[kStepLength] = t;
    }
}

// p ← the taken trial (fields T1, T2, ρ); records whether the trial's echoes are m(p) now
__global__ void gn_commit_kernel(float* __restrict__ params, const float* __restrict__ trial, int64_t pstride,
                                 int nvoxels, int* __restrict__ flags) {
    const bool taken = flags[kAccepted] != 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) flags[kHaveEchoes] = taken ? 1 : 0;
    if (!taken) return;
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvoxels) return;
    for (int f : {0, 1, 4, 5}) params[f * pstride + v] = trial[f * pstride + v];
}

// echos ← the last taken trial's echoes, when they belong to the current estimate
__global__ void gn_take_echoes_kernel(float2* __restrict__ echos, const float2* __restrict__ trial_echos, int64_t n,
                                      const int* __restrict__ flags) {
    if (flags[kHaveEchoes] == 0) return;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        echos[i] = trial_echos[i];
}

}  // namespace
}  // namespace kernels

struct GaussNewtonStep::Impl {
    explicit Impl(const CompasContext& c) : ctx(c) {}
    Impl(const Impl&) = delete;
    Impl& operator=(const Impl&) = delete;
    ~Impl() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }

    CompasContext ctx;
    TissueParameters params;   // the estimate, updated in place by every iteration
    Array<float, 2> perturbed;
    std::variant<FISPSequence, pSSFPSequence> sequence;
    std::variant<CartesianTrajectory, SpiralTrajectory> trajectory;
    Array<cfloat, 2> coils;
    Array<cfloat, 3> data;
    int cg_iterations = 4;
    float delta = DEFAULT_FINITE_DIFFERENCE_DELTA;
    Precision prec = Precision::SplitBF16;
    bool line_search = true;
    Array<float, 2> trial;          // trial parameters of the line search
    Array<cfloat, 2> trial_echos;   // m(trial)
    Array<cfloat, 3> trial_signal;  // s(trial)
    Array<int> flags;               // kernels::Flag
    Array<int> handoff;             // per-CTA flags of the balanced FISP split (zeroed per simulation)
    static constexpr int kHandoffCapacity = 4096;

    Array<cfloat, 2> echos, dT1, dT2;
    Array<cfloat, 3> signal, b, q;
    Array<cfloat, 2> g, d;
    Array<float, 2> x;
    Array<float> scalars, partials;
    int npartials = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    // m(p) into `out`; with `skip`, nothing when *skip != 0 at run time
    void simulate(const TissueParameters& p, cfloat* out, const int* skip = nullptr) const {
        const int V = p.nvoxels;
        if (const auto* f = std::get_if<FISPSequence>(&sequence)) {
            launch_fisp(ctx, p, 0, V, *f, out, V, tuned_fisp_launch(f->max_state, V, int(f->sliceprofiles.size(0))),
                        skip, true, handoff.data(), kHandoffCapacity);
        } else {
            const auto& s = std::get<pSSFPSequence>(sequence);
            launch_pssfp(ctx, p, 0, V, s, out, V, tuned_pssfp_launch(int(s.z.size()), V), skip);
        }
    }

    void norm2(const cfloat* z, int64_t n, bool real_part, int slot, int mode) const {
        kernels::norm2_partials_kernel<<<kernels::kRedBlocks, kernels::kRedThreads, 0, ctx.stream()>>>(
            reinterpret_cast<const float2*>(z), n, real_part, partials.data());
        check_launch("norm2_partials_kernel");
        kernels::finish_norm_kernel<<<1, kernels::kRedThreads, 0, ctx.stream()>>>(
            partials.data(), kernels::kRedBlocks, scalars.data(), slot, mode);
        check_launch("finish_norm_kernel");
    }

    void enqueue() const;
};

void GaussNewtonStep::Impl::enqueue() const {
    using namespace kernels;
    const int V = params.nvoxels;
    const int64_t nv4 = 4 * int64_t(V);
    const int64_t nsig = signal.numel();
    const int64_t necho = echos.numel();
    const int C = int(coils.size(0));
    const float* pdata = params.data.data();
    const int64_t pstride = params.data.size(1);
    const auto* cart = std::get_if<CartesianTrajectory>(&trajectory);
    const auto* spiral = std::get_if<SpiralTrajectory>(&trajectory);
    const CartesianGeom geo = cart ? cartesian_geom(*cart) : CartesianGeom {};
    // J·d and Jᴴ·b on the request's trajectory (spiral: the FP32 spiral kernels)
    auto jv = [&](const cfloat* vec, cfloat* out) {
        if (cart)
            launch_jacobian(ctx, pdata, pstride, V, echos.data(), dT1.data(), dT2.data(), coils.data(), C, vec, geo, out,
                            prec);
        else
            launch_jacobian_spiral(ctx, pdata, pstride, V, echos.data(), dT1.data(), dT2.data(), coils.data(), C, vec,
                                   spiral->nreadouts, spiral->samples_per_readout, spiral->delta_t,
                                   spiral->k_start.data(), spiral->delta_k.data(), out, prec);
    };
    auto jhv = [&](const cfloat* vec, cfloat* out) {
        if (cart)
            launch_jacobian_hermitian(ctx, pdata, pstride, V, echos.data(), dT1.data(), dT2.data(), coils.data(), C,
                                      vec, geo, out, prec);
        else
            launch_jacobian_hermitian_spiral(ctx, pdata, pstride, V, echos.data(), dT1.data(), dT2.data(),
                                             coils.data(), C, vec, spiral->nreadouts, spiral->samples_per_readout,
                                             spiral->delta_t, spiral->k_start.data(), spiral->delta_k.data(), out, prec);
    };
    cudaStream_t st = ctx.stream();
    const int eb = int(std::min<int64_t>((necho + 255) / 256, 148 * 16));
    const int sb = int(std::min<int64_t>((nsig + 255) / 256, 148 * 16));
    const int vb = int(std::min<int64_t>((nv4 + 255) / 256, 148 * 16));

    // model and derivatives: exact tangents in one pass (delta = 0), or forward differences
    if (delta == 0.0f) {
        if (const auto* f = std::get_if<FISPSequence>(&sequence)) {
            launch_fisp_tangent(ctx, params, 0, V, *f, echos.data(), dT1.data(), dT2.data(), V,
                                tuned_fisp_tangent_launch(f->max_state, V, int(f->sliceprofiles.size(0))));
        } else {
            const auto& s = std::get<pSSFPSequence>(sequence);
            launch_pssfp_tangent(ctx, params, 0, V, s, echos.data(), dT1.data(), dT2.data(), V,
                                 tuned_pssfp_launch(int(s.z.size()), V));
        }
    } else if (line_search) {
        // the previous iteration's taken trial already simulated the estimate: copy its echoes
        gn_take_echoes_kernel<<<eb, 256, 0, st>>>(reinterpret_cast<float2*>(echos.data()),
                                                  reinterpret_cast<const float2*>(trial_echos.data()), necho,
                                                  flags.data());
        check_launch("gn_take_echoes_kernel");
        simulate(params, echos.data(), flags.data() + kHaveEchoes);
    } else {
        simulate(params, echos.data());
    }
    const TissueParameters shifted(perturbed, params.has_z, params.has_b0, params.has_b1);
    const Array<cfloat, 2>* dst[2] = {&dT1, &dT2};
    for (int field = 0; field < 2 && delta != 0.0f; field++) {
        add_difference_kernel<<<div_ceil(V, 256), 256, 0, st>>>(pdata, perturbed.data(), V, field, delta);
        check_launch("add_difference_kernel");
        simulate(shifted, dst[field]->data());
        finite_difference_kernel<<<eb, 256, 0, st>>>(reinterpret_cast<const float2*>(echos.data()),
                                                     reinterpret_cast<float2*>(dst[field]->data()), necho,
                                                     1.0f / delta);
        check_launch("finite_difference_kernel");
    }

    // residual b = y - s and the objective ‖b‖²
    if (cart)
        launch_signal_cartesian(ctx, pdata, pstride, V, echos.data(), coils.data(), C, geo, signal.data(), prec);
    else
        launch_signal_spiral(ctx, pdata, pstride, V, echos.data(), coils.data(), C, spiral->nreadouts,
                             spiral->samples_per_readout, spiral->delta_t, spiral->k_start.data(),
                             spiral->delta_k.data(), signal.data(), prec);
    launch_residual(ctx, data.data(), signal.data(), nsig, b.data(), partials.data(), npartials,
                    scalars.data() + kObjective);

    // CGLS, k iterations of one J·d and one Jᴴ·b each
    jhv(b.data(), g.data());
    cg_start_kernel<<<vb, 256, 0, st>>>(reinterpret_cast<const float2*>(g.data()), nv4, x.data(),
                                        reinterpret_cast<float2*>(d.data()));
    check_launch("cg_start_kernel");
    norm2(g.data(), nv4, true, kGamma, 0);
    for (int it = 0; it < cg_iterations; it++) {
        jv(d.data(), q.data());
        norm2(q.data(), nsig, false, kQQ, 1);
        cg_step_x_kernel<<<vb, 256, 0, st>>>(x.data(), reinterpret_cast<const float2*>(d.data()), nv4,
                                             scalars.data());
        check_launch("cg_step_x_kernel");
        if (it + 1 == cg_iterations) break;
        cg_step_b_kernel<<<sb, 256, 0, st>>>(reinterpret_cast<float2*>(b.data()),
                                             reinterpret_cast<const float2*>(q.data()), nsig, scalars.data());
        check_launch("cg_step_b_kernel");
        jhv(b.data(), g.data());
        norm2(g.data(), nv4, true, kGammaNew, 2);
        cg_direction_kernel<<<vb, 256, 0, st>>>(reinterpret_cast<const float2*>(g.data()),
                                                reinterpret_cast<float2*>(d.data()), nv4, scalars.data());
        check_launch("cg_direction_kernel");
    }
    if (!line_search) {
        gn_update_kernel<<<div_ceil(V, 256), 256, 0, st>>>(params.data.data(), pstride, V, x.data());
        check_launch("gn_update_kernel");
        return;
    }

    // line search on the objective: t = 1, then t = ½ (whose kernels return at once if 1 was taken)
    const TissueParameters tp(trial, params.has_z, params.has_b0, params.has_b1);
    const float steps[2] = {1.0f, 0.5f};
    for (int k = 0; k < 2; k++) {
        gn_trial_kernel<<<div_ceil(V, 256), 256, 0, st>>>(pdata, trial.data(), pstride, V, x.data(), steps[k], k == 0,
                                                          flags.data(), scalars.data());
        check_launch("gn_trial_kernel");
        simulate(tp, trial_echos.data(), k == 0 ? nullptr : flags.data() + kAccepted);
        if (cart)
            launch_signal_cartesian(ctx, trial.data(), pstride, V, trial_echos.data(), coils.data(), C, geo,
                                    trial_signal.data(), prec);
        else
            launch_signal_spiral(ctx, trial.data(), pstride, V, trial_echos.data(), coils.data(), C, spiral->nreadouts,
                                 spiral->samples_per_readout, spiral->delta_t, spiral->k_start.data(),
                                 spiral->delta_k.data(), trial_signal.data(), prec);
        launch_residual(ctx, data.data(), trial_signal.data(), nsig, q.data(), partials.data(), npartials,
                        scalars.data() + kTrial);
        gn_decide_kernel<<<1, 1, 0, st>>>(scalars.data(), flags.data(), steps[k]);
        check_launch("gn_decide_kernel");
    }
    gn_commit_kernel<<<div_ceil(V, 256), 256, 0, st>>>(params.data.data(), trial.data(), pstride, V, flags.data());
    check_launch("gn_commit_kernel");
}

GaussNewtonStep::GaussNewtonStep(const CompasContext& ctx, TissueParameters parameters,
                                 std::variant<FISPSequence, pSSFPSequence> sequence,
                                 std::variant<CartesianTrajectory, SpiralTrajectory> trajectory,
                                 Array<cfloat, 2> coil_sensitivities, Array<cfloat, 3> data, int cg_iterations,
                                 float delta, JacobianComputeMethod method) :
    m_impl(std::make_shared<Impl>(ctx)) {
    Impl& im = *m_impl;
    const int dev = ctx.device();
    const int V = parameters.nvoxels;
    const int C = int(coil_sensitivities.size(0));
    const Trajectory& tr = std::holds_alternative<CartesianTrajectory>(trajectory)
                               ? static_cast<const Trajectory&>(std::get<CartesianTrajectory>(trajectory))
                               : static_cast<const Trajectory&>(std::get<SpiralTrajectory>(trajectory));
    const int R = tr.nreadouts, S = tr.samples_per_readout;
    int nreadouts = 0;
    if (const auto* f = std::get_if<FISPSequence>(&sequence)) nreadouts = int(f->RF_train.size()) * f->undersampling_factor;
    else nreadouts = int(std::get<pSSFPSequence>(sequence).RF_train.size());
    if (nreadouts != R) COMPAS_ERROR("trajectory readouts do not match the sequence's echoes");
    COMPAS_CHECK(coil_sensitivities.size(1) == V);
    COMPAS_CHECK(data.size(0) == C && data.size(1) == R && data.size(2) == S);
    if (cg_iterations < 1) COMPAS_ERROR("at least one conjugate-gradient iteration is needed");
    if (!std::isfinite(delta)) COMPAS_ERROR("finite-difference step must be finite (0 selects exact derivatives)");
    COMPAS_CHECK(V > 0);

    // the estimate is a private copy of the parameters (updated in place by every iteration)
    Array<float, 2> own({TissueParameterField::NUM_FIELDS, V}, dev, ctx.stream());
    DeviceGuard guard(dev);
    COMPAS_CUDA_CHECK(cudaMemcpy2DAsync(own.data(), size_t(V) * sizeof(float), parameters.data.data(),
                                        size_t(parameters.data.size(1)) * sizeof(float), size_t(V) * sizeof(float),
                                        TissueParameterField::NUM_FIELDS, cudaMemcpyDeviceToDevice, ctx.stream()));
    im.params = TissueParameters(own, parameters.has_z, parameters.has_b0, parameters.has_b1);
    im.perturbed = Array<float, 2>({TissueParameterField::NUM_FIELDS, V}, dev, ctx.stream());
    im.sequence = std::move(sequence);
    im.trajectory = std::move(trajectory);
    im.coils = std::move(coil_sensitivities);
    im.data = std::move(data);
    im.cg_iterations = cg_iterations;
    im.delta = delta;
    im.prec = (method == JacobianComputeMethod::GemmFast || method == JacobianComputeMethod::GemmLow)
                  ? Precision::SplitBF16
                  : Precision::FP32;
    im.echos = Array<cfloat, 2>({R, V}, dev, ctx.stream());
    im.dT1 = Array<cfloat, 2>({R, V}, dev, ctx.stream());
    im.dT2 = Array<cfloat, 2>({R, V}, dev, ctx.stream());
    im.signal = Array<cfloat, 3>({C, R, S}, dev, ctx.stream());
    im.b = Array<cfloat, 3>({C, R, S}, dev, ctx.stream());
    im.q = Array<cfloat, 3>({C, R, S}, dev, ctx.stream());
    im.g = Array<cfloat, 2>({4, V}, dev, ctx.stream());
    im.d = Array<cfloat, 2>({4, V}, dev, ctx.stream());
    im.x = Array<float, 2>({4, V}, dev, ctx.stream());
    im.scalars = Array<float>({kernels::kNumScalars}, dev, ctx.stream());
    im.handoff = Array<int>({Impl::kHandoffCapacity}, dev, ctx.stream());
    im.trial = Array<float, 2>({TissueParameterField::NUM_FIELDS, V}, dev, ctx.stream());
    COMPAS_CUDA_CHECK(cudaMemcpyAsync(im.trial.data(), own.data(), own.nbytes(), cudaMemcpyDeviceToDevice,
                                      ctx.stream()));
    im.trial_echos = Array<cfloat, 2>({R, V}, dev, ctx.stream());
    im.trial_signal = Array<cfloat, 3>({C, R, S}, dev, ctx.stream());
    im.flags = Array<int>({kernels::kNumFlags}, dev, ctx.stream());
    COMPAS_CUDA_CHECK(cudaMemsetAsync(im.flags.data(), 0, im.flags.nbytes(), ctx.stream()));
    im.npartials = residual_partial_count(im.signal.numel());
    im.partials = Array<float>({std::max(im.npartials, kernels::kRedBlocks)}, dev, ctx.stream());
    COMPAS_CUDA_CHECK(cudaMemsetAsync(im.scalars.data(), 0, im.scalars.nbytes(), ctx.stream()));
    // build the sequence's device table now, so that no capture ever contains its construction
    if (const auto* f = std::get_if<FISPSequence>(&im.sequence)) (void)fisp_excite_table(ctx, *f);
    else (void)pssfp_args(ctx, im.params, 0, V, std::get<pSSFPSequence>(im.sequence), im.echos.data(), V);
    ctx.synchronize();
}

void GaussNewtonStep::run(bool use_graph) {
    Impl& im = *m_impl;
    DeviceGuard guard(im.ctx.device());
    if (!use_graph) {
        im.enqueue();
        return;
    }
    if (!im.exec) {
        cudaStream_t st = im.ctx.stream();
        COMPAS_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        try {
            im.enqueue();
        } catch (...) {
            cudaGraph_t partial = nullptr;
            cudaStreamEndCapture(st, &partial);
            if (partial) cudaGraphDestroy(partial);
            throw;
        }
        COMPAS_CUDA_CHECK(cudaStreamEndCapture(st, &im.graph));
        COMPAS_CUDA_CHECK(cudaGraphInstantiate(&im.exec, im.graph, 0));
    }
    COMPAS_CUDA_CHECK(cudaGraphLaunch(im.exec, im.ctx.stream()));
}

void GaussNewtonStep::set_line_search(bool on) {
    Impl& im = *m_impl;
    if (im.line_search == on) return;
    im.ctx.synchronize();
    if (im.exec) cudaGraphExecDestroy(im.exec);
    if (im.graph) cudaGraphDestroy(im.graph);
    im.exec = nullptr;
    im.graph = nullptr;
    im.line_search = on;
    // the estimate's echoes are simulated again on the next run
    DeviceGuard guard(im.ctx.device());
    COMPAS_CUDA_CHECK(cudaMemsetAsync(im.flags.data(), 0, im.flags.nbytes(), im.ctx.stream()));
}

bool GaussNewtonStep::line_search() const {
    return m_impl->line_search;
}

int GaussNewtonStep::kernels_per_iteration() const {
    // counted by capturing: nodes of the instantiated graph that are kernels
    const Impl& im = *m_impl;
    if (!im.graph) return -1;
    size_t n = 0;
    COMPAS_CUDA_CHECK(cudaGraphGetNodes(im.graph, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    COMPAS_CUDA_CHECK(cudaGraphGetNodes(im.graph, nodes.data(), &n));
    int k = 0;
    for (auto node : nodes) {
        cudaGraphNodeType t;
        COMPAS_CUDA_CHECK(cudaGraphNodeGetType(node, &t));
        if (t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

const TissueParameters& GaussNewtonStep::parameters() const {
    return m_impl->params;
}
const Array<cfloat, 2>& GaussNewtonStep::echos() const {
    return m_impl->echos;
}
const Array<cfloat, 2>& GaussNewtonStep::derivative(int field) const {
    if (field == TissueParameterField::T1) return m_impl->dT1;
    if (field == TissueParameterField::T2) return m_impl->dT2;
    COMPAS_ERROR("derivatives are kept for T1 and T2 only");
}
const Array<cfloat, 3>& GaussNewtonStep::signal() const {
    return m_impl->signal;
}
const Array<cfloat, 2>& GaussNewtonStep::gradient() const {
    return m_impl->g;
}
const Array<float, 2>& GaussNewtonStep::step() const {
    return m_impl->x;
}
const Array<float>& GaussNewtonStep::scalars() const {
    return m_impl->scalars;
}

}  // namespace compas
