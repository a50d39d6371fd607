// capi.cpp — the extern "C" boundary (include/compas_b200.h).
//
// Same symbols and parameter lists as the reference's Julia binding library
// (julia-bindings/src/bindings.cpp:19-411). Handles are heap objects derived from
// compas::Object; arrays are compas::Array<T, N>. Exceptions never cross the boundary:
// they are turned into a Julia error when jl_errorf is resolvable in the process (the
// reference's behaviour, julia-bindings/src/common.h:48-62) and otherwise recorded for
// compas_last_error() while the call returns NULL.
#include <dlfcn.h>

#include <cstring>
#include <string>

#include "../../include/compas_b200.h"
#include "compas/compas.h"
#include "kernels.h"

#ifndef COMPAS_B200_VERSION
#define COMPAS_B200_VERSION "compas-b200-0.1.0"
#endif

using compas::cfloat;

namespace {

thread_local std::string t_last_error;
thread_local bool t_has_error = false;

using jl_errorf_t = void (*)(const char*, ...);

jl_errorf_t julia_error_fn() {
    static jl_errorf_t fn = reinterpret_cast<jl_errorf_t>(dlsym(RTLD_DEFAULT, "jl_errorf"));
    return fn;
}

void record_error(const char* msg) {
    t_last_error = msg;
    t_has_error = true;
    if (auto fn = julia_error_fn()) {
        fn("COMPAS error occurred: %s\n", msg);  // does not return
    }
}

template<typename F>
auto guarded(F fun) -> decltype(fun()) {
    t_has_error = false;
    try {
        return fun();
    } catch (const std::exception& e) {
        record_error(e.what());
    } catch (...) {
        record_error("unknown exception");
    }
    using R = decltype(fun());
    if constexpr (std::is_void_v<R>) {
        return;
    } else {
        return R {};
    }
}

template<typename T>
T* handle(const void* p) {
    return reinterpret_cast<T*>(const_cast<void*>(p));
}

const compas::CompasContext& ctx_of(const compas_context* c) {
    if (!c) throw compas::CompasException("null context");
    return *handle<compas::CompasContext>(c);
}

template<typename T>
const T& unwrap(const void* obj) {
    if (!obj) throw compas::CompasException("null object handle");
    const auto* base = handle<compas::Object>(obj);
    if (const T* p = dynamic_cast<const T*>(base)) return *p;
    throw compas::CompasException(std::string("invalid object (expecting: ") + typeid(T).name() +
                                  ", gotten: " + base->name() + ")");
}

template<typename T, size_t N>
const compas::Array<T, N>& array_of(const void* arr, const char* what) {
    if (!arr) throw compas::CompasException(std::string("null array: ") + what);
    const auto* base = handle<compas::Object>(arr);
    if (const auto* p = dynamic_cast<const compas::Array<T, N>*>(base)) return *p;
    throw compas::CompasException(std::string("array `") + what + "` has the wrong element type or rank");
}

template<typename T>
compas_array* new_array(T&& a) {
    return reinterpret_cast<compas_array*>(static_cast<compas::Object*>(new std::decay_t<T>(std::forward<T>(a))));
}

template<typename T>
compas_object* new_obj(T&& a) {
    return reinterpret_cast<compas_object*>(static_cast<compas::Object*>(new std::decay_t<T>(std::forward<T>(a))));
}

template<typename T>
const compas_array* make_array(const compas_context* context, const T* data, int rank, int64_t* sizes) {
    const auto& ctx = ctx_of(context);
    if (!sizes) throw compas::CompasException("null sizes");
    for (int i = 0; i < rank; i++)
        if (sizes[i] < 0) throw compas::CompasException("negative array size");
    int64_t n = 1;
    for (int i = 0; i < rank; i++) n *= sizes[i];
    if (n > 0 && !data) throw compas::CompasException("null data pointer");
    if (rank == 1) return new_array(ctx.allocate(data, sizes[0]));
    if (rank == 2) return new_array(ctx.allocate(data, sizes[0], sizes[1]));
    if (rank == 3) return new_array(ctx.allocate(data, sizes[0], sizes[1], sizes[2]));
    throw compas::CompasException("cannot support rank > 3");
}

void read_array(const compas_array* arr, void* dest, int64_t length, size_t elem) {
    if (!arr) throw compas::CompasException("null array");
    const auto* base = dynamic_cast<const compas::ArrayBase*>(handle<compas::Object>(arr));
    if (!base) throw compas::CompasException("handle is not an array");
    if (base->element_size() != elem) throw compas::CompasException("array element type mismatch");
    if (length < 0) throw compas::CompasException("negative length");
    if (length > 0 && !dest) throw compas::CompasException("null destination");
    base->copy_bytes_to(dest, size_t(length) * elem);
}

// calls fn with the Cartesian or spiral trajectory behind `obj` (the Jacobians accept both here;
// the reference's accept Cartesian only)
template<typename F>
auto with_trajectory(const void* obj, F fn) {
    if (!obj) throw compas::CompasException("null trajectory");
    const auto* base = handle<compas::Object>(obj);
    if (const auto* c = dynamic_cast<const compas::CartesianTrajectory*>(base)) return fn(*c);
    if (const auto* s = dynamic_cast<const compas::SpiralTrajectory*>(base)) return fn(*s);
    throw compas::CompasException(std::string("invalid trajectory object: ") + base->name());
}

compas::SimulateSignalMethod signal_method(int m) {
    if (m < 0 || m > 5) throw compas::CompasException("invalid SimulateSignalMethod");
    return compas::SimulateSignalMethod(m);
}

compas::JacobianComputeMethod jacobian_method(int m) {
    if (m < 0 || m > 4) throw compas::CompasException("invalid JacobianComputeMethod");
    return compas::JacobianComputeMethod(m);
}

compas::GemmComputeMethod gemm_method(int m) {
    if (m < 0 || m > 2) throw compas::CompasException("invalid GemmComputeMethod");
    return compas::GemmComputeMethod(m);
}

template<typename T, size_t N>
compas::Array<T, N>* mutable_array_of(compas_array* arr, const char* what) {
    if (!arr) throw compas::CompasException(std::string("null array: ") + what);
    if (auto* p = dynamic_cast<compas::Array<T, N>*>(handle<compas::Object>(arr))) return p;
    throw compas::CompasException(std::string("array `") + what + "` has the wrong element type or rank");
}

template<typename T, size_t N>
const compas::Array<T, N>* maybe_array(const compas_array* arr) {
    return arr ? dynamic_cast<const compas::Array<T, N>*>(handle<compas::Object>(arr)) : nullptr;
}

}  // namespace

namespace compas {
void residual_noalloc(int device, const cfloat* lhs, const cfloat* rhs, cfloat* diff, float* objective, int64_t n,
                      cudaStream_t stream);
unsigned long long launch_count();
void set_fisp_override(int config, int warps);
void set_pssfp_override(int config);
void set_fisp_tangent_override(int config);
void set_tc_override(int kind, int tile, int splits);
}  // namespace compas

extern "C" {

const char* compas_version(void) {
    return COMPAS_B200_VERSION;
}

const char* compas_last_error(void) {
    return t_has_error ? t_last_error.c_str() : nullptr;
}

const compas_context* compas_make_context(void) {
    return guarded([&]() -> const compas_context* {
        return reinterpret_cast<const compas_context*>(new compas::CompasContext(compas::make_context()));
    });
}

const compas_context* compas_copy_context_for_device(compas_context* ctx, int device) {
    return guarded([&]() -> const compas_context* {
        return reinterpret_cast<const compas_context*>(new compas::CompasContext(ctx_of(ctx).with_device(device)));
    });
}

void compas_destroy_context(const compas_context* ctx) {
    guarded([&] { delete handle<compas::CompasContext>(ctx); });
}

void compas_destroy_object(const compas_object* obj) {
    guarded([&] { delete handle<compas::Object>(obj); });
}

void compas_synchronize(const compas_context* ctx) {
    guarded([&] { ctx_of(ctx).synchronize(); });
}

const compas_array* compas_make_array_float(const compas_context* context, const float* data, int rank,
                                            int64_t* sizes) {
    return guarded([&] { return make_array(context, data, rank, sizes); });
}

void compas_read_array_float(const compas_context*, const compas_array* array, float* dest, int64_t length) {
    guarded([&] { read_array(array, dest, length, sizeof(float)); });
}

const compas_array* compas_make_array_complex(const compas_context* context, const compas_cfloat* data, int rank,
                                              int64_t* sizes) {
    return guarded([&] { return make_array(context, reinterpret_cast<const cfloat*>(data), rank, sizes); });
}

void compas_read_array_complex(const compas_context*, const compas_array* array, compas_cfloat* dest,
                               int64_t length) {
    guarded([&] { read_array(array, dest, length, sizeof(cfloat)); });
}

void compas_destroy_array(const compas_array* array) {
    guarded([&] { delete handle<compas::Object>(array); });
}

const compas_object* compas_make_tissue_parameters(const compas_context* context, int nvoxels, const float* T1,
                                                   const float* T2, const float* B1, const float* B0,
                                                   const float* rho_x, const float* rho_y, const float* x,
                                                   const float* y, const float* z) {
    return guarded([&]() -> const compas_object* {
        if (nvoxels < 0) throw compas::CompasException("negative voxel count");
        auto view = [&](const float* p) { return compas::View<float>(p, {p ? nvoxels : 0}); };
        return new_obj(compas::make_tissue_parameters(ctx_of(context), nvoxels, nvoxels, view(T1), view(T2),
                                                      view(B1), view(B0), view(rho_x), view(rho_y), view(x),
                                                      view(y), view(z)));
    });
}

namespace {

// bindings.cpp:151-174 with the C++ sequence's two flags (compas/sequences/fisp.h:37-41)
compas_object* make_fisp(const compas_array* RF_train, const compas_array* sliceprofiles, float TR, float TE, float TW,
                         int max_state, float TI, int undersampling_factor, int repetitions, bool inversion_prepulse,
                         bool wait_spoiling) {
    const auto& rf = array_of<cfloat, 1>(RF_train, "RF_train");
    const auto& sp = array_of<cfloat, 2>(sliceprofiles, "sliceprofiles");
    if (sp.size(1) != rf.size(0)) throw compas::CompasException("sliceprofiles must be [npositions][nTR]");
    if (max_state < 1 || max_state > 128) throw compas::CompasException("max_state must be in [1, 128]");
    if (undersampling_factor < 1 || repetitions < 1)
        throw compas::CompasException("undersampling_factor and repetitions must be >= 1");
    return new_obj(compas::FISPSequence(rf, sp, TR, TE, TW, max_state, TI, undersampling_factor, repetitions,
                                        inversion_prepulse, wait_spoiling));
}

}  // namespace

compas_object* compas_make_fisp_sequence(const compas_array* RF_train, const compas_array* sliceprofiles, float TR,
                                         float TE, float TW, int max_state, float TI, int undersampling_factor,
                                         int repetitions) {
    return guarded([&]() -> compas_object* {
        return make_fisp(RF_train, sliceprofiles, TR, TE, TW, max_state, TI, undersampling_factor, repetitions, true,
                         true);
    });
}

compas_object* compas_b200_make_fisp_sequence_ex(const compas_array* RF_train, const compas_array* sliceprofiles,
                                                float TR, float TE, float TW, int max_state, float TI,
                                                int undersampling_factor, int repetitions, int inversion_prepulse,
                                                int wait_spoiling) {
    return guarded([&]() -> compas_object* {
        return make_fisp(RF_train, sliceprofiles, TR, TE, TW, max_state, TI, undersampling_factor, repetitions,
                         inversion_prepulse != 0, wait_spoiling != 0);
    });
}

compas_object* compas_make_pssfp_sequence(const compas_array* RF_train, float TR, const compas_array* gamma_dt_RF,
                                          float dt_ex, float dt_inv, float dt_pr, float gamma_dt_GRz_ex,
                                          float gamma_dt_GRz_inv, float gamma_dt_GRz_pr, const compas_array* z) {
    return guarded([&]() -> compas_object* {
        const auto& rf = array_of<cfloat, 1>(RF_train, "RF_train");
        const auto& g = array_of<cfloat, 1>(gamma_dt_RF, "gamma_dt_RF");
        const auto& zz = array_of<float, 1>(z, "z");
        if (rf.size() == 0) throw compas::CompasException("empty RF train");
        return new_obj(compas::pSSFPSequence(rf, TR, g, compas::RepetitionData {dt_ex, dt_inv, dt_pr},
                                             compas::RepetitionData {gamma_dt_GRz_ex, gamma_dt_GRz_inv,
                                                                     gamma_dt_GRz_pr},
                                             zz));
    });
}

compas_object* compas_make_cartesian_trajectory(int nreadouts, int samples_per_readout, float delta_t,
                                                compas_array* k_start, float delta_k) {
    return guarded([&]() -> compas_object* {
        const auto& ks = array_of<cfloat, 1>(k_start, "k_start");
        if (ks.size() != nreadouts) throw compas::CompasException("k_start must have nreadouts entries");
        if (nreadouts < 0 || samples_per_readout < 0) throw compas::CompasException("negative trajectory size");
        return new_obj(compas::CartesianTrajectory(nreadouts, samples_per_readout, delta_t, ks, cfloat(delta_k, 0)));
    });
}

compas_object* compas_make_spiral_trajectory(int nreadouts, int samples_per_readout, float delta_t,
                                             compas_array* k_start, compas_array* delta_k) {
    return guarded([&]() -> compas_object* {
        const auto& ks = array_of<cfloat, 1>(k_start, "k_start");
        const auto& dk = array_of<cfloat, 1>(delta_k, "delta_k");
        if (ks.size() != nreadouts || dk.size() != nreadouts)
            throw compas::CompasException("k_start and delta_k must have nreadouts entries");
        if (nreadouts < 0 || samples_per_readout < 0) throw compas::CompasException("negative trajectory size");
        return new_obj(compas::SpiralTrajectory(nreadouts, samples_per_readout, delta_t, ks, dk));
    });
}

compas_array* compas_simulate_magnetization_fisp(const compas_context* ctx, const compas_object* parameters,
                                                 const compas_object* sequence) {
    return guarded([&] {
        return new_array(compas::simulate_magnetization(ctx_of(ctx), unwrap<compas::TissueParameters>(parameters),
                                                        unwrap<compas::FISPSequence>(sequence)));
    });
}

compas_array* compas_simulate_magnetization_pssfp(const compas_context* ctx, const compas_object* parameters,
                                                  const compas_object* sequence) {
    return guarded([&] {
        return new_array(compas::simulate_magnetization(ctx_of(ctx), unwrap<compas::TissueParameters>(parameters),
                                                        unwrap<compas::pSSFPSequence>(sequence)));
    });
}

compas_array* compas_magnetization_to_signal_cartesian(const compas_context* ctx, int ncoils,
                                                       const compas_array* echos, const compas_object* parameters,
                                                       const compas_array* coils, const compas_object* trajectory,
                                                       int32_t low_precision) {
    return guarded([&] {
        const auto& co = array_of<cfloat, 2>(coils, "coils");
        if (co.size(0) != ncoils) throw compas::CompasException("ncoils does not match the coil array");
        auto method = low_precision == 0 ? compas::SimulateSignalMethod::MatmulFast
                                         : compas::SimulateSignalMethod::MatmulLow;
        return new_array(compas::magnetization_to_signal(
            ctx_of(ctx), array_of<cfloat, 2>(echos, "echos"), unwrap<compas::TissueParameters>(parameters),
            unwrap<compas::CartesianTrajectory>(trajectory), co, method));
    });
}

compas_array* compas_magnetization_to_signal_spiral(const compas_context* ctx, int ncoils, const compas_array* echos,
                                                    const compas_object* parameters, const compas_array* coils,
                                                    const compas_object* trajectory) {
    return guarded([&] {
        const auto& co = array_of<cfloat, 2>(coils, "coils");
        if (co.size(0) != ncoils) throw compas::CompasException("ncoils does not match the coil array");
        return new_array(compas::magnetization_to_signal(ctx_of(ctx), array_of<cfloat, 2>(echos, "echos"),
                                                         unwrap<compas::TissueParameters>(parameters),
                                                         unwrap<compas::SpiralTrajectory>(trajectory), co));
    });
}

compas_array* compas_compute_jacobian(const compas_context* ctx, int ncoils, const compas_array* echos,
                                      const compas_array* delta_echos_T1, const compas_array* delta_echos_T2,
                                      const compas_object* parameters, const compas_array* coils,
                                      const compas_object* trajectory, const compas_array* vector,
                                      const int32_t low_precision) {
    return guarded([&] {
        const auto& co = array_of<cfloat, 2>(coils, "coils");
        if (co.size(0) != ncoils) throw compas::CompasException("ncoils does not match the coil array");
        auto method =
            low_precision == 0 ? compas::JacobianComputeMethod::GemmFast : compas::JacobianComputeMethod::GemmLow;
        return with_trajectory(trajectory, [&](const auto& traj) {
            return new_array(compas::compute_jacobian(
                ctx_of(ctx), array_of<cfloat, 2>(echos, "echos"),
                array_of<cfloat, 2>(delta_echos_T1, "delta_echos_T1"),
                array_of<cfloat, 2>(delta_echos_T2, "delta_echos_T2"), unwrap<compas::TissueParameters>(parameters),
                traj, co, array_of<cfloat, 2>(vector, "vector"), method));
        });
    });
}

compas_array* compas_compute_jacobian_hermitian(const compas_context* ctx, int ncoils, const compas_array* echos,
                                                const compas_array* delta_echos_T1,
                                                const compas_array* delta_echos_T2, const compas_object* parameters,
                                                const compas_object* trajectory, const compas_array* coils,
                                                const compas_array* vector, const int32_t low_precision) {
    return guarded([&] {
        const auto& co = array_of<cfloat, 2>(coils, "coils");
        if (co.size(0) != ncoils) throw compas::CompasException("ncoils does not match the coil array");
        auto method =
            low_precision == 0 ? compas::JacobianComputeMethod::GemmFast : compas::JacobianComputeMethod::GemmLow;
        return with_trajectory(trajectory, [&](const auto& traj) {
            return new_array(compas::compute_jacobian_hermitian(
                ctx_of(ctx), array_of<cfloat, 2>(echos, "echos"),
                array_of<cfloat, 2>(delta_echos_T1, "delta_echos_T1"),
                array_of<cfloat, 2>(delta_echos_T2, "delta_echos_T2"), unwrap<compas::TissueParameters>(parameters),
                traj, co, array_of<cfloat, 3>(vector, "vector"), method));
        });
    });
}

compas_array* phase_encoding(const compas_context* ctx, const compas_array* echos, const compas_object* parameters,
                             const compas_object* trajectory) {
    return guarded([&] {
        return new_array(compas::phase_encoding(ctx_of(ctx), array_of<cfloat, 2>(echos, "echos"),
                                                unwrap<compas::TissueParameters>(parameters),
                                                unwrap<compas::CartesianTrajectory>(trajectory)));
    });
}

compas_array* compas_compute_residual(const compas_context* ctx, const compas_array* lhs, const compas_array* rhs,
                                      float* sum) {
    return guarded([&] {
        return new_array(compas::compute_residual(ctx_of(ctx), array_of<cfloat, 3>(lhs, "lhs"),
                                                  array_of<cfloat, 3>(rhs, "rhs"), sum));
    });
}

compas_array* compas_simulate_magnetization_derivative_pssfp(const compas_context* ctx, int field,
                                                             const compas_array* echos,
                                                             const compas_object* parameters, float delta,
                                                             const compas_object* sequence) {
    return guarded([&] {
        return new_array(compas::simulate_magnetization_derivative(
            ctx_of(ctx), field, array_of<cfloat, 2>(echos, "echos"), unwrap<compas::TissueParameters>(parameters),
            unwrap<compas::pSSFPSequence>(sequence), delta));
    });
}

compas_array* compas_simulate_magnetization_derivative_fisp(const compas_context* ctx, int field,
                                                            const compas_array* echos, const compas_object* parameters,
                                                            float delta, const compas_object* sequence) {
    return guarded([&] {
        return new_array(compas::simulate_magnetization_derivative(
            ctx_of(ctx), field, array_of<cfloat, 2>(echos, "echos"), unwrap<compas::TissueParameters>(parameters),
            unwrap<compas::FISPSequence>(sequence), delta));
    });
}

int compas_b200_simulate_magnetization_tangents(const compas_context* ctx, const compas_object* parameters,
                                                const compas_object* sequence, compas_array** echos,
                                                compas_array** delta_echos_T1, compas_array** delta_echos_T2) {
    t_has_error = false;
    guarded([&] {
        if (!echos || !delta_echos_T1 || !delta_echos_T2) throw compas::CompasException("null output pointer");
        if (!sequence) throw compas::CompasException("null object handle");
        const auto& params = unwrap<compas::TissueParameters>(parameters);
        const auto* seq = handle<compas::Object>(sequence);
        compas::MagnetizationTangents t;
        if (const auto* fisp = dynamic_cast<const compas::FISPSequence*>(seq))
            t = compas::simulate_magnetization_tangents(ctx_of(ctx), params, *fisp);
        else
            t = compas::simulate_magnetization_tangents(ctx_of(ctx), params, unwrap<compas::pSSFPSequence>(sequence));
        *echos = new_array(std::move(t.echos));
        *delta_echos_T1 = new_array(std::move(t.dT1));
        *delta_echos_T2 = new_array(std::move(t.dT2));
    });
    return t_has_error ? -1 : 0;
}

compas_array* compas_b200_magnetization_to_signal(const compas_context* ctx, const compas_array* echos,
                                                  const compas_object* parameters, const compas_object* trajectory,
                                                  const compas_array* coils, int method) {
    return guarded([&] {
        if (!trajectory) throw compas::CompasException("null trajectory");
        return new_array(compas::magnetization_to_signal(
            ctx_of(ctx), array_of<cfloat, 2>(echos, "echos"), unwrap<compas::TissueParameters>(parameters),
            unwrap<compas::Trajectory>(trajectory), array_of<cfloat, 2>(coils, "coils"), signal_method(method)));
    });
}

compas_array* compas_b200_compute_jacobian(const compas_context* ctx, const compas_array* echos,
                                           const compas_array* delta_echos_T1, const compas_array* delta_echos_T2,
                                           const compas_object* parameters, const compas_object* trajectory,
                                           const compas_array* coils, const compas_array* vector, int method) {
    return guarded([&] {
        return with_trajectory(trajectory, [&](const auto& traj) {
            return new_array(compas::compute_jacobian(
                ctx_of(ctx), array_of<cfloat, 2>(echos, "echos"),
                array_of<cfloat, 2>(delta_echos_T1, "delta_echos_T1"),
                array_of<cfloat, 2>(delta_echos_T2, "delta_echos_T2"), unwrap<compas::TissueParameters>(parameters),
                traj, array_of<cfloat, 2>(coils, "coils"), array_of<cfloat, 2>(vector, "vector"),
                jacobian_method(method)));
        });
    });
}

int compas_b200_compute_gemm(const compas_context* ctx, compas_array* result, const compas_array* lhs,
                             const compas_array* rhs, float alpha, float beta, int method) {
    t_has_error = false;
    guarded([&] {
        auto& out = *mutable_array_of<float, 2>(result, "result");
        if (const auto* l = maybe_array<compas::bfloat16, 2>(lhs)) {
            compas::compute_gemm(ctx_of(ctx), out, *l, array_of<compas::bfloat16, 2>(rhs, "rhs"), alpha, beta,
                                 gemm_method(method));
        } else {
            compas::compute_gemm(ctx_of(ctx), out, array_of<float, 2>(lhs, "lhs"), array_of<float, 2>(rhs, "rhs"),
                                 alpha, beta, gemm_method(method));
        }
    });
    return t_has_error ? -1 : 0;
}

int compas_b200_compute_complex_gemm(const compas_context* ctx, compas_array* result, const compas_array* lhs,
                                     const compas_array* rhs, float alpha, float beta, int method) {
    t_has_error = false;
    guarded([&] {
        auto& out = *mutable_array_of<float, 3>(result, "result");
        if (const auto* l = maybe_array<compas::bfloat16, 3>(lhs)) {
            compas::compute_complex_gemm(ctx_of(ctx), out, *l, array_of<compas::bfloat16, 3>(rhs, "rhs"), alpha, beta,
                                         gemm_method(method));
        } else {
            compas::compute_complex_gemm(ctx_of(ctx), out, array_of<float, 3>(lhs, "lhs"),
                                         array_of<float, 3>(rhs, "rhs"), alpha, beta, gemm_method(method));
        }
    });
    return t_has_error ? -1 : 0;
}

int compas_b200_convert_complex_to_planar(const compas_context* ctx, compas_array* output, const compas_array* input) {
    t_has_error = false;
    guarded([&] {
        const auto& in = array_of<cfloat, 2>(input, "input");
        if (auto* o = output ? dynamic_cast<compas::Array<compas::bfloat16, 3>*>(handle<compas::Object>(output))
                             : nullptr) {
            compas::convert_complex_to_planar(ctx_of(ctx), *o, in);
        } else {
            compas::convert_complex_to_planar(ctx_of(ctx), *mutable_array_of<float, 3>(output, "output"), in);
        }
    });
    return t_has_error ? -1 : 0;
}

int compas_b200_convert_planar_to_complex(const compas_context* ctx, compas_array* output, const compas_array* input) {
    t_has_error = false;
    guarded([&] {
        compas::convert_planar_to_complex(ctx_of(ctx), *mutable_array_of<cfloat, 2>(output, "output"),
                                          array_of<float, 3>(input, "input"));
    });
    return t_has_error ? -1 : 0;
}

const compas_array* compas_b200_make_array_bfloat16(const compas_context* context, const uint16_t* data, int rank,
                                                    int64_t* sizes) {
    return guarded([&] { return make_array(context, reinterpret_cast<const compas::bfloat16*>(data), rank, sizes); });
}

void compas_b200_read_array_bfloat16(const compas_context*, const compas_array* array, uint16_t* dest,
                                     int64_t length) {
    guarded([&] { read_array(array, dest, length, sizeof(uint16_t)); });
}

int compas_b200_voxel_shard(int64_t nvoxels, int rank, int world, int64_t* begin, int64_t* end) {
    t_has_error = false;
    guarded([&] {
        if (!begin || !end) throw compas::CompasException("null output pointer");
        const compas::VoxelRange r = compas::voxel_shard(nvoxels, rank, world);
        *begin = r.begin;
        *end = r.end;
    });
    return t_has_error ? -1 : 0;
}

int compas_b200_comm_unique_id(char* out, int nbytes) {
    t_has_error = false;
    const int n = guarded([&] {
        const std::vector<char> id = compas::Communicator::unique_id();
        if (!out || nbytes < int(id.size())) throw compas::CompasException("the unique id needs 128 bytes");
        std::memcpy(out, id.data(), id.size());
        return int(id.size());
    });
    return t_has_error ? -1 : n;
}

compas_object* compas_b200_make_communicator(const compas_context* ctx, int rank, int world, const char* unique_id) {
    return guarded([&]() -> compas_object* {
        if (!unique_id) throw compas::CompasException("null unique id");
        return new_obj(compas::Communicator(ctx_of(ctx), rank, world, std::vector<char>(unique_id, unique_id + 128)));
    });
}

int compas_b200_allreduce_sum(const compas_context* ctx, const compas_object* comm, compas_array* array) {
    t_has_error = false;
    guarded([&] {
        if (!array) throw compas::CompasException("null array");
        const auto* base = dynamic_cast<const compas::ArrayBase*>(handle<compas::Object>(array));
        if (!base) throw compas::CompasException("handle is not an array");
        if (base->element_size() != sizeof(float) && base->element_size() != 2 * sizeof(float))
            throw compas::CompasException("all-reduce of a float or complex array only");
        unwrap<compas::Communicator>(comm).allreduce_sum(ctx_of(ctx), static_cast<float*>(base->raw_data()),
                                                         int64_t(base->nbytes() / sizeof(float)));
    });
    return t_has_error ? -1 : 0;
}

compas_array* compas_b200_magnetization_to_signal_sharded(const compas_context* ctx, const compas_object* comm,
                                                          const compas_array* echos, const compas_object* parameters,
                                                          const compas_object* trajectory, const compas_array* coils,
                                                          int method) {
    return guarded([&] {
        return with_trajectory(trajectory, [&](const auto& traj) {
            return new_array(compas::magnetization_to_signal_sharded(
                ctx_of(ctx), unwrap<compas::Communicator>(comm), array_of<cfloat, 2>(echos, "echos"),
                unwrap<compas::TissueParameters>(parameters), traj, array_of<cfloat, 2>(coils, "coils"),
                signal_method(method)));
        });
    });
}

compas_array* compas_b200_compute_jacobian_sharded(const compas_context* ctx, const compas_object* comm,
                                                   const compas_array* echos, const compas_array* delta_echos_T1,
                                                   const compas_array* delta_echos_T2, const compas_object* parameters,
                                                   const compas_object* trajectory, const compas_array* coils,
                                                   const compas_array* vector, int method) {
    return guarded([&] {
        return with_trajectory(trajectory, [&](const auto& traj) {
            return new_array(compas::compute_jacobian_sharded(
                ctx_of(ctx), unwrap<compas::Communicator>(comm), array_of<cfloat, 2>(echos, "echos"),
                array_of<cfloat, 2>(delta_echos_T1, "delta_echos_T1"),
                array_of<cfloat, 2>(delta_echos_T2, "delta_echos_T2"), unwrap<compas::TissueParameters>(parameters),
                traj, array_of<cfloat, 2>(coils, "coils"), array_of<cfloat, 2>(vector, "vector"),
                jacobian_method(method)));
        });
    });
}

compas_array* compas_b200_compute_jacobian_hermitian(const compas_context* ctx, const compas_array* echos,
                                                     const compas_array* delta_echos_T1,
                                                     const compas_array* delta_echos_T2,
                                                     const compas_object* parameters,
                                                     const compas_object* trajectory, const compas_array* coils,
                                                     const compas_array* vector, int method) {
    return guarded([&] {
        return with_trajectory(trajectory, [&](const auto& traj) {
            return new_array(compas::compute_jacobian_hermitian(
                ctx_of(ctx), array_of<cfloat, 2>(echos, "echos"),
                array_of<cfloat, 2>(delta_echos_T1, "delta_echos_T1"),
                array_of<cfloat, 2>(delta_echos_T2, "delta_echos_T2"), unwrap<compas::TissueParameters>(parameters),
                traj, array_of<cfloat, 2>(coils, "coils"), array_of<cfloat, 3>(vector, "vector"),
                jacobian_method(method)));
        });
    });
}

void* compas_b200_context_stream(const compas_context* ctx) {
    return guarded([&]() -> void* { return reinterpret_cast<void*>(ctx_of(ctx).stream()); });
}

void* compas_b200_array_device_ptr(const compas_array* array) {
    return guarded([&]() -> void* {
        const auto* base = dynamic_cast<const compas::ArrayBase*>(handle<compas::Object>(array));
        if (!base) throw compas::CompasException("handle is not an array");
        return base->raw_data();
    });
}

int compas_b200_array_rank(const compas_array* array) {
    return guarded([&]() -> int {
        const auto* base = dynamic_cast<const compas::ArrayBase*>(handle<compas::Object>(array));
        if (!base) throw compas::CompasException("handle is not an array");
        return base->rank();
    });
}

int64_t compas_b200_array_extent(const compas_array* array, int axis) {
    return guarded([&]() -> int64_t {
        const auto* base = dynamic_cast<const compas::ArrayBase*>(handle<compas::Object>(array));
        if (!base) throw compas::CompasException("handle is not an array");
        if (axis < 0 || axis >= base->rank()) throw compas::CompasException("axis out of range");
        return base->extent(axis);
    });
}

void compas_b200_set_fisp_launch(int config, int warps) {
    guarded([&] { compas::set_fisp_override(config, warps); });
}

void compas_b200_set_fisp_tangent_launch(int config) {
    guarded([&] { compas::set_fisp_tangent_override(config); });
}

int compas_b200_fisp_tangent_config_count(void) {
    return compas::fisp_tangent_config_count();
}

int compas_b200_fisp_tangent_config_info(int index, int* states_per_lane, int* lanes) {
    return compas::fisp_tangent_config_info(index, states_per_lane, lanes) ? 1 : 0;
}

int compas_b200_fisp_tangent_config_packed(int index) {
    return compas::fisp_tangent_config_packed(index) ? 1 : 0;
}

void compas_b200_set_pssfp_launch(int config) {
    guarded([&] { compas::set_pssfp_override(config); });
}

int compas_b200_compute_residual_noalloc(int device, const compas_cfloat* lhs, const compas_cfloat* rhs,
                                         compas_cfloat* diff, float* objective, int64_t n, void* stream) {
    int rc = -1;
    guarded([&] {
        compas::residual_noalloc(device, reinterpret_cast<const cfloat*>(lhs), reinterpret_cast<const cfloat*>(rhs),
                                 reinterpret_cast<cfloat*>(diff), objective, n, reinterpret_cast<cudaStream_t>(stream));
        rc = 0;
    });
    return rc;
}

int compas_b200_wait_probe(const compas_context* ctx, int64_t limit_cycles) {
    t_has_error = false;
    guarded([&] { compas::launch_wait_probe(ctx_of(ctx), (long long)limit_cycles); });
    return t_has_error ? -1 : 0;
}

uint64_t compas_b200_launch_count(void) {
    return compas::launch_count();
}

int compas_b200_fisp_config_count(void) {
    return compas::fisp_config_count();
}

int compas_b200_fisp_config_info(int index, int* states_per_lane, int* lanes) {
    return compas::fisp_config_info(index, states_per_lane, lanes) ? 1 : 0;
}

int compas_b200_fisp_config_packed(int index) {
    return compas::fisp_config_packed(index) ? 1 : 0;
}

int compas_b200_pssfp_config_count(void) {
    return compas::pssfp_config_count();
}

int compas_b200_pssfp_config_info(int index, int* iso_per_lane, int* lanes) {
    return compas::pssfp_config_info(index, iso_per_lane, lanes) ? 1 : 0;
}

int compas_b200_pssfp_config_packed(int index) {
    return compas::pssfp_config_packed(index) ? 1 : 0;
}

void compas_b200_fisp_launch_choice(int max_state, int64_t nvoxels, int npositions, int* config, int* warps) {
    compas::FispLaunch L = compas::tuned_fisp_launch(max_state, nvoxels, npositions);
    if (L.config < 0) L = compas::fisp_default_launch(max_state, nvoxels, npositions);
    if (config) *config = L.config;
    if (warps) *warps = L.warps;
}

int compas_b200_pssfp_launch_choice(int nz, int64_t nvoxels) {
    compas::PssfpLaunch L = compas::tuned_pssfp_launch(nz, nvoxels);
    return L.config < 0 ? compas::pssfp_default_launch(nz, nvoxels).config : L.config;
}

void compas_b200_set_tc_launch(int kind, int tile, int splits) {
    guarded([&] { compas::set_tc_override(kind, tile, splits); });
}

int compas_b200_tc_launch_choice(int kind, int device, int nvoxels, int nreadouts, int samples_per_readout,
                                 int ncoils, int* tile, int* splits) {
    int rc = -1;
    guarded([&] {
        if (kind < 0 || kind >= int(compas::TcKind::Count)) COMPAS_ERROR("tensor-core contraction kind out of range");
        if (nvoxels < 0 || nreadouts < 0 || samples_per_readout < 0 || ncoils < 0) COMPAS_ERROR("negative size");
        const compas::TcTuning t = compas::tc_launch_choice(device, compas::TcKind(kind), nvoxels, nreadouts,
                                                            samples_per_readout, ncoils);
        if (tile) *tile = t.tile;
        if (splits) *splits = t.splits;
        rc = 0;
    });
    return rc;
}

compas_object* compas_b200_make_batch(const compas_context* context, int njobs, const compas_object* const* parameters,
                                      const compas_object* const* sequences, const compas_object* const* trajectories,
                                      const compas_array* const* coils, int method) {
    return compas_b200_make_batch_tangents(context, njobs, parameters, sequences, trajectories, coils, method, nullptr);
}

compas_object* compas_b200_make_batch_tangents(const compas_context* context, int njobs,
                                               const compas_object* const* parameters,
                                               const compas_object* const* sequences,
                                               const compas_object* const* trajectories,
                                               const compas_array* const* coils, int method,
                                               const int32_t* tangents) {
    return guarded([&] {
        const auto& ctx = ctx_of(context);
        if (njobs < 0) throw compas::CompasException("negative job count");
        if (njobs > 0 && (!parameters || !sequences)) throw compas::CompasException("null job arrays");
        std::vector<compas::SimulationJob> jobs;
        jobs.reserve(size_t(njobs));
        for (int i = 0; i < njobs; i++) {
            compas::SimulationJob job;
            job.parameters = unwrap<compas::TissueParameters>(parameters[i]);
            if (!sequences[i]) throw compas::CompasException("null sequence");
            const auto* seq = handle<compas::Object>(sequences[i]);
            if (const auto* f = dynamic_cast<const compas::FISPSequence*>(seq)) job.sequence = *f;
            else if (const auto* p = dynamic_cast<const compas::pSSFPSequence*>(seq)) job.sequence = *p;
            else throw compas::CompasException(std::string("invalid sequence object: ") + seq->name());
            const void* traj = trajectories ? trajectories[i] : nullptr;
            if (traj) {
                const auto* t = handle<compas::Object>(traj);
                if (const auto* c = dynamic_cast<const compas::CartesianTrajectory*>(t)) job.trajectory = *c;
                else if (const auto* sp = dynamic_cast<const compas::SpiralTrajectory*>(t)) job.trajectory = *sp;
                else throw compas::CompasException(std::string("invalid trajectory object: ") + t->name());
                if (!coils) throw compas::CompasException("null coils array");
                job.coil_sensitivities = array_of<cfloat, 2>(coils[i], "coils");
            }
            job.tangents = tangents && tangents[i] != 0;
            jobs.push_back(std::move(job));
        }
        return new_obj(compas::SimulationBatch(ctx, std::move(jobs), signal_method(method)));
    });
}

int compas_b200_batch_run(const compas_object* batch) {
    t_has_error = false;
    guarded([&] { unwrap<compas::SimulationBatch>(batch).run(); });
    return t_has_error ? -1 : 0;
}

compas_array* compas_b200_batch_echos(const compas_object* batch, int job) {
    return guarded([&] { return new_array(compas::Array<cfloat, 2>(unwrap<compas::SimulationBatch>(batch).echos(job))); });
}

compas_object* compas_b200_make_gauss_newton(const compas_context* context, const compas_object* parameters,
                                             const compas_object* sequence, const compas_object* trajectory,
                                             const compas_array* coils, const compas_array* data, int cg_iterations,
                                             float delta, int method) {
    return guarded([&] {
        const auto& ctx = ctx_of(context);
        if (!sequence) throw compas::CompasException("null sequence");
        const auto* seq = handle<compas::Object>(sequence);
        std::variant<compas::FISPSequence, compas::pSSFPSequence> s;
        if (const auto* f = dynamic_cast<const compas::FISPSequence*>(seq)) s = *f;
        else if (const auto* p = dynamic_cast<const compas::pSSFPSequence*>(seq)) s = *p;
        else throw compas::CompasException(std::string("invalid sequence object: ") + seq->name());
        std::variant<compas::CartesianTrajectory, compas::SpiralTrajectory> t =
            with_trajectory(trajectory, [](const auto& traj) {
                return std::variant<compas::CartesianTrajectory, compas::SpiralTrajectory>(traj);
            });
        return new_obj(compas::GaussNewtonStep(ctx, unwrap<compas::TissueParameters>(parameters), s, t,
                                               array_of<cfloat, 2>(coils, "coils"), array_of<cfloat, 3>(data, "data"),
                                               cg_iterations, delta, jacobian_method(method)));
    });
}

int compas_b200_gauss_newton_run(const compas_object* gn, int use_graph) {
    t_has_error = false;
    guarded([&] { const_cast<compas::GaussNewtonStep&>(unwrap<compas::GaussNewtonStep>(gn)).run(use_graph != 0); });
    return t_has_error ? -1 : 0;
}

int compas_b200_gauss_newton_set_line_search(const compas_object* gn, int on) {
    t_has_error = false;
    guarded([&] { const_cast<compas::GaussNewtonStep&>(unwrap<compas::GaussNewtonStep>(gn)).set_line_search(on != 0); });
    return t_has_error ? -1 : 0;
}

compas_array* compas_b200_gauss_newton_array(const compas_object* gn, int which) {
    return guarded([&]() -> compas_array* {
        const auto& g = unwrap<compas::GaussNewtonStep>(gn);
        switch (which) {
            case 0: return new_array(compas::Array<float, 2>(g.parameters().data));
            case 1: return new_array(compas::Array<cfloat, 2>(g.echos()));
            case 2: return new_array(compas::Array<cfloat, 2>(g.derivative(compas::TissueParameterField::T1)));
            case 3: return new_array(compas::Array<cfloat, 2>(g.derivative(compas::TissueParameterField::T2)));
            case 4: return new_array(compas::Array<cfloat, 3>(g.signal()));
            case 5: return new_array(compas::Array<cfloat, 2>(g.gradient()));
            case 6: return new_array(compas::Array<float, 2>(g.step()));
            case 7: return new_array(compas::Array<float>(g.scalars()));
            default: throw compas::CompasException("invalid Gauss-Newton array index");
        }
    });
}

namespace {
compas::ServeEngine& server_of(const compas_object* server) {
    return const_cast<compas::ServeEngine&>(unwrap<compas::ServeEngine>(server));
}
}  // namespace

compas_object* compas_b200_make_server(const compas_context* context, double memory_budget_gb,
                                       int max_inflight_batches, int max_batch_requests, double echo_cache_gb,
                                       int method, float delta) {
    return guarded([&] {
        if (!(memory_budget_gb > 0) || echo_cache_gb < 0) throw compas::CompasException("invalid memory budget");
        compas::ServeOptions o;
        o.memory_budget_bytes = size_t(memory_budget_gb * double(size_t(1) << 30));
        o.max_inflight_batches = max_inflight_batches;
        o.max_batch_requests = max_batch_requests;
        o.echo_cache_bytes = size_t(echo_cache_gb * double(size_t(1) << 30));
        o.method = signal_method(method);
        o.delta = delta;
        return new_obj(compas::ServeEngine(ctx_of(context), o));
    });
}

int64_t compas_b200_server_submit(const compas_object* server, const compas_object* parameters,
                                  const compas_object* sequence, const compas_object* trajectory,
                                  const compas_array* coils, const compas_array* data, uint64_t echo_key) {
    return compas_b200_server_submit_flags(server, parameters, sequence, trajectory, coils, data, echo_key, 0);
}

int64_t compas_b200_server_submit_flags(const compas_object* server, const compas_object* parameters,
                                        const compas_object* sequence, const compas_object* trajectory,
                                        const compas_array* coils, const compas_array* data, uint64_t echo_key,
                                        int flags) {
    t_has_error = false;
    const int64_t id = guarded([&]() -> int64_t {
        compas::ServeRequest r;
        r.parameters = unwrap<compas::TissueParameters>(parameters);
        if (!sequence) throw compas::CompasException("null sequence");
        const auto* seq = handle<compas::Object>(sequence);
        if (const auto* f = dynamic_cast<const compas::FISPSequence*>(seq)) r.sequence = *f;
        else if (const auto* p = dynamic_cast<const compas::pSSFPSequence*>(seq)) r.sequence = *p;
        else throw compas::CompasException(std::string("invalid sequence object: ") + seq->name());
        if (!trajectory) throw compas::CompasException("null trajectory");
        const auto* t = handle<compas::Object>(trajectory);
        if (const auto* c = dynamic_cast<const compas::CartesianTrajectory*>(t)) r.trajectory = *c;
        else if (const auto* sp = dynamic_cast<const compas::SpiralTrajectory*>(t)) r.trajectory = *sp;
        else throw compas::CompasException(std::string("invalid trajectory object: ") + t->name());
        r.coil_sensitivities = array_of<cfloat, 2>(coils, "coils");
        r.data = array_of<cfloat, 3>(data, "data");
        r.echo_key = echo_key;
        r.inject_wait_timeout = (flags & COMPAS_B200_REQUEST_INJECT_WAIT_TIMEOUT) != 0;
        return int64_t(server_of(server).submit(std::move(r)));
    });
    return t_has_error ? -1 : id;
}

int compas_b200_server_wait(const compas_object* server, int64_t ticket, float* objective, double* times, int* batch) {
    t_has_error = false;
    guarded([&] {
        const compas::ServeResult r = server_of(server).wait(uint64_t(ticket));
        if (objective) *objective = r.objective;
        if (times) {
            times[0] = r.queued_ms;
            times[1] = r.device_ms;
            times[2] = r.latency_ms;
        }
        if (batch) *batch = r.batch;
    });
    return t_has_error ? -1 : 0;
}

compas_array* compas_b200_server_result(const compas_object* server, int64_t ticket, int which) {
    return guarded([&]() -> compas_array* {
        const compas::ServeResult r = server_of(server).wait(uint64_t(ticket));
        if (which == 0) return new_array(compas::Array<cfloat, 3>(r.residual));
        if (which == 1) return new_array(compas::Array<cfloat, 2>(r.gradient));
        throw compas::CompasException("invalid result index");
    });
}

int compas_b200_server_release(const compas_object* server, int64_t ticket) {
    t_has_error = false;
    guarded([&] { server_of(server).release(uint64_t(ticket)); });
    return t_has_error ? -1 : 0;
}

int compas_b200_server_drain(const compas_object* server) {
    t_has_error = false;
    guarded([&] { server_of(server).drain(); });
    return t_has_error ? -1 : 0;
}

int compas_b200_server_stats(const compas_object* server, double* out, int n) {
    t_has_error = false;
    const int written = guarded([&] {
        const compas::ServeStats s = server_of(server).stats();
        const double v[10] = {double(s.completed), double(s.failed), double(s.batches), double(s.echo_cache_hits),
                              s.p50_ms, s.p99_ms, s.mean_ms, s.max_ms, double(s.peak_bytes),
                              double(s.max_concurrent_batches)};
        int k = 0;
        for (; k < n && k < 10; k++) out[k] = v[k];
        return k;
    });
    return t_has_error ? -1 : written;
}

void compas_b200_server_reset_stats(const compas_object* server) {
    guarded([&] { server_of(server).reset_stats(); });
}

int compas_b200_gauss_newton_graph_kernels(const compas_object* gn) {
    t_has_error = false;
    const int n = guarded([&] { return unwrap<compas::GaussNewtonStep>(gn).kernels_per_iteration(); });
    return t_has_error ? -1 : n;
}

compas_array* compas_b200_batch_derivative(const compas_object* batch, int job, int field) {
    return guarded(
        [&] { return new_array(compas::Array<cfloat, 2>(unwrap<compas::SimulationBatch>(batch).derivative(job, field))); });
}

compas_array* compas_b200_batch_signal(const compas_object* batch, int job) {
    // a job without trajectory yields an empty [0][0][0] array
    return guarded([&] { return new_array(compas::Array<cfloat, 3>(unwrap<compas::SimulationBatch>(batch).signal(job))); });
}

}  // extern "C"
