// compas.h — C++ API of the B200 implementation of the compas-toolkit simulation hot path.
//
// Source-level drop-in for the reference's C++ API (namespace `compas`, same type and
// function names and argument meaning; reference headers cited per declaration). The
// runtime under it is a thin single-GPU one: one CUDA stream per device, stream-ordered
// allocations from the device's memory pool, kernels written for sm_100a. There is no
// CPU fallback: every operation runs on the GPU and throws `CompasException` on error.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <array>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <variant>
#include <vector>

#include "compas/vector.h"

namespace compas {

using index_t = int;

// ------------------------------------------------------------------------------------------
// value types   (compas/core/complex_type.h:24-72, 324-325)
// ------------------------------------------------------------------------------------------
template<typename T>
struct alignas(2 * sizeof(T)) complex_type {
    T re, im;
    complex_type(T r = T(0), T i = T(0)) : re(r), im(i) {}
    T real() const { return re; }
    T imag() const { return im; }
};
using cfloat = complex_type<float>;
using cdouble = complex_type<double>;

// ------------------------------------------------------------------------------------------
// errors   (compas/core/assertion.h:35-66: COMPAS_CHECK throws CompasException)
// ------------------------------------------------------------------------------------------
class CompasException: public std::runtime_error {
  public:
    using std::runtime_error::runtime_error;
};

[[noreturn]] void throw_exception(const char* file, int line, const std::string& msg);

#define COMPAS_CHECK(cond)                                                              \
    do {                                                                                \
        if (!(cond)) ::compas::throw_exception(__FILE__, __LINE__, "check failed: " #cond); \
    } while (0)
#define COMPAS_ERROR(msg) ::compas::throw_exception(__FILE__, __LINE__, (msg))
#define COMPAS_CUDA_CHECK(expr)                                                               \
    do {                                                                                      \
        cudaError_t compas_err_ = (expr);                                                     \
        if (compas_err_ != cudaSuccess)                                                       \
            ::compas::throw_exception(__FILE__, __LINE__,                                     \
                                      std::string(#expr ": ") + cudaGetErrorString(compas_err_)); \
    } while (0)

// ------------------------------------------------------------------------------------------
// objects and arrays   (compas/core/object.h; kmm::Array used via compas/core/context.h:16-17)
// ------------------------------------------------------------------------------------------
class Object {
  public:
    virtual ~Object() = default;
    virtual const char* name() const { return "compas::Object"; }
};

namespace detail {
// One device allocation, released stream-ordered on the stream that made it.
struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    Buffer(size_t bytes, int device, cudaStream_t stream);
    ~Buffer();
    Buffer(const Buffer&) = delete;
    Buffer& operator=(const Buffer&) = delete;
};
int current_device();
cudaStream_t device_stream(int device);
}  // namespace detail

template<typename T, size_t N = 1>
struct View {
    const T* ptr = nullptr;
    std::array<int64_t, N> dims {};
    View() = default;
    View(const T* p, std::array<int64_t, N> d) : ptr(p), dims(d) {}
    const T* data() const { return ptr; }
    int64_t size(size_t i) const { return dims[i]; }
    int64_t size() const {
        int64_t n = 1;
        for (auto d : dims) n *= d;
        return n;
    }
    bool is_empty() const { return ptr == nullptr || size() == 0; }
};
template<typename T, size_t N = 1>
using HostView = View<T, N>;

class ArrayBase: public Object {
  public:
    virtual int rank() const = 0;
    virtual int64_t extent(int axis) const = 0;
    virtual size_t element_size() const = 0;
    virtual void* raw_data() const = 0;
    virtual int device() const = 0;
    // the stream the array was allocated on (its producer's stream); reads are ordered on it
    virtual cudaStream_t stream() const = 0;
    int64_t numel() const {
        int64_t n = 1;
        for (int i = 0; i < rank(); i++) n *= extent(i);
        return n;
    }
    size_t nbytes() const { return size_t(numel()) * element_size(); }
    // blocking device-to-host copy of the first `nbytes` bytes
    void copy_bytes_to(void* dst, size_t nbytes) const;
};

template<typename T, size_t N = 1>
class Array: public ArrayBase {
  public:
    Array() { m_dims.fill(0); }
    // allocates (uninitialised) device memory on the current device's stream
    Array(std::array<int64_t, N> dims) : m_dims(dims) {
        allocate(detail::current_device(), detail::device_stream(detail::current_device()));
    }
    Array(std::array<int64_t, N> dims, int device) : m_dims(dims) { allocate(device, detail::device_stream(device)); }
    // allocated and released stream-ordered on `stream` (a context's stream)
    Array(std::array<int64_t, N> dims, int device, cudaStream_t stream) : m_dims(dims) { allocate(device, stream); }

    const char* name() const override { return "compas::Array"; }
    int rank() const override { return int(N); }
    int64_t extent(int axis) const override { return m_dims[size_t(axis)]; }
    size_t element_size() const override { return sizeof(T); }
    void* raw_data() const override { return m_buf ? m_buf->ptr : nullptr; }
    int device() const override { return m_buf ? m_buf->device : 0; }
    cudaStream_t stream() const override { return m_buf ? m_buf->stream : detail::device_stream(device()); }
    // Order later reads and the release of this array on `s` instead of its allocation stream.
    // Only valid once the host has seen every pending use of the array complete (an event or a
    // synchronisation), since `s` is not ordered after that work.
    void set_stream(cudaStream_t s) const {
        if (m_buf) m_buf->stream = s;
    }

    T* data() const { return static_cast<T*>(raw_data()); }
    int64_t size(size_t axis) const { return m_dims[axis]; }
    std::array<int64_t, N> sizes() const { return m_dims; }
    int64_t size() const { return numel(); }
    int64_t chunk_size(size_t axis) const { return m_dims[axis]; }  // one chunk per array
    bool is_valid() const { return bool(m_buf) || numel() == 0; }

    void copy_to(T* dst) const { copy_bytes_to(dst, nbytes()); }
    std::vector<T> copy_to_vector() const {
        std::vector<T> out(static_cast<size_t>(numel()));
        copy_to(out.data());
        return out;
    }

  private:
    void allocate(int device, cudaStream_t stream) {
        int64_t n = 1;
        for (auto d : m_dims) {
            if (d < 0) throw CompasException("negative array dimension");
            n *= d;
        }
        m_buf = std::make_shared<detail::Buffer>(size_t(n) * sizeof(T), device, stream);
    }
    std::array<int64_t, N> m_dims;
    std::shared_ptr<detail::Buffer> m_buf;
};

// ------------------------------------------------------------------------------------------
// context   (compas/core/context.h:19-125)
// ------------------------------------------------------------------------------------------
class CompasContext {
  public:
    explicit CompasContext(int device = 0);
    // a view of the device's context that issues work, and allocates, on `stream` (which the
    // caller keeps alive while work or arrays made through this view exist)
    CompasContext(int device, cudaStream_t stream) : m_device(device), m_stream(stream) {}
    // the same with its own device status word (a device `unsigned int` the caller allocates,
    // zeroes and keeps alive): kernels launched through this view record their errors there, and
    // check_device_status() reads and clears only that word. Concurrent users of one device (the
    // serving engine's slots) keep each other's errors apart this way.
    CompasContext(int device, cudaStream_t stream, unsigned int* status_word) :
        m_device(device), m_stream(stream), m_status(status_word) {}
    CompasContext with_device(int index) const;
    int device() const { return m_device; }
    cudaStream_t stream() const { return m_stream; }
    // the device word this view's kernels report errors in (its own, else the device's)
    unsigned int* status_word() const;

    template<typename T, size_t N>
    Array<std::decay_t<T>, N> allocate(View<T, N> content) const {
        Array<std::decay_t<T>, N> out(content.dims, m_device, m_stream);
        upload(out.data(), content.data(), size_t(content.size()) * sizeof(T));
        return out;
    }
    template<typename T, typename... Sizes>
    Array<std::decay_t<T>, sizeof...(Sizes)> allocate(const T* content, Sizes... sizes) const {
        std::array<int64_t, sizeof...(Sizes)> dims = {int64_t(sizes)...};
        return allocate(View<T, sizeof...(Sizes)>(content, dims));
    }
    template<typename T>
    Array<std::decay_t<T>> allocate(const std::vector<T>& content) const {
        return allocate(content.data(), int64_t(content.size()));
    }

    void synchronize() const;
    // raises CompasException when a kernel recorded an error in the device status word
    void check_device_status() const;

  private:
    void upload(void* dst, const void* src, size_t bytes) const;
    int m_device;
    cudaStream_t m_stream;
    unsigned int* m_status = nullptr;
};

inline CompasContext make_context(int device = 0) {
    return CompasContext(device);
}

// ------------------------------------------------------------------------------------------
// tissue parameters   (compas/parameters/tissue.h:16-67, tissue_view.cuh:42-72)
// ------------------------------------------------------------------------------------------
namespace TissueParameterField {
enum { T1 = 0, T2 = 1, B1 = 2, B0 = 3, RHO_X = 4, RHO_Y = 5, X = 6, Y = 7, Z = 8, NUM_FIELDS = 9 };
}

struct TissueParameters: public Object {
    Array<float, 2> data;  // [NUM_FIELDS][nvoxels]
    int nvoxels = 0;
    int chunk_size = 0;
    bool has_z = true;
    bool has_b0 = true;
    bool has_b1 = true;

    TissueParameters() = default;
    TissueParameters(Array<float, 2> parameters, bool has_z, bool has_b0, bool has_b1) :
        data(parameters),
        nvoxels(int(parameters.size(1))),
        chunk_size(int(parameters.size(1))),
        has_z(has_z),
        has_b0(has_b0),
        has_b1(has_b1) {}
    const char* name() const override { return "compas::TissueParameters"; }
};

TissueParameters make_tissue_parameters(
    const CompasContext& ctx,
    int num_voxels,
    int chunk_size,
    View<float> T1,
    View<float> T2,
    View<float> B1,
    View<float> B0,
    View<float> rho_x,
    View<float> rho_y,
    View<float> x,
    View<float> y,
    View<float> z = {});

// ------------------------------------------------------------------------------------------
// sequences   (compas/sequences/fisp.h:10-60, sequences/pssfp.h:9-72, pssfp_view.h:7-11)
// ------------------------------------------------------------------------------------------
struct FISPSequence: public Object {
    Array<cfloat> RF_train;             // [nTR] flip angle (deg) and phase
    Array<cfloat, 2> sliceprofiles;     // [npositions][nTR]
    float TR = 0;
    float TE = 0;
    float TW = 0;
    int max_state = 0;
    float TI = 0;
    int undersampling_factor = 1;
    int repetitions = 1;
    bool inversion_prepulse = true;
    bool wait_spoiling = true;

    FISPSequence() = default;
    FISPSequence(Array<cfloat> RF_train, Array<cfloat, 2> sliceprofiles, float TR, float TE, float TW,
                 int max_state, float TI, int undersampling_factor = 1, int repetitions = 1,
                 bool inversion_prepulse = true, bool wait_spoiling = true) :
        RF_train(RF_train), sliceprofiles(sliceprofiles), TR(TR), TE(TE), TW(TW), max_state(max_state), TI(TI),
        undersampling_factor(undersampling_factor), repetitions(repetitions),
        inversion_prepulse(inversion_prepulse), wait_spoiling(wait_spoiling) {}
    const char* name() const override { return "compas::FISPSequence"; }

    // device-resident per-(position, TR) excitation table, built on first use; copies of the
    // sequence share it, so repeated simulations reuse it
    struct Cache {
        std::mutex mutex;
        const void* key_rf = nullptr;
        const void* key_sp = nullptr;
        std::shared_ptr<Array<float, 3>> table;
        int real_phases = -1;  // host copy of the table's phase flag: -1 not read yet, else 0 / 1
    };
    std::shared_ptr<Cache> cache = std::make_shared<Cache>();
};

inline FISPSequence make_fisp_sequence(const CompasContext& context, View<cfloat> RF_train,
                                       View<cfloat, 2> sliceprofiles, float TR, float TE, int max_state,
                                       float TI) {
    return FISPSequence(context.allocate(RF_train), context.allocate(sliceprofiles), TR, TE, 0.0F, max_state, TI);
}

struct RepetitionData {
    float ex;
    float inv;
    float pr;
};

struct pSSFPSequence: public Object {
    Array<cfloat> RF_train;
    float TR = 0;
    int nRF = 0;
    int nTR = 0;
    Array<cfloat> gamma_dt_RF;
    RepetitionData dt {};
    RepetitionData gamma_dt_GRz {};
    int nz = 0;
    Array<float> z;

    pSSFPSequence() = default;
    pSSFPSequence(Array<cfloat> RF_train, float TR, Array<cfloat> gamma_dt_RF, RepetitionData dt,
                  RepetitionData gamma_dt_GRz, Array<float> z) :
        RF_train(RF_train), TR(TR), nRF(int(gamma_dt_RF.size())), nTR(int(RF_train.size())),
        gamma_dt_RF(gamma_dt_RF), dt(dt), gamma_dt_GRz(gamma_dt_GRz), nz(int(z.size())), z(z) {}
    const char* name() const override { return "compas::pSSFPSequence"; }

    // device-resident rotation table [nTR+1][nRF] (row 0: the α/2 pulse), built on first use
    // and shared by copies of the sequence
    struct Cache {
        std::mutex mutex;
        const void* key_rf = nullptr;
        const void* key_g = nullptr;
        std::shared_ptr<Array<cfloat, 2>> table;
        int real_rf = -1;  // host copy of the table's flag: -1 not read yet, 1 every RF sample real, else 0
    };
    std::shared_ptr<Cache> cache = std::make_shared<Cache>();
};

inline pSSFPSequence make_pssfp_sequence(const CompasContext& context, View<cfloat> RF_train, float TR,
                                         View<cfloat> gamma_dt_RF, RepetitionData dt, RepetitionData gamma_dt_GRz,
                                         View<float> z) {
    COMPAS_CHECK(RF_train.size() > 0);
    return pSSFPSequence(context.allocate(RF_train), TR, context.allocate(gamma_dt_RF), dt, gamma_dt_GRz,
                         context.allocate(z));
}

// ------------------------------------------------------------------------------------------
// trajectories   (compas/trajectories/trajectory.h:10-19, cartesian.h:17-58, spiral.h:14-57)
// ------------------------------------------------------------------------------------------
struct Trajectory: public Object {
    int nreadouts = 0;
    int samples_per_readout = 0;
    float delta_t = 0;
    Trajectory() = default;
    Trajectory(int nreadouts, int samples_per_readout, float delta_t) :
        nreadouts(nreadouts), samples_per_readout(samples_per_readout), delta_t(delta_t) {}
};

struct CartesianTrajectory: public Trajectory {
    Array<cfloat> k_start;  // [nreadouts]
    cfloat delta_k;
    CartesianTrajectory() = default;
    CartesianTrajectory(int nreadouts, int samples_per_readout, float delta_t, Array<cfloat> k_start,
                        cfloat delta_k) :
        Trajectory(nreadouts, samples_per_readout, delta_t), k_start(k_start), delta_k(delta_k) {}
    const char* name() const override { return "compas::CartesianTrajectory"; }
};

inline CartesianTrajectory make_cartesian_trajectory(const CompasContext& context, int nreadouts,
                                                     int samples_per_readout, float delta_t,
                                                     HostView<cfloat> k_start, cfloat delta_k) {
    COMPAS_CHECK(k_start.size() == nreadouts);
    return CartesianTrajectory(nreadouts, samples_per_readout, delta_t, context.allocate(k_start), delta_k);
}

struct SpiralTrajectory: public Trajectory {
    Array<cfloat> k_start;  // [nreadouts]
    Array<cfloat> delta_k;  // [nreadouts]
    SpiralTrajectory() = default;
    SpiralTrajectory(int nreadouts, int samples_per_readout, float delta_t, Array<cfloat> k_start,
                     Array<cfloat> delta_k) :
        Trajectory(nreadouts, samples_per_readout, delta_t), k_start(k_start), delta_k(delta_k) {}
    const char* name() const override { return "compas::SpiralTrajectory"; }
};

inline SpiralTrajectory make_spiral_trajectory(const CompasContext& context, int nreadouts,
                                               int samples_per_readout, float delta_t, View<cfloat> k_start,
                                               View<cfloat> delta_k) {
    COMPAS_CHECK(k_start.size() == nreadouts);
    COMPAS_CHECK(delta_k.size() == nreadouts);
    return SpiralTrajectory(nreadouts, samples_per_readout, delta_t, context.allocate(k_start),
                            context.allocate(delta_k));
}

// ------------------------------------------------------------------------------------------
// operations
// ------------------------------------------------------------------------------------------

// FISP EPG simulation; echos [nTR*undersampling][nvoxels]   (compas/simulate/fisp.h:17-20)
Array<cfloat, 2> simulate_magnetization(const CompasContext& context, TissueParameters parameters,
                                        FISPSequence sequence);

// pSSFP isochromat simulation; echos [nTR][nvoxels]   (compas/simulate/pssfp.h:17-20)
Array<cfloat, 2> simulate_magnetization(const CompasContext& context, TissueParameters parameters,
                                        pSSFPSequence sequence);

static constexpr float DEFAULT_FINITE_DIFFERENCE_DELTA = 1e-4F;

// forward finite difference (m(p + Δ e_field) - m(p)) / Δ   (compas/simulate/derivative.h:7-47)
Array<cfloat, 2> simulate_magnetization_derivative(const CompasContext& context, int field, Array<cfloat, 2> echos,
                                                   TissueParameters parameters, pSSFPSequence sequence,
                                                   float delta = DEFAULT_FINITE_DIFFERENCE_DELTA);
Array<cfloat, 2> simulate_magnetization_derivative(const CompasContext& context, int field, Array<cfloat, 2> echos,
                                                   TissueParameters parameters, FISPSequence sequence,
                                                   float delta = DEFAULT_FINITE_DIFFERENCE_DELTA);

// m, ∂m/∂T1 and ∂m/∂T2 in one pass: forward-mode tangents propagated with the state, the
// Δ → 0 limit of simulate_magnetization_derivative for the fields T1 and T2 without the
// difference's cancellation error. echos is the value recurrence of simulate_magnetization (equal
// to FP32 rounding: the compiler may contract a different multiply-add in the two kernels).
struct MagnetizationTangents {
    Array<cfloat, 2> echos, dT1, dT2;  // [nreadouts][nvoxels] each
};
MagnetizationTangents simulate_magnetization_tangents(const CompasContext& context, TissueParameters parameters,
                                                      FISPSequence sequence);
MagnetizationTangents simulate_magnetization_tangents(const CompasContext& context, TissueParameters parameters,
                                                      pSSFPSequence sequence);

// echo[r][v] · exp(i y_v Im k_start[r])   (compas/trajectories/phase_encoding.h:19-23)
Array<cfloat, 2> phase_encoding(const CompasContext& ctx, const Array<cfloat, 2>& echos,
                                const TissueParameters& parameters, const CartesianTrajectory& trajectory);

// (compas/trajectories/signal.h:14-44). Naive, Direct, MatmulPedantic and Matmul run the plain
// FP32 SIMT kernels; MatmulFast and MatmulLow run the split-BF16 tcgen05 tensor-core kernels
// (three BF16 products accumulated in FP32, relative error ≤1e-4 against FP64).
enum struct SimulateSignalMethod { Naive, Direct, MatmulPedantic, Matmul, MatmulFast, MatmulLow };

// MR signal [ncoils][nreadouts][samples_per_readout]   (compas/trajectories/signal.h:46-63)
Array<cfloat, 3> magnetization_to_signal(const CompasContext& context, Array<cfloat, 2> echos,
                                         TissueParameters parameters, const Trajectory& trajectory,
                                         Array<cfloat, 2> coil_sensitivities,
                                         SimulateSignalMethod method = SimulateSignalMethod::MatmulFast);

// (compas/jacobian/product.h:10). Naive, Direct and Gemm: plain FP32; GemmFast and GemmLow:
// split-BF16 tensor cores.
enum struct JacobianComputeMethod { Naive, Direct, Gemm, GemmFast, GemmLow };

// J·v, v [4][nvoxels] -> [ncoils][nreadouts][ns]   (compas/jacobian/product.h:12-34)
Array<cfloat, 3> compute_jacobian(const CompasContext& ctx, Array<cfloat, 2> echos, Array<cfloat, 2> delta_echos_T1,
                                  Array<cfloat, 2> delta_echos_T2, TissueParameters parameters,
                                  CartesianTrajectory trajectory, Array<cfloat, 2> coil_sensitivities,
                                  Array<cfloat, 2> vector, JacobianComputeMethod kind = JacobianComputeMethod::Direct);

// Jᴴ·v, v [ncoils][nreadouts][ns] -> [4][nvoxels]   (compas/jacobian/hermitian.h:12-33)
Array<cfloat, 2> compute_jacobian_hermitian(const CompasContext& ctx, Array<cfloat, 2> echos,
                                            Array<cfloat, 2> delta_echos_T1, Array<cfloat, 2> delta_echos_T2,
                                            TissueParameters parameters, CartesianTrajectory trajectory,
                                            Array<cfloat, 2> coil_sensitivities, Array<cfloat, 3> vector,
                                            JacobianComputeMethod kind = JacobianComputeMethod::Direct);

// J·v and Jᴴ·v on a spiral trajectory (no counterpart in the reference, whose Jacobians take a
// CartesianTrajectory only): the derivatives of the spiral signal model with the Cartesian
// column scaling; FP32 kernels for every method
Array<cfloat, 3> compute_jacobian(const CompasContext& ctx, Array<cfloat, 2> echos, Array<cfloat, 2> delta_echos_T1,
                                  Array<cfloat, 2> delta_echos_T2, TissueParameters parameters,
                                  SpiralTrajectory trajectory, Array<cfloat, 2> coil_sensitivities,
                                  Array<cfloat, 2> vector, JacobianComputeMethod kind = JacobianComputeMethod::Direct);
Array<cfloat, 2> compute_jacobian_hermitian(const CompasContext& ctx, Array<cfloat, 2> echos,
                                            Array<cfloat, 2> delta_echos_T1, Array<cfloat, 2> delta_echos_T2,
                                            TissueParameters parameters, SpiralTrajectory trajectory,
                                            Array<cfloat, 2> coil_sensitivities, Array<cfloat, 3> vector,
                                            JacobianComputeMethod kind = JacobianComputeMethod::Direct);

// lhs - rhs and Σ|lhs - rhs|²   (compas/utils/residual.h:20-24)
Array<cfloat, 3> compute_residual(CompasContext ctx, Array<cfloat, 3> lhs, Array<cfloat, 3> rhs,
                                  float* objective_out = nullptr);

// ------------------------------------------------------------------------------------------
// batched execution (no counterpart in the reference, which runs one operation per call)
// ------------------------------------------------------------------------------------------

// One independent simulate → signal job: its own voxels, sequence, trajectory and coils.
// Without a trajectory the job only simulates.
struct SimulationJob {
    TissueParameters parameters;
    std::variant<FISPSequence, pSSFPSequence> sequence;
    std::variant<std::monostate, CartesianTrajectory, SpiralTrajectory> trajectory;
    Array<cfloat, 2> coil_sensitivities;  // [ncoils][nvoxels]
    bool tangents = false;  // also ∂echos/∂T1 and ∂echos/∂T2 (forward-mode tangents): derivative()
};

// Many jobs of uneven size in a handful of launches: every FISP job of one launch layout runs
// in one persistent work-queue kernel, every pSSFP job likewise (on a second stream, so the two
// families overlap), then the Cartesian signals of each family in one batched tensor-core
// launch and the spiral signals in one batched launch per coil grouping. Each job gives the
// same bits as simulate_magnetization + magnetization_to_signal called for it alone.
// All buffers are allocated at construction; run() only enqueues kernels (and can be captured
// into a CUDA graph).
class SimulationBatch: public Object {
  public:
    SimulationBatch(const CompasContext& ctx, std::vector<SimulationJob> jobs,
                    SimulateSignalMethod method = SimulateSignalMethod::MatmulFast);
    // enqueue every job on the context's stream (returns without waiting)
    void run() const;
    int size() const;
    const Array<cfloat, 2>& echos(int job) const;   // [nreadouts][nvoxels]
    const Array<cfloat, 3>& signal(int job) const;  // [ncoils][nreadouts][ns]; empty without trajectory
    // ∂echos/∂T1 (field 0) or ∂echos/∂T2 (field 1) of a job with `tangents` set (the same bits as
    // simulate_magnetization_tangents for it alone)
    const Array<cfloat, 2>& derivative(int job, int field) const;
    const char* name() const override { return "compas::SimulationBatch"; }

    struct Impl;

  private:
    std::shared_ptr<Impl> m_impl;
};

// ------------------------------------------------------------------------------------------
// serving (no counterpart in the reference)
// ------------------------------------------------------------------------------------------

// A reconstruction request: simulate the echoes of `parameters` under `sequence`, form the
// signal on `trajectory` with `coil_sensitivities`, the residual b = data - s and its norm, and
// the gradient Jᴴ·b with forward-difference ∂m/∂T1, ∂m/∂T2 (on a spiral trajectory through the
// spiral Jacobian, which the reference does not have). Requests with the same nonzero `echo_key` share echoes and
// derivatives: while an entry is resident, a request with its key skips the simulations (the
// caller guarantees that equal keys mean equal parameters and sequence).
struct ServeRequest {
    TissueParameters parameters;
    std::variant<FISPSequence, pSSFPSequence> sequence;
    std::variant<CartesianTrajectory, SpiralTrajectory> trajectory;
    Array<cfloat, 2> coil_sensitivities;  // [ncoils][nvoxels]
    Array<cfloat, 3> data;                // measured signal [ncoils][nreadouts][ns]
    uint64_t echo_key = 0;
    // failure-path test hook: the batch holding this request also runs a kernel whose bounded wait
    // on a barrier that nothing completes gives up, so that batch (and only it) reports
    // STATUS_WAIT_TIMEOUT and its requests fail
    bool inject_wait_timeout = false;
};

struct ServeResult {
    Array<cfloat, 3> residual;  // data - s
    Array<cfloat, 2> gradient;  // Jᴴ·(data - s) [4][nvoxels]
    float objective = 0;        // ‖data - s‖²
    double queued_ms = 0;       // submit → admitted to a batch
    double device_ms = 0;       // admitted → results complete on the device
    double latency_ms = 0;      // submit → complete
    int batch = -1;             // batch it ran in
    bool echo_cache_hit = false;
};

struct ServeOptions {
    size_t memory_budget_bytes = size_t(150) << 30;  // admission budget for working sets and results
    int max_inflight_batches = 4;                     // batches on the device at once, one stream each
    int max_batch_requests = 16;                      // requests admitted into one batch
    size_t echo_cache_bytes = size_t(16) << 30;      // resident echoes/derivatives (within the budget)
    SimulateSignalMethod method = SimulateSignalMethod::MatmulFast;
    float delta = DEFAULT_FINITE_DIFFERENCE_DELTA;  // forward-difference step; 0: exact tangents
};

struct ServeStats {
    uint64_t completed = 0, failed = 0, batches = 0, echo_cache_hits = 0;
    double p50_ms = 0, p99_ms = 0, mean_ms = 0, max_ms = 0;
    size_t peak_bytes = 0;        // peak of the admitted footprints plus cached echoes
    int max_concurrent_batches = 0;
};

// Continuous-batching request loop on one GPU. submit() queues a request (thread-safe); a
// worker thread admits queued requests in arrival order while their estimated device footprint
// fits the memory budget and a batch slot is free, runs each admitted group as one
// SimulationBatch (persistent work-queue simulations of all requests, their derivative
// simulations and batched signals) followed by the per-request residuals and gradients, on the
// slot's own stream, so batches admitted while others run overlap on the device. Each result is
// the same, bit for bit, as the one-request operations give.
class ServeEngine: public Object {
  public:
    explicit ServeEngine(const CompasContext& ctx, ServeOptions options = {});
    ~ServeEngine() override;
    uint64_t submit(ServeRequest request);
    bool ready(uint64_t ticket) const;
    // blocks until the request completed; throws CompasException if it failed. The result's
    // arrays stay valid after release().
    ServeResult wait(uint64_t ticket);
    void release(uint64_t ticket);  // forget a completed request (frees its budget share)
    void drain();                   // blocks until every submitted request completed
    ServeStats stats() const;
    void reset_stats();
    const char* name() const override { return "compas::ServeEngine"; }

    struct Impl;

  private:
    std::shared_ptr<Impl> m_impl;
};

// One Gauss–Newton iteration of MR-STAT parameter fitting, on the device and captured as a CUDA
// graph on first use (no counterpart in the reference, whose callers chain the operations):
// simulate m(p), ∂m/∂T1 and ∂m/∂T2 (forward differences with step `delta`; delta = 0 takes the
// exact forward-mode tangents of simulate_magnetization_tangents), s = signal(m), b = y - s, then
// `cg_iterations` CGLS iterations (one J·d and one Jᴴ·b each) on min ‖J δ - b‖² over real δ in
// the Jacobian's scaled coordinates (δT1/T1, δT2/T2, δRe ρ, δIm ρ), and the update
// T1·c(δ0), T2·c(δ1), ρ + δ2 + iδ3 with c(x) = clamp(1 + x, ½, 2). The estimate is a private
// copy of `parameters`; every buffer is allocated at construction.
class GaussNewtonStep: public Object {
  public:
    GaussNewtonStep(const CompasContext& ctx, TissueParameters parameters,
                    std::variant<FISPSequence, pSSFPSequence> sequence,
                    std::variant<CartesianTrajectory, SpiralTrajectory> trajectory,
                    Array<cfloat, 2> coil_sensitivities, Array<cfloat, 3> data, int cg_iterations = 4,
                    float delta = DEFAULT_FINITE_DIFFERENCE_DELTA,
                    JacobianComputeMethod method = JacobianComputeMethod::GemmFast);
    // enqueue one iteration on the context's stream: a replay of the captured graph (captured
    // on the first call), or the kernels one by one
    void run(bool use_graph = true);
    const TissueParameters& parameters() const;       // current estimate
    const Array<cfloat, 2>& echos() const;            // m(p) of the last iteration
    const Array<cfloat, 2>& derivative(int field) const;  // ∂m/∂T1 or ∂m/∂T2
    const Array<cfloat, 3>& signal() const;           // s(p)
    const Array<cfloat, 2>& gradient() const;         // Jᴴ·b of the last CG iteration [4][V]
    const Array<float, 2>& step() const;              // δ [4][V]
    // device scalars: [0] ‖y - s(p)‖² before the update, [1] γ, [2] γ', [3] ‖q‖², [4] α, [5] β,
    // [6] objective of the last line-search trial, [7] step length taken (1, ½ or 0)
    const Array<float>& scalars() const;
    // line search on the objective before the update (on by default): the first of the steps
    // t = 1, ½ that does not raise ‖y - s(p)‖² is taken, else none. Changing it drops the graph.
    void set_line_search(bool on);
    bool line_search() const;
    int kernels_per_iteration() const;  // kernel nodes of the captured graph (-1 before capture)
    const char* name() const override { return "compas::GaussNewtonStep"; }

    struct Impl;

  private:
    std::shared_ptr<Impl> m_impl;
};

// ------------------------------------------------------------------------------------------
// GEMM utilities   (compas/utils/gemm.h:7-70)
// ------------------------------------------------------------------------------------------
using bfloat16 = __nv_bfloat16;

enum struct GemmComputeMethod {
    Pedantic,  // highest precision: FP32 on the CUDA cores
    Regular,   // FP32 on the CUDA cores
    Fast       // split-BF16 on the tensor cores, ~1e-5 relative (the reference: TF32, ~1e-3)
};

// result = alpha·lhs·rhsᵀ + beta·result, lhs [m][k], rhs [n][k], result [m][n] (result is not read
// when beta == 0). BF16 inputs run on the tensor cores with FP32 accumulation for every method.
void compute_gemm(const CompasContext& ctx, Array<float, 2>& result, const Array<float, 2>& lhs,
                  const Array<float, 2>& rhs, float alpha, float beta,
                  GemmComputeMethod kind = GemmComputeMethod::Regular);
void compute_gemm(const CompasContext& ctx, Array<float, 2>& result, const Array<bfloat16, 2>& lhs,
                  const Array<bfloat16, 2>& rhs, float alpha, float beta,
                  GemmComputeMethod kind = GemmComputeMethod::Regular);
// the same for complex matrices in planar form: [2][rows][cols], plane 0 real, plane 1 imaginary
// (no conjugation: result = alpha·lhs·rhsᵀ + beta·result)
void compute_complex_gemm(const CompasContext& ctx, Array<float, 3>& result, const Array<float, 3>& lhs,
                          const Array<float, 3>& rhs, float alpha, float beta,
                          GemmComputeMethod kind = GemmComputeMethod::Regular);
void compute_complex_gemm(const CompasContext& ctx, Array<float, 3>& result, const Array<bfloat16, 3>& lhs,
                          const Array<bfloat16, 3>& rhs, float alpha, float beta,
                          GemmComputeMethod kind = GemmComputeMethod::Regular);
// interleaved complex [n][m] <-> planar [2][n][m]
void convert_complex_to_planar(const CompasContext& ctx, Array<float, 3>& output, const Array<cfloat, 2>& input);
void convert_complex_to_planar(const CompasContext& ctx, Array<bfloat16, 3>& output, const Array<cfloat, 2>& input);
void convert_planar_to_complex(const CompasContext& ctx, Array<cfloat, 2>& output, const Array<float, 3>& input);

// ------------------------------------------------------------------------------------------
// one slice sharded over processes, one GPU each (no counterpart in the reference's API: its kmm
// runtime chunks voxels over the devices of one process, include/compas/core/context.h:51-68,
// and sums the chunks' signals, src/trajectories/signal.cu:289-300)
// ------------------------------------------------------------------------------------------
struct VoxelRange {
    int64_t begin = 0, end = 0;
    int64_t size() const { return end - begin; }
};
// voxels [begin, end) of `rank` among `world` ranks: contiguous, sizes differ by at most one
VoxelRange voxel_shard(int64_t nvoxels, int rank, int world);

// An NCCL communicator over `world` processes, one GPU each (the context's device). Every rank
// passes the same 128-byte unique id, made once by one rank with unique_id() and sent to the
// others by the caller; construction blocks until all ranks have joined. NCCL (libnccl.so.2) is
// loaded on first use.
class Communicator: public Object {
  public:
    static std::vector<char> unique_id();
    Communicator(const CompasContext& ctx, int rank, int world, const std::vector<char>& unique_id);
    int rank() const;
    int world() const;
    // in-place sum of `count` floats over the ranks, stream-ordered on ctx's stream
    void allreduce_sum(const CompasContext& ctx, float* data, int64_t count) const;
    const char* name() const override { return "compas::Communicator"; }

  private:
    struct Impl;
    std::shared_ptr<Impl> m_impl;
};

// The signal / J·v of a slice whose voxels are sharded over the communicator's ranks: every rank
// passes its own voxels (echoes [R][V_rank], their parameters and coil sensitivities, for J·v their
// derivative echoes and the [4][V_rank] direction) and receives the full [C][R][S] result, the sum
// of the ranks' partials. Jᴴ·v needs no such variant: each rank computes its voxels' gradient from
// the full residual with compute_jacobian_hermitian.
Array<cfloat, 3> magnetization_to_signal_sharded(const CompasContext& ctx, const Communicator& comm,
                                                 const Array<cfloat, 2>& echos, const TissueParameters& parameters,
                                                 const Trajectory& trajectory, const Array<cfloat, 2>& coils,
                                                 SimulateSignalMethod method = SimulateSignalMethod::MatmulFast);
template<typename Traj>
Array<cfloat, 3> compute_jacobian_sharded(const CompasContext& ctx, const Communicator& comm,
                                          const Array<cfloat, 2>& echos, const Array<cfloat, 2>& dT1,
                                          const Array<cfloat, 2>& dT2, const TissueParameters& parameters,
                                          const Traj& trajectory, const Array<cfloat, 2>& coils,
                                          const Array<cfloat, 2>& vector,
                                          JacobianComputeMethod method = JacobianComputeMethod::GemmFast);

}  // namespace compas
