// runtime.cu — the thin single-GPU runtime under the compas API: one stream per device,
// stream-ordered allocations from the device memory pool, blocking transfers, and a
// per-device status word that kernels use to report errors instead of trapping.
//
// Replaces the reference's kmm runtime for this path (compas/core/context.h:19-125):
// no chunking across devices, no task graph — operations are issued in order on the
// device's stream, so every result is ready for any later operation on that stream.
#include <atomic>
#include <cstdio>
#include <mutex>
#include <sstream>

#include "common.cuh"
#include "compas/compas.h"

namespace compas {

void throw_exception(const char* file, int line, const std::string& msg) {
    std::ostringstream s;
    s << msg << " (" << file << ":" << line << ")";
    throw CompasException(s.str());
}

namespace {

std::atomic<unsigned long long> g_launches {0};

struct DeviceState {
    bool ready = false;
    cudaStream_t stream = nullptr;
    unsigned int* status = nullptr;  // device word, see common.cuh STATUS_*
};

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
DeviceState g_devices[kMaxDevices];

DeviceState& device_state(int device) {
    if (device < 0 || device >= kMaxDevices) COMPAS_ERROR("invalid device index");
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceState& st = g_devices[device];
    if (!st.ready) {
        int count = 0;
        COMPAS_CUDA_CHECK(cudaGetDeviceCount(&count));
        if (device >= count) COMPAS_ERROR("device index out of range");
        int prev = 0;
        COMPAS_CUDA_CHECK(cudaGetDevice(&prev));
        COMPAS_CUDA_CHECK(cudaSetDevice(device));
        // Keep freed blocks in this process's pool so repeated operations reuse them.
        cudaMemPool_t pool;
        COMPAS_CUDA_CHECK(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t threshold = UINT64_MAX;
        COMPAS_CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
        COMPAS_CUDA_CHECK(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking));
        COMPAS_CUDA_CHECK(cudaMalloc(&st.status, sizeof(unsigned int)));
        COMPAS_CUDA_CHECK(cudaMemset(st.status, 0, sizeof(unsigned int)));
        COMPAS_CUDA_CHECK(cudaSetDevice(prev));
        st.ready = true;
    }
    return st;
}

}  // namespace

void note_launch() {
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

unsigned long long launch_count() {
    return g_launches.load(std::memory_order_relaxed);
}

namespace detail {

int current_device() {
    int d = 0;
    COMPAS_CUDA_CHECK(cudaGetDevice(&d));
    return d;
}

cudaStream_t device_stream(int device) {
    return device_state(device).stream;
}

unsigned int* device_status_word(int device) {
    return device_state(device).status;
}

Buffer::Buffer(size_t nbytes, int dev, cudaStream_t s) : bytes(nbytes), device(dev), stream(s) {
    if (bytes == 0) return;
    DeviceGuard guard(device);
    cudaError_t err = cudaMallocAsync(&ptr, bytes, stream);
    if (err != cudaSuccess) {
        (void)cudaGetLastError();
        std::ostringstream msg;
        msg << "device allocation of " << bytes << " bytes failed: " << cudaGetErrorString(err);
        throw CompasException(msg.str());
    }
}

Buffer::~Buffer() {
    if (ptr) {
        int prev = 0;
        if (cudaGetDevice(&prev) == cudaSuccess && prev != device) cudaSetDevice(device);
        cudaFreeAsync(ptr, stream);
        if (prev != device) cudaSetDevice(prev);
    }
}

}  // namespace detail

void ArrayBase::copy_bytes_to(void* dst, size_t n) const {
    if (n > nbytes()) COMPAS_ERROR("read of more bytes than the array holds");
    if (n == 0) return;
    DeviceGuard guard(device());
    cudaStream_t s = stream();
    COMPAS_CUDA_CHECK(cudaMemcpyAsync(dst, raw_data(), n, cudaMemcpyDeviceToHost, s));
    COMPAS_CUDA_CHECK(cudaStreamSynchronize(s));
    CompasContext(device(), s).check_device_status();
}

CompasContext::CompasContext(int device) : m_device(device), m_stream(detail::device_stream(device)) {}

CompasContext CompasContext::with_device(int index) const {
    int count = 0;
    COMPAS_CUDA_CHECK(cudaGetDeviceCount(&count));
    return CompasContext(index % count);
}

void CompasContext::upload(void* dst, const void* src, size_t bytes) const {
    if (bytes == 0) return;
    if (src == nullptr) COMPAS_ERROR("null host pointer");
    DeviceGuard guard(m_device);
    COMPAS_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, m_stream));
}

void CompasContext::synchronize() const {
    DeviceGuard guard(m_device);
    COMPAS_CUDA_CHECK(cudaStreamSynchronize(m_stream));
    check_device_status();
}

unsigned int* CompasContext::status_word() const {
    return m_status ? m_status : detail::device_status_word(m_device);
}

void CompasContext::check_device_status() const {
    DeviceGuard guard(m_device);
    unsigned int* word = status_word();
    unsigned int value = 0;
    COMPAS_CUDA_CHECK(cudaMemcpyAsync(&value, word, sizeof(value), cudaMemcpyDeviceToHost, m_stream));
    COMPAS_CUDA_CHECK(cudaStreamSynchronize(m_stream));
    if (value != 0) {
        COMPAS_CUDA_CHECK(cudaMemsetAsync(word, 0, sizeof(unsigned int), m_stream));
        std::ostringstream s;
        s << "a kernel reported an error (status 0x" << std::hex << value << "): " << status_message(value);
        throw CompasException(s.str());
    }
}

const char* status_message(unsigned int value) {
    if (value & STATUS_WAIT_TIMEOUT) return "a bounded device-side wait gave up";
    if (value & STATUS_BAD_ARGUMENT) return "invalid argument detected on the device";
    if (value & STATUS_TMEM) return "tensor-memory allocation failed";
    return "unknown device status";
}

TissueParameters make_tissue_parameters(const CompasContext& ctx, int num_voxels, int /*chunk_size*/,
                                        View<float> T1, View<float> T2, View<float> B1, View<float> B0,
                                        View<float> rho_x, View<float> rho_y, View<float> x, View<float> y,
                                        View<float> z) {
    COMPAS_CHECK(num_voxels >= 0);
    using F = int;
    namespace TF = TissueParameterField;
    Array<float, 2> params({TF::NUM_FIELDS, num_voxels}, ctx.device(), ctx.stream());
    DeviceGuard guard(ctx.device());
    cudaStream_t s = ctx.stream();
    size_t row = size_t(num_voxels) * sizeof(float);
    COMPAS_CUDA_CHECK(cudaMemsetAsync(params.data(), 0, row * TF::NUM_FIELDS, s));
    auto put = [&](F field, const View<float>& v) {
        if (v.is_empty()) return false;
        COMPAS_CHECK(v.size() >= num_voxels);
        COMPAS_CUDA_CHECK(cudaMemcpyAsync(params.data() + size_t(field) * num_voxels, v.data(), row,
                                          cudaMemcpyHostToDevice, s));
        return true;
    };
    if (num_voxels > 0) {
        COMPAS_CHECK(!T1.is_empty() && !T2.is_empty());
        put(TF::T1, T1);
        put(TF::T2, T2);
        put(TF::RHO_X, rho_x);
        put(TF::RHO_Y, rho_y);
        put(TF::X, x);
        put(TF::Y, y);
    }
    bool has_z = num_voxels > 0 && put(TF::Z, z);
    bool has_b0 = num_voxels > 0 && put(TF::B0, B0);
    bool has_b1 = num_voxels > 0 && put(TF::B1, B1);
    if (!has_b1 && num_voxels > 0) fill_float(params.data() + size_t(TF::B1) * num_voxels, num_voxels, 1.0F, s);
    return TissueParameters(params, has_z, has_b0, has_b1);
}

}  // namespace compas
