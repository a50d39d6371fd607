// shard.cu — one slice sharded over processes, one GPU each, with an NCCL sum of the partials.
//
// Every operation of the path is independent per voxel (simulation, derivatives, Jᴴ·v) or a sum
// over voxels (signal, J·v). A slice of V voxels is therefore split into contiguous voxel ranges,
// one per rank (voxel_shard, sizes differ by at most one): each rank simulates its voxels, the
// sums over voxels become per-rank partial [C][R][S] arrays, and one all-reduce (sum) over the
// ranks gives every rank the full result. Jᴴ·r needs no exchange: every rank holds the same
// residual and computes the gradient of its own voxels. This is the reference's chunking of the
// voxels over devices with a summing reduction of the signal (include/compas/core/context.h:51-68,
// src/trajectories/signal.cu:289-300), across processes instead of inside one.
//
// The all-reduce is NCCL's (over NVLink / NVSwitch between the GPUs of a node). The partial signal
// is 8·C·R·S bytes (8 MB at 4 coils × 1120 × 224), about 0.03 ms of NVLink time against tens of ms
// of simulation per rank, so it is issued as one collective after the contraction rather than
// fused into it. NCCL is loaded at run time (libnccl.so.2, the one the process already has, e.g.
// PyTorch's, or the system's), so the library does not link it and single-GPU users never load it.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "compas/compas.h"
#include "kernels.h"

namespace compas {

VoxelRange voxel_shard(int64_t nvoxels, int rank, int world) {
    if (world < 1) COMPAS_ERROR("world size must be at least 1");
    if (rank < 0 || rank >= world) COMPAS_ERROR("rank out of range");
    if (nvoxels < 0) COMPAS_ERROR("negative voxel count");
    const int64_t q = nvoxels / world, r = nvoxels % world;
    const int64_t begin = int64_t(rank) * q + std::min<int64_t>(rank, r);
    return {begin, begin + q + (rank < r ? 1 : 0)};
}

namespace {

struct NcclApi {
    void* handle = nullptr;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};

const NcclApi& nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) return;
        NcclApi a;
        a.handle = h;
        a.get_unique_id = reinterpret_cast<decltype(a.get_unique_id)>(dlsym(h, "ncclGetUniqueId"));
        a.comm_init_rank = reinterpret_cast<decltype(a.comm_init_rank)>(dlsym(h, "ncclCommInitRank"));
        a.all_reduce = reinterpret_cast<decltype(a.all_reduce)>(dlsym(h, "ncclAllReduce"));
        a.comm_destroy = reinterpret_cast<decltype(a.comm_destroy)>(dlsym(h, "ncclCommDestroy"));
        a.error_string = reinterpret_cast<decltype(a.error_string)>(dlsym(h, "ncclGetErrorString"));
        if (a.get_unique_id && a.comm_init_rank && a.all_reduce && a.comm_destroy && a.error_string) api = a;
    });
    if (!api.handle) COMPAS_ERROR("NCCL (libnccl.so.2) could not be loaded");
    return api;
}

void nccl_check(ncclResult_t r, const char* what) {
    if (r != ncclSuccess) throw CompasException(std::string(what) + ": " + nccl().error_string(r));
}

}  // namespace

struct Communicator::Impl {
    ncclComm_t comm = nullptr;
    int rank = 0, world = 1, device = 0;
    ~Impl() {
        if (comm) nccl().comm_destroy(comm);
    }
};

std::vector<char> Communicator::unique_id() {
    ncclUniqueId id;
    nccl_check(nccl().get_unique_id(&id), "ncclGetUniqueId");
    return std::vector<char>(id.internal, id.internal + sizeof(id.internal));
}

Communicator::Communicator(const CompasContext& ctx, int rank, int world, const std::vector<char>& id) :
    m_impl(std::make_shared<Impl>()) {
    if (world < 1 || rank < 0 || rank >= world) COMPAS_ERROR("invalid rank / world size");
    ncclUniqueId uid;
    if (id.size() != sizeof(uid.internal)) COMPAS_ERROR("an NCCL unique id has 128 bytes");
    std::memcpy(uid.internal, id.data(), sizeof(uid.internal));
    DeviceGuard guard(ctx.device());
    nccl_check(nccl().comm_init_rank(&m_impl->comm, world, uid, rank), "ncclCommInitRank");
    m_impl->rank = rank;
    m_impl->world = world;
    m_impl->device = ctx.device();
}

int Communicator::rank() const {
    return m_impl->rank;
}

int Communicator::world() const {
    return m_impl->world;
}

void Communicator::allreduce_sum(const CompasContext& ctx, float* data, int64_t count) const {
    if (ctx.device() != m_impl->device) COMPAS_ERROR("the communicator belongs to another device");
    if (count <= 0 || m_impl->world == 1) return;
    DeviceGuard guard(ctx.device());
    nccl_check(nccl().all_reduce(data, data, size_t(count), ncclFloat32, ncclSum, m_impl->comm, ctx.stream()),
               "ncclAllReduce");
}

Array<cfloat, 3> magnetization_to_signal_sharded(const CompasContext& ctx, const Communicator& comm,
                                                 const Array<cfloat, 2>& echos, const TissueParameters& parameters,
                                                 const Trajectory& trajectory, const Array<cfloat, 2>& coils,
                                                 SimulateSignalMethod method) {
    Array<cfloat, 3> s = magnetization_to_signal(ctx, echos, parameters, trajectory, coils, method);
    comm.allreduce_sum(ctx, reinterpret_cast<float*>(s.data()), 2 * s.numel());
    return s;
}

template<typename Traj>
Array<cfloat, 3> compute_jacobian_sharded(const CompasContext& ctx, const Communicator& comm,
                                          const Array<cfloat, 2>& echos, const Array<cfloat, 2>& dT1,
                                          const Array<cfloat, 2>& dT2, const TissueParameters& parameters,
                                          const Traj& trajectory, const Array<cfloat, 2>& coils,
                                          const Array<cfloat, 2>& vector, JacobianComputeMethod method) {
    Array<cfloat, 3> jv = compute_jacobian(ctx, echos, dT1, dT2, parameters, trajectory, coils, vector, method);
    comm.allreduce_sum(ctx, reinterpret_cast<float*>(jv.data()), 2 * jv.numel());
    return jv;
}

template Array<cfloat, 3> compute_jacobian_sharded(const CompasContext&, const Communicator&, const Array<cfloat, 2>&,
                                                   const Array<cfloat, 2>&, const Array<cfloat, 2>&,
                                                   const TissueParameters&, const CartesianTrajectory&,
                                                   const Array<cfloat, 2>&, const Array<cfloat, 2>&,
                                                   JacobianComputeMethod);
template Array<cfloat, 3> compute_jacobian_sharded(const CompasContext&, const Communicator&, const Array<cfloat, 2>&,
                                                   const Array<cfloat, 2>&, const Array<cfloat, 2>&,
                                                   const TissueParameters&, const SpiralTrajectory&,
                                                   const Array<cfloat, 2>&, const Array<cfloat, 2>&,
                                                   JacobianComputeMethod);

}  // namespace compas
