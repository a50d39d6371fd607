"""Voxel-sharded signal on the GPU through torch.distributed/NCCL with one rank: the partial-signal
callable, the zero-copy torch view of a library array (__cuda_array_interface__) and the NCCL
all-reduce give the unsharded signal. (Several ranks need several GPUs; the multi-rank partition
and reduction logic is covered by the gloo test on CPU.)"""
import os
import socket

import numpy as np
import pytest

import workloads as W

pytestmark = pytest.mark.gpu


def test_single_rank_nccl_sharded_signal_equals_unsharded():
    import torch
    import torch.distributed as dist

    import compas_b200 as cb
    from sharding import VoxelShard, gpu_partial_signal, gpu_to_tensor, sharded_signal

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        ctx = cb.Context(0)
        w = W.tiny(seed=8, n_side=9, ntr=17, ns=10, nc=2)
        seq = cb.FispSequence.from_dict(ctx, w["seq"])
        traj = cb.CartesianTrajectory.from_dict(ctx, w["traj"])
        shard = VoxelShard(w["params"].shape[1], 0, 1)
        fn = gpu_partial_signal(cb, ctx, seq, traj)
        out = sharded_signal(shard, fn, w["params"], w["coils"], None, gpu_to_tensor(ctx))
        torch.cuda.synchronize()
        got = torch.view_as_complex(out).cpu().numpy()
        p = cb.TissueParameters.from_soa(ctx, w["params"])
        ref = cb.magnetization_to_signal(ctx, cb.simulate_magnetization(ctx, p, seq), p, traj, w["coils"],
                                         method="MatmulFast").to_numpy()
        assert np.array_equal(got, ref)
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def one_rank():
    import compas_b200 as cb

    ctx = cb.Context(0)
    return cb, ctx, cb.Communicator(ctx, 0, 1, cb.comm_unique_id())


def test_library_communicator_one_rank_is_the_identity(one_rank):
    # the library's NCCL communicator with one rank: sharded signal and J·v equal the unsharded
    # operations bit for bit, and an all-reduce leaves an array as it was
    cb, ctx, comm = one_rank
    w = W.tiny(seed=9, n_side=9, ntr=17, ns=10, nc=2)
    p = cb.TissueParameters.from_soa(ctx, w["params"])
    traj = cb.CartesianTrajectory.from_dict(ctx, w["traj"])
    e = cb.simulate_magnetization(ctx, p, cb.FispSequence.from_dict(ctx, w["seq"]))
    for m in ("MatmulFast", "Direct"):
        a = cb.magnetization_to_signal_sharded(ctx, comm, e, p, traj, w["coils"], method=m).to_numpy()
        assert np.array_equal(a, cb.magnetization_to_signal(ctx, e, p, traj, w["coils"], method=m).to_numpy()), m
    rng = np.random.default_rng(4)
    d = {"T1": W.cn(rng, (17, 81)), "T2": W.cn(rng, (17, 81))}
    v = W.cn(rng, (4, 81))
    for m in ("GemmFast", "Direct"):
        a = cb.compute_jacobian_sharded(ctx, comm, e, d, p, traj, w["coils"], v, method=m).to_numpy()
        assert np.array_equal(a, cb.compute_jacobian(ctx, e, d, p, traj, w["coils"], v, method=m).to_numpy()), m
    x = cb.CompasArray.from_numpy(ctx, W.cn(rng, (3, 5)))
    before = x.to_numpy()
    assert np.array_equal(comm.allreduce_sum(x).to_numpy(), before)


@pytest.mark.parametrize("world", [2, 3])
def test_library_shards_sum_to_the_whole_slice(one_rank, oracle, world):
    # the ranks' shares computed one after the other on one GPU (each rank's work depends on no
    # other rank's, so this runs nothing that waits): simulate + signal per voxel range of
    # compas_b200_voxel_shard, summed here, equal the whole slice's signal within FP32 rounding
    cb, ctx, _ = one_rank
    w = W.tiny(seed=10, n_side=11, ntr=19, ns=12, nc=3)
    V = w["params"].shape[1]
    seq = cb.FispSequence.from_dict(ctx, w["seq"])
    traj = cb.CartesianTrajectory.from_dict(ctx, w["traj"])
    total = 0
    for rank in range(world):
        b, e = cb.voxel_shard(V, rank, world)
        p = cb.TissueParameters.from_soa(ctx, np.ascontiguousarray(w["params"][:, b:e]))
        echo = cb.simulate_magnetization(ctx, p, seq)
        total = total + cb.magnetization_to_signal(ctx, echo, p, traj, np.ascontiguousarray(w["coils"][:, b:e]),
                                                   method="Direct").to_numpy().astype(np.complex128)
    ref = oracle.signal_cartesian(oracle.fisp(w["params"], w["seq"]), w["params"], w["traj"], w["coils"])
    assert oracle.rel_l2(total, ref) < 1e-5
