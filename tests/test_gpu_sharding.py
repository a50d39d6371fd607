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
