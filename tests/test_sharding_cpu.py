"""Voxel sharding over torch.distributed ranks: partition, sum of the partial signals and J·v,
gather of the per-voxel Jᴴ·r — run as world_size-2 gloo ranks on CPU with the oracle as each
rank's compute, against the oracle on the whole slice.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "compas-toolkit_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

from sharding import VoxelShard  # noqa: E402


def test_shards_partition_the_voxels():
    for nv in (0, 1, 7, 36, 50176):
        for world in (1, 2, 3, 8):
            shards = [VoxelShard(nv, r, world) for r in range(world)]
            assert shards[0].begin == 0 and shards[-1].end == nv
            assert all(a.end == b.begin for a, b in zip(shards, shards[1:]))
            sizes = [s.size for s in shards]
            assert max(sizes) - min(sizes) <= 1 and sum(sizes) == nv


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT / "compas-toolkit_b200"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    import workloads as W
    from sharding import VoxelShard, allreduce_sum, gather_voxels, sharded_signal

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = W.tiny(seed=7, n_side=7, ntr=11, ns=6, nc=3)  # 49 voxels: shards of 25 and 24
        params, seq, traj, coils = w["params"], w["seq"], w["traj"], w["coils"]
        V = params.shape[1]
        shard = VoxelShard(V, rank, world)
        to_t = lambda a: torch.view_as_real(torch.from_numpy(np.ascontiguousarray(a, np.complex128)))

        # signal: per-rank simulate + contract of its voxels, summed over the ranks
        def partial(p, c, _):
            return O.signal_cartesian(O.fisp(p, seq), p, traj, c)

        s = torch.view_as_complex(sharded_signal(shard, partial, params, coils, None, to_t)).numpy()
        echo = O.fisp(params, seq)
        ref = O.signal_cartesian(echo, params, traj, coils)
        assert O.rel_l2(s, ref) < 1e-12

        # J·v: sum over voxels as well
        rng = np.random.default_rng(3)
        dT1 = W.cn(rng, echo.shape).astype(np.complex128)
        dT2 = W.cn(rng, echo.shape).astype(np.complex128)
        v = W.cn(rng, (4, V)).astype(np.complex128)
        loc = lambda a: shard.take(a)
        jv = O.jacobian(loc(echo), loc(dT1), loc(dT2), loc(params), traj, loc(coils), loc(v))
        jv = torch.view_as_complex(allreduce_sum(to_t(jv))).numpy()
        assert O.rel_l2(jv, O.jacobian(echo, dT1, dT2, params, traj, coils, v)) < 1e-12

        # Jᴴ·r: every rank has the full r and produces its voxels; gathered in rank order
        r = W.cn(rng, s.shape).astype(np.complex128)
        jh = O.jacobian_hermitian(loc(echo), loc(dT1), loc(dT2), loc(params), traj, loc(coils), r)
        full = torch.view_as_complex(_gather_complex(jh, shard, torch, gather_voxels)).numpy()
        assert full.shape == (4, V)
        assert O.rel_l2(full, O.jacobian_hermitian(echo, dT1, dT2, params, traj, coils, r)) < 1e-12
    finally:
        dist.destroy_process_group()


def _gather_complex(jh, shard, torch, gather_voxels):
    # the voxel axis must stay last: gather re and im parts separately
    re = gather_voxels(torch.from_numpy(np.ascontiguousarray(jh.real)), shard)
    im = gather_voxels(torch.from_numpy(np.ascontiguousarray(jh.imag)), shard)
    return torch.view_as_real(torch.complex(re, im))


def test_two_gloo_ranks_match_the_whole_slice():
    import torch.multiprocessing as mp

    pytest.importorskip("torch")
    port = _free_port()
    mp.start_processes(_rank, args=(2, port), nprocs=2, join=True, start_method="spawn")
