"""Voxel sharding of the simulation hot path over torch.distributed ranks (one GPU per rank).

Every operation of the path is either independent per voxel (simulation, derivatives, Jᴴ·v) or a
sum over voxels (signal, J·v). So a slice is split into contiguous voxel ranges, one per rank:

* signal and J·v: each rank contracts its voxels into a partial [C][R][S] and one all-reduce
  (sum) over the ranks forms the full result (NCCL over NVLink on GPUs);
* Jᴴ·r: each rank needs the full residual r (identical on every rank after the all-reduce) and
  produces its own voxels of [4][V]; `gather_voxels` assembles the full vector when needed.

This mirrors the reference's chunking of voxels across devices with a summing reduction of the
signal (src/trajectories/signal.cu:289-300, compas/core/context.h:51-68). The partition is the
library's (compas_b200_voxel_shard, host code); on GPUs the library's own NCCL communicator sums
the partials (compas_b200_magnetization_to_signal_sharded / _compute_jacobian_sharded, see
`library_communicator`). The functions below also take the per-rank compute as callables with
torch.distributed for the sum, so the same partition and reduction run on CPU ranks (gloo) with a
CPU restatement as the compute.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class VoxelShard:
    """Contiguous voxel range [begin, end) of `rank` among `world` ranks (sizes differ by ≤ 1)."""

    nvoxels: int
    rank: int
    world: int

    @property
    def begin(self) -> int:
        return _library_range(self.nvoxels, self.rank, self.world)[0]

    @property
    def end(self) -> int:
        return _library_range(self.nvoxels, self.rank, self.world)[1]

    @property
    def size(self) -> int:
        return self.end - self.begin

    def take(self, a: np.ndarray) -> np.ndarray:
        """This rank's voxels of an array whose last axis is the voxel axis (tissue [9][V],
        coils [C][V], echoes [R][V], J·v input [4][V])."""
        return np.ascontiguousarray(a[..., self.begin:self.end])

    def counts(self) -> list:
        return [VoxelShard(self.nvoxels, r, self.world).size for r in range(self.world)]


def _library_range(nvoxels: int, rank: int, world: int) -> tuple:
    import compas_b200

    return compas_b200.voxel_shard(nvoxels, rank, world)


def library_communicator(cb, ctx, rank: int, world: int, group=None):
    """The library's NCCL communicator for this rank: rank 0 makes the unique id and
    torch.distributed broadcasts it (any backend), then every rank joins."""
    import torch
    import torch.distributed as dist

    uid = torch.zeros(128, dtype=torch.uint8)
    if rank == 0:
        uid = torch.frombuffer(bytearray(cb.comm_unique_id()), dtype=torch.uint8).clone()
    if world > 1:
        if dist.get_backend(group) == "nccl":
            uid = uid.cuda()
        dist.broadcast(uid, src=0, group=group)
    return cb.Communicator(ctx, rank, world, bytes(uid.cpu().numpy().tobytes()))


def allreduce_sum(tensor, group=None):
    """Sum a partial signal / J·v over the ranks in place (torch.distributed, NCCL or gloo)."""
    import torch.distributed as dist

    dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor


def gather_voxels(local, shard: VoxelShard, group=None):
    """Assemble [..., V] from every rank's [..., V_rank] (torch tensors on the backend's device)."""
    import torch
    import torch.distributed as dist

    counts = shard.counts()
    width = max(counts)
    pad = torch.zeros(local.shape[:-1] + (width,), dtype=local.dtype, device=local.device)
    pad[..., :local.shape[-1]] = local
    parts = [torch.empty_like(pad) for _ in counts]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[..., :c] for p, c in zip(parts, counts)], dim=-1)


def sharded_signal(shard: VoxelShard, partial_signal, params: np.ndarray, coils: np.ndarray, echos_or_none,
                   to_tensor, group=None):
    """Full signal [C][R][S] on every rank: `partial_signal(params_local, coils_local, echos_local)`
    contracts this rank's voxels (echos_local is None when the callable simulates them itself);
    `to_tensor` turns its result into a torch tensor on the collective's device."""
    local = partial_signal(shard.take(params), shard.take(coils),
                           None if echos_or_none is None else shard.take(echos_or_none))
    return allreduce_sum(to_tensor(local), group)


def gpu_partial_signal(cb, ctx, sequence, trajectory, method: str = "MatmulFast"):
    """Per-rank compute for `sharded_signal` on the GPU library: simulate this rank's voxels and
    contract them; returns the device array (view it with torch.as_tensor(..., device="cuda"))."""

    def fn(params_local, coils_local, echos_local):
        p = cb.TissueParameters.from_soa(ctx, params_local)
        e = cb.simulate_magnetization(ctx, p, sequence) if echos_local is None else echos_local
        return cb.magnetization_to_signal(ctx, e, p, trajectory, coils_local, method=method)

    return fn


def gpu_to_tensor(ctx):
    """`to_tensor` for `sharded_signal` on the GPU library: a torch copy of the library array on
    torch's current stream, ordered after the context's stream that produced it (the collective
    then runs on torch's stream)."""
    import torch

    def fn(arr):
        lib_stream = torch.cuda.ExternalStream(ctx.stream)
        torch.cuda.current_stream().wait_stream(lib_stream)
        view = torch.as_tensor(arr, device="cuda")  # zero-copy float32 view [..., 2] of the buffer
        out = view.clone()
        # the library releases `arr` on its own stream: order that after the copy
        lib_stream.wait_stream(torch.cuda.current_stream())
        return out

    return fn

