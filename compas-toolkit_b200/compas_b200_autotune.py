"""Autotuner for the simulation kernels' launch layouts and the tensor-core contractions' launches.

The FISP EPG kernel is instantiated for several register layouts — K states per lane × G lanes
per (voxel, slice position), and packed one-lane layouts that hold K states as K/2 pairs of
two-wide FP32 registers — and runs with W warps per CTA (W slice positions in flight per voxel
tile); the pSSFP kernel for ZT isochromats per lane × GZ lanes per voxel. The split-BF16
tensor-core contractions (Cartesian and spiral signal, J·v and Jᴴ·v) take a readout tile (the MMA
N of the Cartesian signal / J·v kernel) and a split count (voxel splits of the signal and J·v
kernels, pair-tile or readout splits of the Jᴴ·v kernels, each split's partial sums added
afterwards). Which choice is fastest depends on the shape. This script times the candidates on
the current GPU for a set of shape classes (the search spaces of the reference's kernel_tuner
scripts, tune_signal.py / tune_jacobian.py / tune_hermitian.py, restated for these kernels) and
writes the winners to a tuning table that the library reads from the file named by
COMPAS_B200_TUNING:

    fisp  <N> <log2 voxels> <log2 positions> <layout> <warps>
    pssfp <nz> <log2 voxels> <layout>
    tc    <kind> <log2 readouts> <log2 voxels> <log2 coils·samples> <tile> <splits>

Layouts change only the work distribution; the FISP echoes are the same bits for every layout and
warp count (slice positions are summed one at a time in increasing order). Tensor-core tiles and
splits change the FP32 order in which partial sums are added, within the split-BF16 tolerance.
The stage count of the tensor-core pipelines is not searched: each ring already takes the most
64 KB / 32 KB stages that fit the 227 KB of shared memory of a CTA.

    python compas-toolkit_b200/compas_b200_autotune.py --out tuning.txt [--quick] [--kinds tc]

With --kinds, only those kinds are tuned and the other kinds' lines of an existing --out table are
kept.
"""
from __future__ import annotations

import argparse
import math
import sys
import zlib
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))

import compas_b200 as cb  # noqa: E402
import workloads as W  # noqa: E402


def _time(ctx, fn, reps):
    import torch

    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    fn()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    ctx.synchronize()
    return e0.elapsed_time(e1) / reps


def _fisp_name(cfg):
    K, G = cb.fisp_configs()[cfg]
    return f"({K}, {G}{', packed' if cb.fisp_config_packed(cfg) else ''})"


def tune_fisp(ctx, N, nv, P, ntr, reps, warps=(4, 5, 6, 7, 8)):
    rng = np.random.default_rng(N * 1000 + P)
    params = cb.TissueParameters.from_soa(ctx, W.tissue_voxels(rng, nv, 22.4))
    seq = cb.FispSequence.from_dict(ctx, W.fisp_sequence(W.smooth_flip_train(rng, ntr),
                                                        W.gaussian_slice_profile(P, ntr), 8.7e-3, 4.35e-3,
                                                        25e-3, N))
    cb.set_fisp_launch(-1, -1)
    default = cb.fisp_launch_choice(N, nv, P)
    candidates = {default}
    for cfg, (K, G) in enumerate(cb.fisp_configs()):
        if K * G < N or K * G > max(2 * N, 32):
            continue
        for w in {min(P, w) for w in warps}:  # more warps than positions would idle
            candidates.add((cfg, w))
    results = []
    for cfg, w in sorted(candidates):
        cb.set_fisp_launch(cfg, w)
        ms = _time(ctx, lambda: cb.simulate_magnetization(ctx, params, seq), reps)
        results.append((ms, cfg, w))
    cb.set_fisp_launch(-1, -1)
    default_ms = next(ms for ms, cfg, w in results if (cfg, w) == default)
    return sorted(results), default, default_ms


def tune_pssfp(ctx, nz, nv, ntr, reps):
    rng = np.random.default_rng(nz)
    params = cb.TissueParameters.from_soa(ctx, W.tissue_voxels(rng, nv, 22.4))
    seq = cb.pSSFPSequence.from_dict(ctx, W.pssfp_sequence(rng, ntr, nrf=15, nz=nz))
    cb.set_pssfp_launch(-1)
    default = cb.pssfp_launch_choice(nz, nv)
    candidates = {default} | {cfg for cfg, (ZT, GZ) in enumerate(cb.pssfp_configs()) if nz <= ZT * GZ <= 2 * nz + 30}
    results = []
    for cfg in sorted(candidates):
        cb.set_pssfp_launch(cfg)
        ms = _time(ctx, lambda: cb.simulate_magnetization(ctx, params, seq), reps)
        results.append((ms, cfg))
    cb.set_pssfp_launch(-1)
    default_ms = next(ms for ms, cfg in results if cfg == default)
    return sorted(results), default, default_ms


# ---- tensor-core contractions --------------------------------------------------------------------
TC_SPLITS = (1, 2, 3, 4, 6, 8, 12, 16, 20, 24, 32, 40, 48, 64)


def _cn32(rng, shape):
    """complex normal CN(0,1) drawn in FP32 (large inputs without an FP64 intermediate)."""
    x = rng.standard_normal(tuple(shape) + (2,), dtype=np.float32) * np.float32(math.sqrt(0.5))
    return x.view(np.complex64).reshape(shape)


def _builtin_tile(R):
    """the library's built-in Cartesian readout tile: the fewest tiles of at most 256 readouts, then
    the least padding (a multiple of 16)"""
    r = max(R, 1)
    tiles = -(-r // 256)
    return -(-(-(-r // tiles)) // 16) * 16


def _tc_call(ctx, kind, nv, R, S, C, seed):
    """a closure running one split-BF16 contraction of `kind` on seeded inputs of this shape"""
    rng = np.random.default_rng(seed)
    params = cb.TissueParameters.from_soa(ctx, W.tissue_voxels(rng, nv, 22.4))
    if kind.startswith("cartesian"):
        traj = cb.CartesianTrajectory.from_dict(ctx, W.cartesian(R, S, 22.4, 5e-6, S))
    else:
        traj = cb.SpiralTrajectory.from_dict(ctx, W.spiral(rng, R, S, 22.4, 4e-6))
    coils = cb.CompasArray.from_numpy(ctx, _cn32(rng, (C, nv)))
    echo = cb.CompasArray.from_numpy(ctx, _cn32(rng, (R, nv)) * np.float32(0.1))
    if kind.endswith("signal"):
        return lambda: cb.magnetization_to_signal(ctx, echo, params, traj, coils, method="MatmulFast")
    d = {"T1": cb.CompasArray.from_numpy(ctx, _cn32(rng, (R, nv)) * np.float32(0.05)),
         "T2": cb.CompasArray.from_numpy(ctx, _cn32(rng, (R, nv)) * np.float32(0.5))}
    if kind.endswith("jacobian"):
        v = cb.CompasArray.from_numpy(ctx, _cn32(rng, (4, nv)))
        return lambda: cb.compute_jacobian(ctx, echo, d, params, traj, coils, v, method="GemmFast")
    r = cb.CompasArray.from_numpy(ctx, _cn32(rng, (C, R, S)))
    return lambda: cb.compute_jacobian_hermitian(ctx, echo, d, params, traj, coils, r, method="GemmFast")


def tune_tc(ctx, kind, nv, R, S, C, reps):
    """time every distinct (tile, splits) the library accepts for this shape; returns the sorted
    results [(ms, tile, splits)], the built-in choice and its time"""
    fn = _tc_call(ctx, kind, nv, R, S, C, seed=zlib.crc32(f"{kind} {nv} {R} {S} {C}".encode()))
    cb.set_tc_launch(kind, 0, 0)
    default = cb.tc_launch_choice(kind, nv, R, S, C)
    if kind in ("cartesian_signal", "cartesian_jacobian"):
        # tiles of at least 64 readouts that the library accepts for this R (≤ 17/16 of the rows of
        # the built-in tile), and the built-in tile
        pad = -(-R // _builtin_tile(R)) * _builtin_tile(R)
        tiles = sorted({t for t in range(64, 257, 16) if 16 * (-(-R // t) * t) <= 17 * pad} | {_builtin_tile(R)})
    else:
        tiles = [0]
    candidates = {default}
    for tile in tiles:
        for sp in TC_SPLITS:
            cb.set_tc_launch(kind, tile, sp)
            candidates.add(cb.tc_launch_choice(kind, nv, R, S, C))  # the launch it runs (clamped)
    results = []
    for tile, sp in sorted(candidates):
        cb.set_tc_launch(kind, tile, sp)
        results.append((_time(ctx, fn, reps), tile, sp))
    cb.set_tc_launch(kind, 0, 0)
    default_ms = next(ms for ms, t, sp in results if (t, sp) == default)
    return sorted(results), default, default_ms


# (kind, readouts, samples per readout, coils): the MR-STAT Cartesian slice (1120 readouts x 224
# samples, 4 and 8 coils) and the 760-interleave spiral of 1000 samples with 8 coils
TC_CLASSES = [("cartesian_signal", 1120, 224, 4), ("cartesian_signal", 1120, 224, 8),
              ("cartesian_jacobian", 1120, 224, 8), ("cartesian_hermitian", 1120, 224, 8),
              ("spiral_signal", 760, 1000, 8), ("spiral_jacobian", 760, 1000, 8),
              ("spiral_hermitian", 760, 1000, 8)]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True, help="tuning table to write")
    ap.add_argument("--quick", action="store_true", help="fewer shape classes (a smoke run)")
    ap.add_argument("--ntr", type=int, default=320, help="TRs of the timed sequences (cost is linear in it)")
    ap.add_argument("--kinds", default="fisp,pssfp,tc", help="comma-separated kinds to tune (fisp, pssfp, tc)")
    args = ap.parse_args(argv)
    kinds = {k.strip() for k in args.kinds.split(",") if k.strip()}
    ctx = cb.Context(0)
    voxel_classes = [4096, 50176] if args.quick else [4096, 16384, 50176, 200704]
    fisp_classes = [(8, 1), (25, 35)] if args.quick else [(8, 1), (8, 35), (16, 35), (25, 1), (25, 35), (32, 35)]
    lines, report = {k: [] for k in ("fisp", "pssfp", "tc")}, {k: [] for k in ("fisp", "pssfp", "tc")}
    out = Path(args.out)
    if out.exists():  # keep the lines of kinds not tuned now
        for line in out.read_text().splitlines():
            words = line.lstrip("# ").split()
            k = words[0] if words else ""
            if k in lines and k not in kinds:
                (report if line.startswith("#") else lines)[k].append(line)
    reps = 2 if args.quick else 3
    if "fisp" in kinds:
        for N, P in fisp_classes:
            for nv in voxel_classes:
                res, default, dms = tune_fisp(ctx, N, nv, P, args.ntr, reps=reps)
                ms, cfg, w = res[0]
                lines["fisp"].append(f"fisp {N} {int(math.log2(nv))} {int(math.log2(P))} {cfg} {w}")
                report["fisp"].append(f"# fisp N={N} P={P} V={nv}: best {_fisp_name(cfg)} W={w} {ms:.3f} ms; "
                                      f"built-in {_fisp_name(default[0])} W={default[1]} {dms:.3f} ms "
                                      f"({len(res)} candidates)")
    if "pssfp" in kinds:
        for nz in ([35] if args.quick else [9, 35]):
            for nv in voxel_classes:
                res, default, dms = tune_pssfp(ctx, nz, nv, args.ntr, reps=reps)
                ms, cfg = res[0]
                lines["pssfp"].append(f"pssfp {nz} {int(math.log2(nv))} {cfg}")
                report["pssfp"].append(f"# pssfp nz={nz} V={nv}: best {tuple(cb.pssfp_configs()[cfg])} {ms:.3f} ms; "
                                       f"built-in {tuple(cb.pssfp_configs()[default])} {dms:.3f} ms "
                                       f"({len(res)} candidates)")
    if "tc" in kinds:
        tc_voxels = [4096, 50176] if args.quick else [4096, 16384, 50176]
        for kind, R, S, C in (TC_CLASSES[:1] + TC_CLASSES[3:5] if args.quick else TC_CLASSES):
            for nv in tc_voxels:
                res, default, dms = tune_tc(ctx, kind, nv, R, S, C, reps=reps)
                ms, tile, sp = res[0]
                # a line only where the search beats the built-in choice by more than 2 %: a table
                # line applies to a whole class of shapes, the built-in plan to the exact one
                if dms > 1.02 * ms:
                    lines["tc"].append(f"tc {cb.TC_KINDS[kind]} {int(math.log2(R))} {int(math.log2(nv))} "
                                       f"{int(math.log2(C * S))} {tile} {sp}")
                report["tc"].append(f"# tc {kind} R={R} S={S} C={C} V={nv}: best (tile {tile}, splits {sp}) "
                                    f"{ms:.3f} ms; built-in (tile {default[0]}, splits {default[1]}) {dms:.3f} ms "
                                    f"({len(res)} candidates)")
    order = ("fisp", "pssfp", "tc")
    text = [l for k in order for l in report[k]] + [l for k in order for l in lines[k]]
    out.write_text("\n".join(text) + "\n")
    print("\n".join(l for k in order if k in kinds for l in report[k]))
    return 0


if __name__ == "__main__":
    sys.exit(main())
