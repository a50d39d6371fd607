"""Autotuner for the simulation kernels' launch layouts.

The FISP EPG kernel is instantiated for several register layouts — K states per lane × G lanes
per (voxel, slice position), and packed one-lane layouts that hold K states as K/2 pairs of
two-wide FP32 registers — and runs with W warps per CTA (W slice positions in flight per voxel
tile); the pSSFP kernel for ZT isochromats per lane × GZ lanes per voxel. Which layout is
fastest depends on the number of states / z positions, the voxel count and the slice positions.
This script times every covering layout on the current GPU for a set of shape classes and writes
the winners to a tuning table that the library reads from the file named by COMPAS_B200_TUNING:

    fisp  <N> <log2 voxels> <log2 positions> <layout> <warps>
    pssfp <nz> <log2 voxels> <layout>

Layouts change only the work distribution; the FISP echoes are the same bits for every layout and
warp count (slice positions are summed one at a time in increasing order).

    python compas-toolkit_b200/compas_b200_autotune.py --out tuning.txt [--quick]
"""
from __future__ import annotations

import argparse
import math
import sys
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


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True, help="tuning table to write")
    ap.add_argument("--quick", action="store_true", help="fewer shape classes (a smoke run)")
    ap.add_argument("--ntr", type=int, default=320, help="TRs of the timed sequences (cost is linear in it)")
    args = ap.parse_args(argv)
    ctx = cb.Context(0)
    voxel_classes = [4096, 50176] if args.quick else [4096, 16384, 50176, 200704]
    fisp_classes = [(8, 1), (25, 35)] if args.quick else [(8, 1), (8, 35), (16, 35), (25, 1), (25, 35), (32, 35)]
    lines, report = [], []
    for N, P in fisp_classes:
        for nv in voxel_classes:
            res, default, dms = tune_fisp(ctx, N, nv, P, args.ntr, reps=2 if args.quick else 3)
            ms, cfg, w = res[0]
            lines.append(f"fisp {N} {int(math.log2(nv))} {int(math.log2(P))} {cfg} {w}")
            report.append(f"# fisp N={N} P={P} V={nv}: best {_fisp_name(cfg)} W={w} {ms:.3f} ms; "
                          f"built-in {_fisp_name(default[0])} W={default[1]} {dms:.3f} ms ({len(res)} candidates)")
    for nz in ([35] if args.quick else [9, 35]):
        for nv in voxel_classes:
            res, default, dms = tune_pssfp(ctx, nz, nv, args.ntr, reps=2 if args.quick else 3)
            ms, cfg = res[0]
            lines.append(f"pssfp {nz} {int(math.log2(nv))} {cfg}")
            report.append(f"# pssfp nz={nz} V={nv}: best {tuple(cb.pssfp_configs()[cfg])} {ms:.3f} ms; built-in "
                          f"{tuple(cb.pssfp_configs()[default])} {dms:.3f} ms ({len(res)} candidates)")
    Path(args.out).write_text("\n".join(report + lines) + "\n")
    print("\n".join(report))
    return 0


if __name__ == "__main__":
    sys.exit(main())
