"""Benchmark of the compas-toolkit simulation hot path on B200.

One step = one MR-STAT-scale forward pass: FISP EPG simulate_magnetization (224×224
voxels, 1120 TRs, 25 states, 35 slice positions) followed by magnetization_to_signal
(4 coils, Cartesian 1120×224) on the split-BF16 tensor-core path (the C ABI's
default method), inputs resident in HBM. The metric is EPG voxel·TR/s (voxels × TRs
per step ÷ step time, whole job over all ranks); the signal and, optionally, the
Jᴴ·v product are reported beside it in TFLOP/s.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) the one slice is sharded over the ranks (strong scaling): each rank
takes its voxel range (compas_b200_voxel_shard), simulates it and contracts it into a partial
signal, and the library's NCCL communicator sums the partials, so every rank ends the step with
the full signal (compas_b200_magnetization_to_signal_sharded; the all-reduce is inside the timed
region). Timing is device-side (CUDA events on the library's stream), max over ranks. The
secondary blocks (Jacobian products, batches, Gauss-Newton, serving, CPU baseline) run on the
single-GPU run only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "compas-toolkit_b200"))

METRIC = "EPG voxel·TR/s"
# FMA-pipe lane operations the FISP kernel executes per (voxel, slice position, TR): every state
# slot of the layout takes 26 one-wide operations for the excitation update (24 in the real-phase
# form of the packed layouts, without the d_re products), and every lane 56 more for the per-TR
# coefficients, dephasing moves and sample (ncu, profiles/fisp_epg_mrstat.txt: 732 for the 26-slot
# packed layout in the general form)
FISP_LANE_OPS_PER_LANE = 56


def fisp_lane_ops_per_item(cb, N, V, P, real_phases):
    cfg, _ = cb.fisp_launch_choice(N, V, P)
    K, G = cb.fisp_configs()[cfg]
    per_slot = 24 if real_phases and cb.fisp_config_packed(cfg) else 26
    return K * G * per_slot + G * FISP_LANE_OPS_PER_LANE, f"{K}x{G}{' packed' if cb.fisp_config_packed(cfg) else ''}"


UNIT = "voxel·TR/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "sm_max_mhz": 1965.0}


def load_peaks():
    try:
        return json.loads(PEAKS_FILE.read_text()), "measured"
    except Exception:
        return FALLBACK_PEAKS, "fallback"


def profile_traffic(name):
    """DRAM bytes per launch from a committed ncu summary (profiles/<name>.txt, line
    'dram_bytes_per_launch: <n>'), or None."""
    p = ROOT / "profiles" / f"{name}.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.window = (0, None)  # the lines sampled inside the timed region (mark_start / mark_end)

    def _lines(self):
        try:
            return Path(self.path).read_text().count("\n")
        except OSError:
            return 0

    def mark_start(self):
        self.window = (self._lines(), None)

    def mark_end(self):
        # the sample in flight when the region ends belongs to it too
        time.sleep(0.25)
        self.window = (self.window[0], self._lines())

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-i", str(self.gpu),
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # start timing only once nvidia-smi has been polling for a while: its start-up (NVML
        # initialisation) and its first queries occupy the NVIDIA kernel driver for up to a second,
        # and a driver call of the timed steps that waits on it leaves the GPU idle (a 0.5 s stall
        # in one step was seen with timing started after the first sample)
        deadline = time.perf_counter() + 5.0
        while self.proc is not None and time.perf_counter() < deadline and self._lines() < 4:
            time.sleep(0.05)
        time.sleep(0.1)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            lines = Path(self.path).read_text().splitlines()
            lo, hi = self.window
            timed = lines[lo:hi] if hi is not None and hi > lo else lines[lo:]
            for line in timed or lines[-1:]:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def cpu_forward_rate(w, nv_sample=2048, ne_sample=64):
    """One forward step (FISP simulation + Cartesian signal) on the host cores, timed on a fixed
    sample — `nv_sample` voxels evenly spaced over the slice for the simulation and `ne_sample`
    signal entries (each a sum over all voxels) — and extrapolated to the full step; both arms of
    the bench use the same sample. Runs the reference's own kernels compiled for the host
    (oracle/_ref/libref_kernels.so: simulate_fisp, sum_signal_cartesian_naive) where they were
    built, else the oracle's FP32 restatement of the reference arithmetic."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    threads = oracle.nthreads_default()
    ref = oracle.ref_kernels() is not None
    if ref:
        sim = lambda idx: oracle.ref_fisp(w["params"], w["seq"], vidx=idx, nthreads=threads)  # noqa: E731
        sig = lambda e, ent: oracle.ref_signal_cartesian(e, w["params"], w["traj"], w["coils"], ent,  # noqa: E731
                                                         nthreads=threads)
    else:
        sim = lambda idx: oracle.fisp(w["params"], w["seq"], vidx=idx, dtype="f32", nthreads=threads)  # noqa: E731
        sig = lambda e, ent: oracle.signal_cartesian(e, w["params"], w["traj"], w["coils"], entries=ent,  # noqa: E731
                                                     dtype="f32", nthreads=threads)
    V = w["params"].shape[1]
    nTR = len(w["seq"]["rf"])
    C_, R, S = w["coils"].shape[0], w["traj"]["nr"], w["traj"]["ns"]
    nv = min(V, nv_sample)
    idx = np.arange(nv) * (V // nv)
    t0 = time.perf_counter()
    sim(idx)
    t_sim = time.perf_counter() - t0
    per_voxel = t_sim / nv
    # signal: a few entries, each a full sum over all voxels
    ne = ne_sample
    rng = np.random.default_rng(0)
    ent = np.stack([rng.integers(0, C_, ne), rng.integers(0, R, ne), rng.integers(0, S, ne)], 1)
    echo_full = np.zeros((R, V), np.complex64)
    echo_full[:, :] = 0.01
    t0 = time.perf_counter()
    sig(echo_full, ent)
    t_sig = time.perf_counter() - t0
    per_entry = t_sig / ne
    full = per_voxel * V + per_entry * C_ * R * S
    what = ("the reference's simulate_fisp and sum_signal_cartesian_naive kernels built for the host "
            "(oracle/_ref/libref_kernels.so)" if ref else "oracle FP32 twin")
    return {"value": V * nTR / full, "unit": UNIT, "cores": threads, "kind": "reference" if ref else "port",
            "sample": f"{what}: FISP on a fixed sample of {nv} of {V} voxels ({100.0 * nv / V:.1f} %, {t_sim:.1f} s) "
                      f"+ signal on {ne} of {C_ * R * S} entries, each summed over all {V} voxels ({t_sig:.1f} s); "
                      f"extrapolated to one full forward step ({full:.0f} s)"}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    import workloads

    w = workloads.mrstat()
    per_step = []
    base = None
    for i in range(args.warmup + args.steps):
        r = cpu_forward_rate(w)
        if i >= args.warmup:
            per_step.append(r["value"])
            base = r
    val = statistics.median(per_step)
    line = {"metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "mrstat 224x224 voxels, FISP 1120 TR / 25 states / 35 positions, 4 coils, "
                                   "Cartesian 1120x224", "parallelism": "host threads"},
            "cpu_baseline": dict(base, value=val),
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU implementation and its GPU build needs the absent kmm runtime: "
                    "this arm runs its own FISP and signal kernels compiled for the host "
                    "(one-thread launches, OpenMP over voxels / entries) when oracle/_ref was built, else the "
                    "oracle's FP32 restatement"}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-jacobian", action="store_true", help="skip the J·v / Jᴴ·v measurements")
    ap.add_argument("--no-reference-kernels", action="store_true",
                    help="skip timing the reference's own kernels built for the GPU")
    ap.add_argument("--no-gn", action="store_true", help="skip the Gauss-Newton iteration timings")
    ap.add_argument("--serve-rates", default="2,4,8",
                    help="Poisson arrival rates (requests/s) of the served stream, empty to skip")
    ap.add_argument("--serve-requests", type=int, default=32, help="requests per arrival rate")
    ap.add_argument("--batch-jobs", type=int, default=256,
                    help="jobs of the batched uneven workload (0 skips it)")
    ap.add_argument("--batch-vmax", type=int, default=64000,
                    help="largest voxel count of a batched job (smaller values for profiler captures)")
    ap.add_argument("--tangent-layout", type=int, default=-1,
                    help="FISP tangent layout index for the derivatives block (-1: the built-in choice; "
                         "for profiler comparisons of layouts)")
    ap.add_argument("--n-side", type=int, default=224,
                    help="voxel grid side (224 = the MR-STAT workload; smaller values for profiler captures)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    # launch layouts from the committed autotuner table (compas_b200_autotune.py) unless the
    # caller names another one
    table = Path(__file__).resolve().parent / "compas-toolkit_b200" / "tuning" / "b200.txt"
    if "COMPAS_B200_TUNING" not in os.environ and table.exists():
        os.environ["COMPAS_B200_TUNING"] = str(table)

    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import compas_b200 as cb
    import workloads

    peaks, peak_kind = load_peaks()
    w = workloads.mrstat(seed=2, n_side=args.n_side)
    V = w["params"].shape[1]
    nTR = len(w["seq"]["rf"])
    P, N = w["seq"]["slices"].shape[0], w["seq"]["max_state"]
    C_, R, S = w["coils"].shape[0], w["traj"]["nr"], w["traj"]["ns"]
    # this rank's voxels of the slice (all of them on one GPU)
    vb, ve = cb.voxel_shard(V, rank, world)
    p_local = np.ascontiguousarray(w["params"][:, vb:ve])
    c_local = np.ascontiguousarray(w["coils"][:, vb:ve])

    ctx = cb.Context(local)
    params = cb.TissueParameters.from_soa(ctx, p_local)
    seq = cb.FispSequence.from_dict(ctx, w["seq"])
    traj = cb.CartesianTrajectory.from_dict(ctx, w["traj"])
    coils = cb.CompasArray.from_numpy(ctx, c_local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    comm = None
    if world > 1:
        from sharding import library_communicator

        comm = library_communicator(cb, ctx, rank, world)

    def signal_of(e, p, c):
        if comm is None:
            return cb.magnetization_to_signal(ctx, e, p, traj, c)
        return cb.magnetization_to_signal_sharded(ctx, comm, e, p, traj, c)  # partials summed by NCCL

    def step(events=None):
        if events:
            events[0].record(stream)
        e = cb.simulate_magnetization(ctx, params, seq)
        if events:
            events[1].record(stream)
        s = signal_of(e, params, coils)
        if events:
            events[2].record(stream)
        return e, s

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(local)
        ctx.synchronize()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    keep = []
    # the clock sampler polls from before the warm-up on, so that its start-up is over before the
    # timed steps; its summary covers the samples taken between mark_start and mark_end
    with ClockSampler(local) as clk:
        # the warm-up keeps results alive as the timed loop does (the last step's while the next
        # one allocates), so that the memory pool has grown to two steps' worth before the timed
        # region: growing it there maps memory and stalled a timed step by 225 ms
        warm = []
        for _ in range(args.warmup):
            warm.append(step())
            if len(warm) > 1:
                warm.pop(0)
        ctx.synchronize()
        warm.clear()
        barrier()
        clk.mark_start()
        launches0 = cb.launch_count()
        t_start.record(stream)
        for i in range(args.steps):
            keep.append(step(evs[i]))
            if len(keep) > 1:
                keep.pop(0)
        t_end.record(stream)
        barrier()
        launches = cb.launch_count() - launches0
        clk.mark_end()
    last_signal = keep[-1][1] if keep else None
    keep.clear()
    total_ms = t_start.elapsed_time(t_end)
    sim_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    sig_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    ms_step = total_ms / args.steps
    if world > 1:
        t = torch.tensor([ms_step], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_step = float(t.item())
    value = V * nTR / (ms_step / 1e3)  # the whole slice per step, over all ranks
    clocks = clk.summary()

    # roofline of the dominant kernel (FISP EPG): FP32-SIMT bound, 86·N·P flops per voxel·TR
    f_mhz = clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    fp32_peak_tf = 148 * 128 * 2 * f_mhz * 1e6 / 1e12
    Vl = ve - vb  # voxels this rank simulates
    epg_flops = 86.0 * N * P * Vl * nTR
    epg_tf = epg_flops / (sim_ms / 1e3) / 1e12
    # the FP32 work the kernel executes: FMA-pipe lane operations per (voxel, slice position, TR),
    # measured by ncu on the packed 26-slot layout (profiles/fisp_epg_mrstat.txt: FMA pipe busy
    # cycles x 32 lanes / (voxels x positions x TRs)); against 148 SM x 128 lanes per cycle
    # the kernel's form: real phases (sin φ = 0 for every RF sample times slice profile, as the table
    # kernel computes it in FP64) run the update without the d_re products
    seqd = w["seq"]
    real_phases = not np.any(np.imag(np.asarray(seqd["slices"], np.complex128)
                                     * np.asarray(seqd["rf"], np.complex128)[None, :]))
    per_item, layout = fisp_lane_ops_per_item(cb, N, Vl, P, real_phases)
    lane_ops = per_item * P * Vl * nTR
    exec_frac = lane_ops / (sim_ms / 1e3) / (148 * 128 * f_mhz * 1e6)
    roofline = {"bound": "fp32", "kernel": "fisp_epg_kernel", "achieved": epg_tf, "peak": fp32_peak_tf,
                "unit": "TFLOP/s", "frac": epg_tf / fp32_peak_tf,
                "traffic": profile_traffic("fisp_epg_mrstat"),
                "executed": {"fp32_lane_ops_per_voxel_position_tr": per_item, "layout": layout,
                             "real_phase_form": real_phases,
                             "fp32_lane_ops": lane_ops, "frac_of_fp32_peak": exec_frac},
                "note": f"FP32 SIMT peak 148 SM x 128 lanes x 2 x {f_mhz:.0f} MHz (median SM clock under load). "
                        "achieved/frac count the reference formulation's 86·N·P flops per voxel·TR; the kernel "
                        f"executes {24 if real_phases else 26} FP32 operations per EPG state and TR where that "
                        "formulation has 48, so frac can pass 1. executed.frac_of_fp32_peak is the FP32 work actually "
                        "issued (FMA-pipe lane operations, two per FFMA2) over the FP32 peak. HBM is not binding "
                        "(8 B written per voxel·TR)"}
    # the HBM fraction beside it: algorithmic bytes = echoes written (8 B per voxel·readout) + the
    # nine parameter rows read (36 B per voxel)
    epg_bytes = 8.0 * Vl * nTR + 36.0 * Vl
    roofline["hbm"] = {"achieved_gbs": epg_bytes / (sim_ms / 1e3) / 1e9, "peak_gbs": peaks["hbm_gbs"],
                       "frac": epg_bytes / (sim_ms / 1e3) / 1e9 / peaks["hbm_gbs"]}
    sig_flops = 8.0 * C_ * R * S * Vl
    sig_tf = sig_flops / (sig_ms / 1e3) / 1e12
    roofline_signal = {"bound": "tensor", "kernel": "signal (split-BF16 tcgen05)", "achieved": sig_tf,
                       "peak": peaks["bf16_tflops_sustained"], "unit": "TFLOP/s",
                       "frac": sig_tf / peaks["bf16_tflops_sustained"], "traffic": profile_traffic("cartesian_contraction_pairs_mrstat160"),
                       "note": f"algorithmic 8·C·R·S·V flops; split-BF16 issues 3 BF16 MMAs per product, so the "
                               f"attainable algorithmic rate is 1/3 of the BF16 peak ({peak_kind})"}
    # algorithmic bytes: echoes read (8·R·V), coils and parameters (8·C·V + 36·V), signal written (8·C·R·S)
    sig_bytes = 8.0 * R * Vl + 8.0 * C_ * Vl + 36.0 * Vl + 8.0 * C_ * R * S
    roofline_signal["frac_of_split_bf16_ceiling"] = sig_tf / (peaks["bf16_tflops_sustained"] / 3)
    roofline_signal["hbm"] = {"achieved_gbs": sig_bytes / (sig_ms / 1e3) / 1e9, "peak_gbs": peaks["hbm_gbs"],
                              "frac": sig_bytes / (sig_ms / 1e3) / 1e9 / peaks["hbm_gbs"]}

    # FP64 error of the step's split-BF16 signal against the oracle on 256 entries, each summed over
    # this rank's voxels with the GPU's own echoes (outside the timed region; one GPU only)
    signal_err = None
    if world == 1 and last_signal is not None:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle

        e_host = cb.simulate_magnetization(ctx, params, seq).to_numpy()
        rng = np.random.default_rng(5)
        ent = np.stack([rng.integers(0, C_, 256), rng.integers(0, R, 256), rng.integers(0, S, 256)], 1)
        ref = oracle.signal_cartesian(e_host, p_local, w["traj"], c_local, entries=ent)
        got = last_signal.to_numpy()[ent[:, 0], ent[:, 1], ent[:, 2]]
        signal_err = oracle.rel_l2(got, ref)
        del e_host
    roofline_signal["rel_err_fp64"] = signal_err
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "fp32 (EPG), bf16x3->fp32 (signal)", "data": "synthetic",
           "config": {"workload": f"mrstat: {args.n_side}x{args.n_side}={V} voxels, FISP 1120 TR, 25 EPG states, "
                                  f"35 slice positions, 4 coils, Cartesian 1120x{args.n_side} readouts; the one "
                                  "slice sharded over the GPUs",
                      "parallelism": (f"voxel shards over {world} ranks ({ve - vb} voxels on rank {rank}), NCCL "
                                      "all-reduce of the partial signal inside the step" if world > 1 else
                                      "one GPU"),
                      "l2": "working set > L2 (echo array 450 MB per step)", "seed": 2},
           "gpu_launches": launches, "clocks": clocks, "roofline": roofline, "roofline_signal": roofline_signal,
           "stage_ms": {"simulate_fisp": sim_ms, "signal_cartesian": sig_ms},
           "stage_ms_per_step": {"simulate_fisp": [round(e[0].elapsed_time(e[1]), 3) for e in evs],
                                 "signal_cartesian": [round(e[1].elapsed_time(e[2]), 3) for e in evs]},
           "signal_tflops": sig_tf, "peaks": peak_kind}

    single = world == 1
    if single and not args.no_reference_kernels:
        out["reference_kernels_gpu"] = reference_kernels_gpu(cb, ctx, stream, w, sim_ms, args)
    if single and not args.no_jacobian:
        out["jacobian"] = jacobian_products(cb, ctx, stream, args, peaks, rank)
    if single and args.batch_jobs > 0:
        out["batched"] = batched(cb, ctx, stream, args, rank)
    if single:
        out["elementwise"] = elementwise(cb, ctx, stream, w, params, seq, traj, peaks)
    if single and not args.no_gn:
        out["derivatives"] = derivatives(cb, ctx, stream, args, rank)
        out["gauss_newton"] = gauss_newton(cb, ctx, stream, args, rank)
    if single and args.serve_rates:
        out["served"] = served(cb, ctx, args)
    if not args.no_e2e:
        out["e2e"] = e2e(cb, ctx, w, args, local, (vb, ve), signal_of, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_forward_rate(w)
    if world > 1:
        torch.distributed.barrier()
        del comm
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


def batched(cb, ctx, stream, args, rank):
    """Uneven independent jobs (V logU[1k,64k], nTR U{400..1120}, C U{1..16}, FISP/pSSFP and
    Cartesian/spiral 50/50) through one SimulationBatch — persistent work-queue simulation
    kernels and batched signal kernels — against the same jobs as one call chain each."""
    import torch
    import workloads

    dicts = workloads.batch_jobs(seed=4 + rank, njobs=args.batch_jobs, vmax=args.batch_vmax)
    jobs = [cb.job_from_dict(ctx, d) for d in dicts]
    batch = cb.SimulationBatch(ctx, jobs)
    vtr = sum(d["nvoxels"] * d["ntr"] for d in dicts)
    flops = {"cartesian": 0.0, "spiral": 0.0}
    for d in dicts:
        flops[d["traj"]["kind"]] += 8.0 * d["ncoils"] * d["traj"]["nr"] * d["traj"]["ns"] * d["nvoxels"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch.run()  # warm-up
    ctx.synchronize()
    n0 = cb.launch_count()
    e0.record(stream)
    batch.run()
    e1.record(stream)
    ctx.synchronize()
    launches = cb.launch_count() - n0
    t_batch = e0.elapsed_time(e1)

    def one_by_one():
        for j, (params, seq, traj, _) in enumerate(jobs):
            e = cb.simulate_magnetization(ctx, params, seq)
            if traj is not None:
                cb.magnetization_to_signal(ctx, e, params, traj, batch.coil_arrays[j])

    one_by_one()  # warm-up
    ctx.synchronize()
    e0.record(stream)
    one_by_one()
    e1.record(stream)
    ctx.synchronize()
    t_seq = e0.elapsed_time(e1)
    kinds = {}
    for d in dicts:
        key = f'{d["kind"]}+{d["traj"]["kind"]}'
        kinds[key] = kinds.get(key, 0) + 1
    return {"workload": f"{len(dicts)} jobs: voxels logU[1k,{args.batch_vmax}], TRs U{{400..1120}}, coils U{{1..16}}, FISP (25 "
                        "states, 35 positions) or pSSFP (35 z, 15 RF samples), Cartesian (S=sqrt V) or spiral "
                        f"(TRs x 1000), seed {4 + rank}",
            "mix": kinds, "voxel_tr": vtr, "batch_ms": t_batch, "voxel_tr_per_s": vtr / (t_batch / 1e3),
            "signal_flops": flops, "gpu_launches": launches, "one_call_chain_per_job_ms": t_seq,
            "speedup_vs_one_call_chain_per_job": t_seq / t_batch,
            "note": "simulation: one persistent work-queue launch per kernel layout (FISP and pSSFP families on "
                    "two streams); signal: one batched launch per kind and family; results bit-identical to "
                    "the one-job calls"}


def served(cb, ctx, args):
    """Served request stream: Poisson arrivals at each rate of reconstruction requests (simulate,
    FD derivative simulations — or one exact tangent pass in the delta = 0 run — signal, residual,
    Jᴴ·r) drawn from 12
    distinct requests (voxels logU[4k,200k], coils U{4..16}, FISP/pSSFP, Cartesian/spiral, TRs
    U{400..1120}) whose sequences, trajectories, coils and data stay resident; HBM budget 150 GB.
    Latency = submit -> results complete on the device, measured by the engine."""
    import threading
    import time

    import numpy as np
    import workloads

    dicts = workloads.serve_requests(seed=5, n=12)
    objs = []
    for d in dicts:
        p, s, t, _ = cb.job_from_dict(ctx, d)
        objs.append((p, s, t, cb.CompasArray.from_numpy(ctx, d["coils"]), cb.CompasArray.from_numpy(ctx, d["data"])))
    vtr = [d["nvoxels"] * d["ntr"] for d in dicts]
    rng = np.random.default_rng(6)
    out = {"workload": "12 distinct requests reused: voxels logU[4k,200k], coils U{4..16}, TRs U{400..1120}, "
                       "FISP (25 states, 35 positions) / pSSFP (35 z), Cartesian (S=sqrt V) / spiral (TRs x 1000); "
                       "request = simulate + FD derivative simulations + signal + residual + J^H r",
           "memory_budget_gb": 150, "max_inflight_batches": 4, "max_batch_requests": 16, "runs": []}

    warmed = set()

    def stream_run(rate, method, nreq, echo_keys, delta=1e-4):
        eng = cb.ServeEngine(ctx, memory_budget_gb=150.0, max_inflight_batches=4, max_batch_requests=16,
                             method=method, delta=delta)
        if (method, delta) not in warmed:  # first use of each kernel family and of every sequence table
            for t in [eng.submit(*o) for o in objs]:
                eng.wait(t)
                eng.release(t)
            eng.reset_stats()
            warmed.add((method, delta))
        picks = rng.integers(0, len(objs), nreq)
        gaps = rng.exponential(1.0 / rate, nreq)
        tickets = [None] * nreq
        t0 = time.perf_counter()

        def client():
            due = t0
            for k in range(nreq):
                due += gaps[k]
                delay = due - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                i = int(picks[k])
                tickets[k] = eng.submit(*objs[i], echo_key=(i + 1) if echo_keys else 0)

        th = threading.Thread(target=client)
        th.start()
        th.join()
        for t in tickets:
            eng.wait(t)
        wall = time.perf_counter() - t0
        for t in tickets:
            eng.release(t)
        st = eng.stats()
        done_vtr = float(sum(vtr[int(i)] for i in picks))
        return {"rate_per_s": rate, "method": method, "requests": nreq, "echo_reuse": echo_keys,
                "derivatives": "exact tangents" if delta == 0 else f"forward differences, step {delta}",
                "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "max_ms": st["max_ms"],
                "voxel_tr_per_s": done_vtr / wall, "requests_per_s": nreq / wall, "batches": st["batches"],
                "max_concurrent_batches": st["max_concurrent_batches"], "peak_gb": st["peak_bytes"] / 2 ** 30,
                "echo_cache_hits": st["echo_cache_hits"], "failed": st["failed"]}

    rates = [float(r) for r in args.serve_rates.split(",") if r]
    for r in rates:
        out["runs"].append(stream_run(r, "MatmulFast", args.serve_requests, False))
    out["runs"].append(stream_run(rates[len(rates) // 2], "Direct", args.serve_requests, False))
    out["runs"].append(stream_run(rates[-1], "MatmulFast", args.serve_requests, True))
    out["runs"].append(stream_run(rates[len(rates) // 2], "MatmulFast", args.serve_requests, False, delta=0.0))
    return out


def elementwise(cb, ctx, stream, w, params, seq, traj, peaks):
    """The HBM-bound operations of the path, against the measured HBM copy bandwidth:
    phase_encoding of the MR-STAT echoes [1120][50176] (read + write 8 B per element, through the
    public API) and the residual diff = lhs - rhs, Σ|diff|² over 2^24 complex values (read 16 B,
    write 8 B per element; the allocation-free entry point on caller-owned buffers, since the
    public one returns the objective to the host). Calls are enqueued behind a 20 ms spin kernel,
    so the timed span holds the kernels only, not the host's per-call overhead."""
    import torch

    echos = cb.simulate_magnetization(ctx, params, seq)
    ctx.synchronize()
    R, V = echos.shape
    reps = 5

    def gpu_ms(fn):
        # warm-up with as many results alive as the timed loop keeps, so that the memory pool has
        # grown to its size before timing (growing it maps memory on the host, which would show up
        # inside the timed span)
        warm = [fn() for _ in range(reps)]
        ctx.synchronize()
        del warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            torch.cuda._sleep(40_000_000)
            e0.record(stream)
            keep = [fn() for _ in range(reps)]
            e1.record(stream)
        ctx.synchronize()
        del keep
        return e0.elapsed_time(e1) / reps

    n_pe = R * V
    pe_ms = gpu_ms(lambda: cb.phase_encoding(ctx, echos, params, traj))
    n = 1 << 24
    g = torch.Generator(device="cuda").manual_seed(9)
    a = torch.randn(2 * n, device="cuda", generator=g)
    b = torch.randn(2 * n, device="cuda", generator=g)
    diff = torch.empty_like(a)
    obj = torch.empty(1, device="cuda")
    fn = cb.library().compas_b200_compute_residual_noalloc
    res_ms = gpu_ms(lambda: fn(ctx.device, a.data_ptr(), b.data_ptr(), diff.data_ptr(), obj.data_ptr(), n,
                               ctx.stream or None))
    hbm = peaks["hbm_gbs"]
    pe_gbs = 16.0 * n_pe / (pe_ms / 1e3) / 1e9
    res_gbs = 24.0 * n / (res_ms / 1e3) / 1e9
    return {"phase_encoding": {"elements": n_pe, "ms": pe_ms, "algorithmic_bytes": 16.0 * n_pe, "gbs": pe_gbs,
                               "frac_of_hbm": pe_gbs / hbm},
            "residual": {"elements": n, "ms": res_ms, "algorithmic_bytes": 24.0 * n, "gbs": res_gbs,
                         "frac_of_hbm": res_gbs / hbm}}


def ref_gpu_timed(oracle, timed, fn, stream):
    """One re-hosted reference call, timed: the index-checked build runs first and gives the result;
    where its out-of-bounds flag stays clear, the build without index checks (which kmm's own views
    do not make either) is timed on the same launches, else the checked build. Returns
    (ms, result, which build was timed)."""
    import torch

    with torch.cuda.stream(stream):
        out = fn(unchecked=False)
    torch.cuda.synchronize()
    if oracle.ref_gpu_out_of_bounds() == 0 and oracle.ref_gpu(unchecked=True) is not None:
        ms, _ = timed(lambda: fn(unchecked=True), stream)
        return ms, out, "unchecked views"
    ms, _ = timed(lambda: fn(unchecked=False), stream)
    return ms, out, "index-checked views"


def reference_kernels_gpu(cb, ctx, stream, w, sim_ms, args):
    """The reference's own FISP and pSSFP kernels on the same B200 ("reference kernels, re-hosted":
    oracle/_ref/libref_gpu.so, its unmodified src/simulate/*_kernels.cuh with its CUDA flags and
    launch shapes), timed with CUDA events on the same workloads as this library: the MR-STAT FISP
    slice of the main measurement, a pSSFP slice (35 z, 15 RF samples, 320 TRs) and a 16-coil spiral
    signal (its only spiral method). rel_l2 compares the two implementations' results over the
    whole array."""
    import torch
    import workloads

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    if oracle.ref_gpu() is None:
        return {"unavailable": "oracle/_ref/libref_gpu.so not built (the reference tree was absent at build time)"}

    def timed(fn, s, reps=2):
        with torch.cuda.stream(s):
            # the loop below holds two results at once (the last one and the new one): warm up with
            # two alive, so that the memory pools have grown to that before the timed span (growing
            # a pool maps memory, which would land inside it)
            warm = [fn() for _ in range(2)]
            torch.cuda.synchronize()
            del warm
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(reps):
                r = fn()
            e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, r

    def rel(a, b):
        a, b = torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda")
        a, b = torch.view_as_real(a) if a.is_complex() else a, torch.view_as_real(b) if b.is_complex() else b
        return float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double()))

    ts = torch.cuda.Stream()
    res = {"what": "the reference's simulate_fisp / simulate_pssfp kernels (fisp_kernels.cuh, pssfp_kernels.cuh), "
                   "unmodified, compiled with nvcc --use_fast_math for sm_100 against stand-ins for the absent "
                   "kmm views; launch code restated from src/simulate/fisp.cu and pssfp.cu"}
    V = w["params"].shape[1]
    nTR = len(w["seq"]["rf"])
    ref_ms, ref_e, build = ref_gpu_timed(oracle, timed, lambda **kw: oracle.ref_gpu_fisp(w["params"], w["seq"], **kw),
                                         ts)
    res["timed_build"] = build
    p = cb.TissueParameters.from_soa(ctx, w["params"])
    mine = cb.simulate_magnetization(ctx, p, cb.FispSequence.from_dict(ctx, w["seq"]))
    ctx.synchronize()
    res["fisp_mrstat"] = {"voxels": V, "readouts": nTR, "reference_ms": ref_ms, "this_ms": sim_ms,
                          "reference_voxel_tr_per_s": V * nTR / (ref_ms / 1e3),
                          "this_voxel_tr_per_s": V * nTR / (sim_ms / 1e3), "speedup": ref_ms / sim_ms,
                          "rel_l2": rel(torch.view_as_real(ref_e), mine)}
    del ref_e, mine
    rng = np.random.default_rng(7)
    pd = workloads.pssfp_sequence(rng, 320, nrf=15, nz=35)
    pp = workloads.tissue(rng, args.n_side, 22.4)
    ref_ms, ref_e, _ = ref_gpu_timed(oracle, timed, lambda **kw: oracle.ref_gpu_pssfp(pp, pd, **kw), ts)
    p = cb.TissueParameters.from_soa(ctx, pp)
    seq = cb.pSSFPSequence.from_dict(ctx, pd)
    this_ms, mine = timed(lambda: cb.simulate_magnetization(ctx, p, seq), stream)
    res["pssfp_320tr"] = {"voxels": pp.shape[1], "readouts": 320, "reference_ms": ref_ms, "this_ms": this_ms,
                          "reference_voxel_tr_per_s": pp.shape[1] * 320 / (ref_ms / 1e3),
                          "this_voxel_tr_per_s": pp.shape[1] * 320 / (this_ms / 1e3), "speedup": ref_ms / this_ms,
                          "rel_l2": rel(torch.view_as_real(ref_e), mine)}
    del ref_e, mine
    # spiral signal: 30000 voxels, 760 interleaves x 1000 samples, 16 coils (the reference's only
    # spiral method; here split-BF16 tensor cores)
    rng = np.random.default_rng(8)
    sp = workloads.tissue_voxels(rng, 30000, 22.4)
    st = workloads.spiral(rng, 760, 1000, 22.4, 4e-6)
    coils = workloads.cn(rng, (16, 30000))
    echo = workloads.cn(rng, (760, 30000)) * 0.1
    ref_ms, ref_s, _ = ref_gpu_timed(oracle, timed, lambda **kw: oracle.ref_gpu_signal_spiral(sp, echo, st, coils, **kw),
                                     ts)
    p = cb.TissueParameters.from_soa(ctx, sp)
    traj = cb.trajectory_from_dict(ctx, st)
    e_arr, c_arr = cb.CompasArray.from_numpy(ctx, echo), cb.CompasArray.from_numpy(ctx, coils)
    this_ms, mine = timed(lambda: cb.magnetization_to_signal(ctx, e_arr, p, traj, c_arr, method="MatmulFast"), stream)
    flops = 8.0 * 16 * 760 * 1000 * 30000
    res["spiral_signal_16coils"] = {"voxels": 30000, "readouts": 760, "samples": 1000, "reference_ms": ref_ms,
                                    "this_ms": this_ms, "reference_tflops": flops / ref_ms / 1e9,
                                    "this_tflops": flops / this_ms / 1e9, "speedup": ref_ms / this_ms,
                                    "rel_l2": rel(torch.view_as_real(ref_s), mine)}
    res["out_of_bounds_flag"] = oracle.ref_gpu_out_of_bounds()
    return res


def reference_products_gpu(w, stream, reps, this_ms, lib):
    """The reference's default product paths on the same B200 and inputs: MatmulFast signal and
    GemmFast J·v / Jᴴ·v (its kernels plus TF32 cuBLAS, re-hosted: oracle/_ref/libref_gpu.so). rel_l2
    compares their results with this library's split-BF16 ones."""
    import torch

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    if oracle.ref_gpu() is None:
        return {"unavailable": "oracle/_ref/libref_gpu.so not built (the reference tree was absent at build time)"}
    cb, ctx, params, traj, arr, d = lib
    ins = {k: torch.as_tensor(np.ascontiguousarray(w[k]), device="cuda")
           for k in ("echo", "dT1", "dT2", "v", "r", "coils")}
    ts = torch.cuda.Stream()
    runs = {"signal": lambda **kw: oracle.ref_gpu_signal_cartesian(w["params"], ins["echo"], w["traj"], ins["coils"],
                                                                   **kw),
            "jv": lambda **kw: oracle.ref_gpu_jacobian(w["params"], ins["echo"], ins["dT1"], ins["dT2"], w["traj"],
                                                       ins["coils"], ins["v"], **kw),
            "jhv": lambda **kw: oracle.ref_gpu_jacobian(w["params"], ins["echo"], ins["dT1"], ins["dT2"], w["traj"],
                                                        ins["coils"], ins["r"], hermitian=True, **kw)}
    mine = {"signal": lambda: cb.magnetization_to_signal(ctx, arr["echo"], params, traj, arr["coils"],
                                                         method="MatmulFast"),
            "jv": lambda: cb.compute_jacobian(ctx, arr["echo"], d, params, traj, arr["coils"], arr["v"],
                                              method="GemmFast"),
            "jhv": lambda: cb.compute_jacobian_hermitian(ctx, arr["echo"], d, params, traj, arr["coils"], arr["r"],
                                                         method="GemmFast")}
    res = {"what": "the reference's MatmulFast signal and GemmFast J·v / Jᴴ·v (the C ABI's defaults): its unmodified "
                   "kernels and its four-GEMM complex products on TF32 cuBLAS, launch code restated from "
                   "src/trajectories/signal.cu, src/jacobian/product.cu, hermitian.cu"}
    def timed(fn, s):
        with torch.cuda.stream(s):
            warm = [fn() for _ in range(2)]  # two results alive, as in the timed loop (pool growth)
            torch.cuda.synchronize()
            del warm
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(reps):
                r = fn()
            e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, r

    for name, fn in runs.items():
        ms, out, build = ref_gpu_timed(oracle, timed, fn, ts)
        res["timed_build"] = build
        ours = torch.as_tensor(mine[name](), device="cuda")
        ctx.synchronize()
        a = torch.view_as_real(out).double()
        rel = float(torch.linalg.vector_norm(a - ours.double()) / torch.linalg.vector_norm(ours.double()))
        res[name] = {"reference_ms": ms, "this_ms": this_ms[name], "speedup": ms / this_ms[name], "rel_l2": rel}
        del out, ours
    res["out_of_bounds_flag"] = oracle.ref_gpu_out_of_bounds()
    return res


def derivatives(cb, ctx, stream, args, rank):
    """∂m/∂T1 and ∂m/∂T2 two ways: the reference's forward differences (value simulation plus one
    simulation per field at p + Δ, Δ = 1e-4) and the forward-mode tangents (value and both
    derivatives in one pass), on the MR-STAT FISP slice and a 224² pSSFP case (35 z, 15 RF
    samples, 320 TRs). fd_rel_error = ‖FD − tangent‖/‖tangent‖ over the whole array: the
    difference's truncation and FP32 cancellation error (the tangents match the FP64 central
    difference to 1e-5 in the parity tests)."""
    import numpy as np
    import torch
    import workloads

    if args.tangent_layout >= 0:
        cb.set_fisp_tangent_launch(args.tangent_layout)

    def timed(fn, reps=2):
        warm = [fn() for _ in range(2)]  # two results alive, as in the timed loop (pool growth)
        ctx.synchronize()
        del warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            r = fn()
        e1.record(stream)
        ctx.synchronize()
        return e0.elapsed_time(e1) / reps, r

    rng = np.random.default_rng(3 + rank)
    w = workloads.mrstat(seed=2 + rank, n_side=args.n_side)
    pd = workloads.pssfp_sequence(rng, 320, nrf=15, nz=35)
    cases = (("fisp_mrstat", w["params"], cb.FispSequence.from_dict(ctx, w["seq"])),
             ("pssfp_320tr", workloads.tissue(rng, args.n_side, 22.4), cb.pSSFPSequence.from_dict(ctx, pd)))
    res = {}
    for name, params, seq in cases:
        p = cb.TissueParameters.from_soa(ctx, params)

        def fd():
            e = cb.simulate_magnetization(ctx, p, seq)
            return e, cb.simulate_magnetization_derivatives(ctx, e, p, seq)

        fd_ms, (_, d_fd) = timed(fd)
        tan_ms, d_tan = timed(lambda: cb.simulate_magnetization_tangents(ctx, p, seq))
        err = {}
        for f in ("T1", "T2"):
            a = torch.as_tensor(d_fd[f], device="cuda")
            b = torch.as_tensor(d_tan[f], device="cuda")
            err[f] = float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double()))
        res[name] = {"voxels": int(params.shape[1]), "readouts": int(seq.nreadouts),
                     "forward_difference_ms": fd_ms, "tangent_ms": tan_ms, "fd_rel_error": err}
    if args.tangent_layout >= 0:
        cb.set_fisp_tangent_launch(-1)
    return res


def gauss_newton(cb, ctx, stream, args, rank):
    """One Gauss-Newton iteration (3 FISP simulations or one tangent pass, signal, residual, 4
    CGLS steps of J·d and Jᴴ·b, update) per step, replayed as a CUDA graph vs issued kernel by
    kernel, on the MR-STAT slice (fit of data simulated from the true parameters, start perturbed)
    with forward-difference and with exact derivatives, and on the 64x64 case."""
    import numpy as np
    import torch
    import workloads

    res = {}
    for name, w, delta in (("mrstat", workloads.mrstat(seed=2 + rank, n_side=args.n_side), 1e-4),
                           ("mrstat_exact_derivatives", workloads.mrstat(seed=2 + rank, n_side=args.n_side), 0.0),
                           ("fisp_small", workloads.fisp_small(seed=1 + rank), 1e-4)):
        rng = np.random.default_rng(5)
        truth = w["params"]
        start = truth.copy()
        start[0] *= rng.uniform(0.9, 1.1, truth.shape[1])
        start[1] *= rng.uniform(0.9, 1.1, truth.shape[1])
        seq = cb.FispSequence.from_dict(ctx, w["seq"])
        traj = cb.CartesianTrajectory.from_dict(ctx, w["traj"])
        p_true = cb.TissueParameters.from_soa(ctx, truth)
        y = cb.magnetization_to_signal(ctx, cb.simulate_magnetization(ctx, p_true, seq), p_true, traj, w["coils"])
        gn = cb.GaussNewtonStep(ctx, cb.TissueParameters.from_soa(ctx, start), seq, traj, w["coils"], y,
                                delta=delta)
        times = {}
        for mode in (False, True):
            gn.run(graph=mode)  # warm-up (captures the graph)
            ctx.synchronize()
            reps = 3
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                gn.run(graph=mode)
            e1.record(stream)
            ctx.synchronize()
            times["graph" if mode else "eager"] = e0.elapsed_time(e1) / reps
        objs = []
        for _ in range(2):
            gn.run(graph=True)
            objs.append(gn.objective())
        V = truth.shape[1]
        res[name] = {"voxels": V, "coils": int(w["coils"].shape[0]), "cg_iterations": 4,
                     "derivatives": "exact tangents" if delta == 0 else f"forward differences, step {delta}",
                     "ms_per_iteration_graph": times["graph"], "ms_per_iteration_eager": times["eager"],
                     "kernels_per_iteration": gn.graph_kernels(), "objective_last_two": objs}
    return res


def jacobian_products(cb, ctx, stream, args, peaks, rank):
    """J·v and Jᴴ·v on the Jacobian workload (224x224 voxels, 1120x224 Cartesian, 8 coils),
    split-BF16 tensor cores, plus signal + Jᴴ·v on the plain FP32 path for comparison."""
    import torch
    import workloads

    w = workloads.jacobian_inputs(seed=3 + rank, n_side=args.n_side)
    V = w["params"].shape[1]
    C_, R, S = w["coils"].shape[0], w["traj"]["nr"], w["traj"]["ns"]
    params = cb.TissueParameters.from_soa(ctx, w["params"])
    traj = cb.CartesianTrajectory.from_dict(ctx, w["traj"])
    arr = {k: cb.CompasArray.from_numpy(ctx, w[k]) for k in ("echo", "dT1", "dT2", "v", "r", "coils")}
    d = {"T1": arr["dT1"], "T2": arr["dT2"]}

    def timed(fn, reps):
        fn()
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    reps = max(2, min(args.steps, 5))
    jv = timed(lambda: cb.compute_jacobian(ctx, arr["echo"], d, params, traj, arr["coils"], arr["v"],
                                           method="GemmFast"), reps)
    jhv = timed(lambda: cb.compute_jacobian_hermitian(ctx, arr["echo"], d, params, traj, arr["coils"], arr["r"],
                                                      method="GemmFast"), reps)
    sig = timed(lambda: cb.magnetization_to_signal(ctx, arr["echo"], params, traj, arr["coils"],
                                                   method="MatmulFast"), reps)
    sig_plain = timed(lambda: cb.magnetization_to_signal(ctx, arr["echo"], params, traj, arr["coils"],
                                                         method="Direct"), 1)
    jhv_plain = timed(lambda: cb.compute_jacobian_hermitian(ctx, arr["echo"], d, params, traj, arr["coils"],
                                                            arr["r"], method="Direct"), 1)
    err = products_error_fp64(cb, ctx, w, params, traj, arr, d)
    f_sig = 8.0 * C_ * R * S * V
    f_j = 16.0 * C_ * R * S * V
    f_jh = 16.0 * C_ * R * S * V + 24.0 * C_ * R * V
    peak = peaks["bf16_tflops_sustained"]
    tf = lambda f, ms: f / (ms / 1e3) / 1e12
    reference = reference_products_gpu(w, stream, reps, {"signal": sig, "jv": jv, "jhv": jhv},
                                       (cb, ctx, params, traj, arr, d))
    return {"workload": f"{args.n_side}x{args.n_side}={V} voxels, Cartesian {R}x{S}, {C_} coils, random echoes / "
                        "∂echoes, v and residual CN(0,1)",
            "reference_default_paths_gpu": reference,
            "jv_ms": jv, "jv_tflops": tf(f_j, jv), "jhv_ms": jhv, "jhv_tflops": tf(f_jh, jhv),
            "signal_ms": sig, "signal_tflops": tf(f_sig, sig),
            "signal_plus_jhv_tflops": tf(f_sig + f_jh, sig + jhv),
            "signal_plus_jhv_frac_of_bf16": tf(f_sig + f_jh, sig + jhv) / peak,
            "plain_fp32_signal_ms": sig_plain, "plain_fp32_jhv_ms": jhv_plain,
            "tensor_vs_plain_signal_plus_jhv": (sig_plain + jhv_plain) / (sig + jhv),
            "rel_err_fp64": err,
            "note": "algorithmic flops 8·C·R·S·V (signal), 16·C·R·S·V (J·v), 16·C·R·S·V + 24·C·R·V (Jᴴ·v); "
                    "split-BF16 issues 3 MMAs per product; fraction of the sustained BF16 peak (measured)"}


def products_error_fp64(cb, ctx, w, params, traj, arr, d, nent=256, nvox=128):
    """Relative L2 error against the FP64 oracle of the signal, J·v and Jᴴ·v on the Jacobian
    workload, split-BF16 (MatmulFast / GemmFast) and plain FP32 (Direct): 256 random
    (coil, readout, sample) entries, each summed over all voxels, and Jᴴ·v on 128 random voxels
    (outside any timed region)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    V = w["params"].shape[1]
    C_, R, S = w["coils"].shape[0], w["traj"]["nr"], w["traj"]["ns"]
    rng = np.random.default_rng(17)
    ent = np.stack([rng.integers(0, C_, nent), rng.integers(0, R, nent), rng.integers(0, S, nent)], 1)
    idx = np.sort(rng.choice(V, nvox, replace=False))
    at = lambda a: a[ent[:, 0], ent[:, 1], ent[:, 2]]  # noqa: E731
    ref = {"signal": oracle.signal_cartesian(w["echo"], w["params"], w["traj"], w["coils"], entries=ent),
           "jv": oracle.jacobian(w["echo"], w["dT1"], w["dT2"], w["params"], w["traj"], w["coils"], w["v"],
                                 entries=ent),
           "jhv": oracle.jacobian_hermitian(w["echo"], w["dT1"], w["dT2"], w["params"], w["traj"], w["coils"],
                                            w["r"], vidx=idx)}
    out = {"sample": f"{nent} entries summed over all {V} voxels (signal, J·v), {nvox} voxels (Jᴴ·v)"}
    for tc, plain in (("MatmulFast", "Direct"),):
        for m in (tc, plain):
            s = cb.magnetization_to_signal(ctx, arr["echo"], params, traj, arr["coils"], method=m).to_numpy()
            out[f"signal_{m}"] = oracle.rel_l2(at(s), ref["signal"])
    for m in ("GemmFast", "Direct"):
        jv = cb.compute_jacobian(ctx, arr["echo"], d, params, traj, arr["coils"], arr["v"], method=m).to_numpy()
        out[f"jv_{m}"] = oracle.rel_l2(at(jv), ref["jv"])
        jh = cb.compute_jacobian_hermitian(ctx, arr["echo"], d, params, traj, arr["coils"], arr["r"],
                                           method=m).to_numpy()
        out[f"jhv_{m}"] = oracle.rel_l2(jh[:, idx], ref["jhv"])
    return out


def e2e(cb, ctx, w, args, local, voxels, signal_of, world):
    """Same step through the public API from pinned host buffers: every step uploads the
    tissue parameters, sequence, trajectory and coils (this rank's voxels) and reads the signal
    back; over several ranks the signal call is the sharded one (NCCL sum of the partials) and the
    time is the slowest rank's."""
    import torch

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t.numpy()

    vb, ve = voxels
    p_h = pinned(w["params"][:, vb:ve])
    rf_h, sl_h = pinned(w["seq"]["rf"]), pinned(w["seq"]["slices"])
    ks_h, co_h = pinned(w["traj"]["k_start"]), pinned(w["coils"][:, vb:ve])
    C_, R, S = co_h.shape[0], w["traj"]["nr"], w["traj"]["ns"]
    out_h = pinned(np.zeros((C_, R, S), np.complex64))
    s = w["seq"]
    t = w["traj"]

    def step():
        params = cb.TissueParameters.from_soa(ctx, p_h)
        seq = cb.FispSequence(ctx, rf_h, sl_h, s["TR"], s["TE"], s["max_state"], s["TI"], s["uf"], s["reps"])
        traj = cb.CartesianTrajectory(ctx, t["nr"], t["ns"], t["dt"], ks_h, t["dk"])
        coils = cb.CompasArray.from_numpy(ctx, co_h)
        e = cb.simulate_magnetization(ctx, params, seq)
        sig = signal_of(e, params, coils)
        sig.read_into(out_h)

    for _ in range(max(1, args.warmup)):
        step()
    steps = max(1, min(args.steps, 3))
    ctx.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    ctx.synchronize()
    dt = (time.perf_counter() - t0) / steps
    if world > 1:
        t = torch.tensor([dt], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        dt = float(t.item())
    V, nTR = w["params"].shape[1], len(rf_h)
    h2d = p_h.nbytes + rf_h.nbytes + sl_h.nbytes + ks_h.nbytes + co_h.nbytes
    return {"value": V * nTR / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(out_h.nbytes), "ms_per_step": dt * 1e3,
            "note": "host wall clock around the public C-ABI calls (each read blocks on the device)"}


if __name__ == "__main__":
    sys.exit(main())
