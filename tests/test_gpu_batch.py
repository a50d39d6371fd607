"""Batched execution of uneven simulate -> signal jobs (compas_b200_make_batch / _batch_run).

A batch runs every FISP job of one launch layout in one persistent work-queue kernel, every
pSSFP job likewise on a second stream, then the Cartesian signals of each family in one batched
tensor-core launch and the spiral signals in one batched launch per coil grouping. The tests
check that each job's echoes and signal are bit-identical to the one-job calls, on a mix of
FISP/pSSFP, Cartesian/spiral, coil counts 1..5, several launch layouts and ragged sizes, for the
split-BF16 and the FP32 signal methods, and that a second run reproduces the first.
"""
import numpy as np
import pytest

import workloads as W

pytestmark = pytest.mark.gpu


def _mixed_jobs():
    jobs = W.batch_jobs(seed=11, njobs=10, vmin=150, vmax=2500, ntr_min=17, ntr_max=70, cmax=5, ns_spiral=90,
                        P=5, nz=12, nrf=5)
    # a different FISP layout group (8 states, 1 position) and a simulate-only job
    small = W.fisp_small()
    sub = {"kind": "fisp", "params": np.ascontiguousarray(small["params"][:, :777]),
           "seq": {**small["seq"], "rf": small["seq"]["rf"][:40], "slices": small["seq"]["slices"][:, :40]},
           "traj": W.cartesian(40, 21, small["fov"], 1e-5, 21),
           "coils": np.ones((1, 777), np.complex64)}
    jobs.append(sub)
    only = dict(jobs[0])
    only["traj"] = None
    jobs.append(only)
    # a pSSFP job with few z positions (another pSSFP layout)
    ps = dict(jobs[1])
    ps = {**W.batch_jobs(seed=12, njobs=1, vmin=300, vmax=301, ntr_min=25, ntr_max=25, cmax=2, ns_spiral=50,
                         nz=3, nrf=4)[0]}
    ps["kind"] = "pssfp"
    ps["seq"] = W.pssfp_sequence(np.random.default_rng(5), 25, nrf=4, nz=3)
    jobs.append(ps)
    # a FISP and a pSSFP job with complex RF samples: they run the general forms of the packed
    # layouts, in work-queue groups of their own beside the real-RF jobs of the same layouts
    for kind, seed in (("fisp", 13), ("pssfp", 14)):
        d = next(j for j in jobs if j["kind"] == kind and j["traj"] is not None)
        rf = np.asarray(d["seq"]["rf"])
        phase = np.exp(1j * np.random.default_rng(seed).uniform(-0.5, 0.5, rf.shape[0]))
        jobs.append({**d, "seq": {**d["seq"], "rf": (rf * phase).astype(np.complex64)}})
    return jobs


@pytest.fixture(scope="module")
def ctx():
    import compas_b200 as cb

    return cb.Context(0)


@pytest.mark.parametrize("method", ["MatmulFast", "Direct"])
def test_batch_matches_one_job_calls_bitwise(ctx, method):
    import compas_b200 as cb

    dicts = _mixed_jobs()
    kinds = {(d["kind"], None if d["traj"] is None else d["traj"]["kind"]) for d in dicts}
    assert {("fisp", "cartesian"), ("fisp", "spiral"), ("pssfp", "cartesian"), ("pssfp", "spiral")} <= kinds
    jobs = [cb.job_from_dict(ctx, d) for d in dicts]
    batch = cb.SimulationBatch(ctx, jobs, method=method)
    for rerun in range(2):
        n0 = cb.launch_count()
        batch.run()
        ctx.synchronize()
        assert cb.launch_count() > n0
        for j, (params, seq, traj, coils) in enumerate(jobs):
            echos = cb.simulate_magnetization(ctx, params, seq)
            e_ref = echos.to_numpy()
            e_b = batch.echos(j).to_numpy()
            assert np.array_equal(e_b, e_ref), (rerun, j, "echos")
            if traj is None:
                continue
            s_ref = cb.magnetization_to_signal(ctx, echos, params, traj, coils, method=method).to_numpy()
            s_b = batch.signal(j).to_numpy()
            assert s_b.shape == s_ref.shape
            assert np.array_equal(s_b, s_ref), (rerun, j, dicts[j]["kind"], dicts[j]["traj"]["kind"],
                                                float(np.abs(s_b - s_ref).max()))


def test_batch_rejects_mismatched_trajectory(ctx):
    import compas_b200 as cb

    d = _mixed_jobs()[0]
    params, seq, traj, coils = cb.job_from_dict(ctx, d)
    wrong = cb.CartesianTrajectory.from_dict(ctx, W.cartesian(d["ntr"] + 1, 8, 22.4, 5e-6, 8))
    with pytest.raises(cb.CompasError, match="readouts"):
        cb.SimulationBatch(ctx, [(params, seq, wrong, coils)])


@pytest.mark.parametrize("layout", ["default", "packed4x8"])
def test_batch_tangent_jobs_match_one_job_calls_bitwise(ctx, layout):
    # jobs flagged for tangents run on the tangent work-queue kernels in groups of their own; their
    # echoes and derivatives are the bits of simulate_magnetization_tangents for each alone, the
    # other jobs keep the bits of simulate_magnetization. packed4x8: every tangent job on the
    # two-wide layout of 4 lanes x 8 states, the 25-state job in its slot-0 truncation form
    # ((25 - 1) % 8 == 0), the 8-state jobs in the bit-test form
    import compas_b200 as cb

    if layout == "packed4x8":
        configs = [tuple(c) for c in cb.fisp_tangent_configs()]
        cb.set_fisp_tangent_launch(next(i for i, c in enumerate(configs)
                                        if c == (8, 4) and cb.fisp_tangent_config_packed(i)))
    try:
        _check_tangent_batch(cb, ctx)
    finally:
        cb.set_fisp_tangent_launch(-1)


def _check_tangent_batch(cb, ctx):
    dicts = _mixed_jobs()
    # the MR-STAT sequence (25 states, 35 positions: 8 warps, 48 KB of dynamic shared memory in the
    # tangent queue kernel beside its static argument block) on a few voxels
    m = W.mrstat(n_side=20, ntr=64)
    dicts.append({"kind": "fisp", "params": m["params"], "seq": m["seq"], "traj": m["traj"], "coils": m["coils"]})
    jobs = [cb.job_from_dict(ctx, d) for d in dicts]
    flags = [j % 2 == 0 for j in range(len(jobs))]
    flags[-1] = True
    batch = cb.SimulationBatch(ctx, jobs, method="MatmulFast", tangents=flags)
    batch.run()
    ctx.synchronize()
    for j, (params, seq, traj, coils) in enumerate(jobs):
        if flags[j]:
            t = cb.simulate_magnetization_tangents(ctx, params, seq)
            echos = t["echos"]
            for f in ("T1", "T2"):
                assert np.array_equal(batch.derivative(j, f).to_numpy(), t[f].to_numpy()), (j, f)
        else:
            echos = cb.simulate_magnetization(ctx, params, seq)
            with pytest.raises(cb.CompasError):
                batch.derivative(j, "T1")
        assert np.array_equal(batch.echos(j).to_numpy(), echos.to_numpy()), (j, "echos")
        if traj is not None:
            s_ref = cb.magnetization_to_signal(ctx, echos, params, traj, coils, method="MatmulFast").to_numpy()
            assert np.array_equal(batch.signal(j).to_numpy(), s_ref), (j, "signal")


@pytest.mark.parametrize("P", [7, 35])
def test_balanced_fisp_split_matches_whole_tiles_bitwise(ctx, P):
    # With at least two voxel tiles per CTA, the one-simulation FISP kernel splits the (tile,
    # position) items evenly over its CTAs: neighbours share a tile and the later one adds its
    # positions to the earlier one's partial sums. The work-queue kernel of a batch runs whole tiles
    # per item. Both add every tile's positions one at a time in increasing order: the same bits.
    import compas_b200 as cb

    rng = np.random.default_rng(40 + P)
    nv, ntr = 13000, 48  # 407 tiles of 32 voxels on at most 148 CTAs
    d = {"kind": "fisp", "params": W.tissue_voxels(rng, nv, 22.4),
         "seq": W.fisp_sequence(W.smooth_flip_train(rng, ntr), W.gaussian_slice_profile(P, ntr), 8.7e-3, 4.35e-3,
                                25e-3, 25),
         "traj": None, "coils": np.ones((1, nv), np.complex64)}
    packed = next(i for i, (k, g) in enumerate(cb.fisp_configs()) if (k, g) == (26, 1) and cb.fisp_config_packed(i))
    cb.set_fisp_launch(packed, 8)
    try:
        params, seq, traj, coils = cb.job_from_dict(ctx, d)
        single = cb.simulate_magnetization(ctx, params, seq).to_numpy()
        batch = cb.SimulationBatch(ctx, [(params, seq, traj, coils)], method="MatmulFast")
        batch.run()
        ctx.synchronize()
        assert np.array_equal(single, batch.echos(0).to_numpy())
        again = cb.simulate_magnetization(ctx, params, seq).to_numpy()
        assert np.array_equal(single, again)
    finally:
        cb.set_fisp_launch(-1, -1)
