"""Gauss-Newton iteration on the device (compas_b200_make_gauss_newton / _run).

One iteration simulates m(p), the derivatives dm/dT1 and dm/dT2 (forward differences, or exact
tangents for delta = 0), the signal s(p), the residual b = y - s, runs CGLS steps of J·d / Jᴴ·b
on min ‖J δ - b‖² and updates the parameters after a line search on the objective (the first of
t = 1, ½ that does not raise ‖y - s‖², else no step). The tests check that (1) the CUDA-graph
replay gives the same bits as the eager kernel sequence over two iterations, (2) with one CGLS
step the step equals α·Re(Jᴴ b) with α = ‖g‖²/‖J g‖², recomputed here from the public
operations, within the FP32 tolerance of the other tests, (3) fitting data simulated from known
parameters lowers the objective, (4) the same with exact derivatives, which equal
simulate_magnetization_tangents, and (5) with the line search the objective never rises and the
update is the step length it reports.
"""
import numpy as np
import pytest

import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5


def _problem(seed=21, n_side=12, ntr=60, ns=12, nc=2):
    rng = np.random.default_rng(seed)
    fov = 22.4
    truth = W.tissue(rng, n_side, fov)
    rf = W.smooth_flip_train(rng, ntr)
    seq = W.fisp_sequence(rf, W.gaussian_slice_profile(3, ntr), 8.7e-3, 4.35e-3, 25e-3, 8)
    traj = W.cartesian(ntr, ns, fov, 5e-6, ns)
    coils = W.gaussian_coils(nc, truth, fov)
    start = truth.copy()
    start[0] *= rng.uniform(0.85, 1.15, start.shape[1])
    start[1] *= rng.uniform(0.85, 1.15, start.shape[1])
    start[4] += 0.05 * rng.standard_normal(start.shape[1])
    start[5] += 0.05 * rng.standard_normal(start.shape[1])
    return truth, start.astype(np.float32), seq, traj, coils


@pytest.fixture(scope="module")
def setup():
    import compas_b200 as cb

    ctx = cb.Context(0)
    truth, start, seq_d, traj_d, coils = _problem()
    seq = cb.FispSequence.from_dict(ctx, seq_d)
    traj = cb.CartesianTrajectory.from_dict(ctx, traj_d)
    p_true = cb.TissueParameters.from_soa(ctx, truth)
    y = cb.magnetization_to_signal(ctx, cb.simulate_magnetization(ctx, p_true, seq), p_true, traj, coils,
                                   method="MatmulFast").to_numpy()
    return cb, ctx, start, seq, traj, coils, y


def _gn(cb, ctx, start, seq, traj, coils, y, **kw):
    return cb.GaussNewtonStep(ctx, cb.TissueParameters.from_soa(ctx, start), seq, traj, coils, y, **kw)


def test_graph_replay_matches_eager_bitwise(setup):
    cb, ctx, start, seq, traj, coils, y = setup
    eager = _gn(cb, ctx, start, seq, traj, coils, y, cg_iterations=3)
    graph = _gn(cb, ctx, start, seq, traj, coils, y, cg_iterations=3)
    for it in range(2):
        eager.run(graph=False)
        graph.run(graph=True)
        ctx.synchronize()
        for name in ("parameters", "echos", "dT1", "dT2", "signal", "gradient", "step", "scalars"):
            a, b = eager.array(name).to_numpy(), graph.array(name).to_numpy()
            assert np.array_equal(a, b), (it, name)
    assert graph.graph_kernels() > 10
    assert eager.graph_kernels() == -1


def test_single_cg_step_is_the_exact_line_minimiser(setup):
    # without the line search the full CGLS step is applied
    cb, ctx, start, seq, traj, coils, y = setup
    gn = _gn(cb, ctx, start, seq, traj, coils, y, cg_iterations=1, line_search=False)
    params0 = cb.TissueParameters.from_soa(ctx, start)
    gn.run(graph=False)
    ctx.synchronize()
    echos = gn.array("echos")
    d = {"T1": gn.array("dT1"), "T2": gn.array("dT2")}
    s = cb.magnetization_to_signal(ctx, echos, params0, traj, coils, method="MatmulFast").to_numpy()
    assert np.array_equal(s, gn.array("signal").to_numpy())
    b = (y - s).astype(np.complex64)
    obj = float(gn.array("scalars").to_numpy()[0])
    ref = float(np.sum(np.abs(b.astype(np.complex128)) ** 2))
    assert abs(obj - ref) <= TOL_FP32 * ref
    g = cb.compute_jacobian_hermitian(ctx, echos, d, params0, traj, coils, b, method="GemmFast").to_numpy()
    gr = g.real.astype(np.float32)
    Jg = cb.compute_jacobian(ctx, echos, d, params0, traj, coils, gr.astype(np.complex64),
                             method="GemmFast").to_numpy()
    alpha = np.sum(gr.astype(np.float64) ** 2) / np.sum(np.abs(Jg.astype(np.complex128)) ** 2)
    step = gn.array("step").to_numpy()
    expect = alpha * gr
    assert np.linalg.norm(step - expect) <= 1e-4 * np.linalg.norm(expect)
    # the update applied to the parameters
    p1 = gn.array("parameters").to_numpy()
    c = np.clip(1.0 + step[:2].astype(np.float64), 0.5, 2.0)
    np.testing.assert_allclose(p1[0], start[0] * c[0], rtol=1e-6)
    np.testing.assert_allclose(p1[1], start[1] * c[1], rtol=1e-6)
    np.testing.assert_allclose(p1[4], start[4] + step[2], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(p1[5], start[5] + step[3], rtol=1e-6, atol=1e-7)


def test_iterations_lower_the_objective(setup):
    cb, ctx, start, seq, traj, coils, y = setup
    gn = _gn(cb, ctx, start, seq, traj, coils, y, cg_iterations=4)
    objs = []
    for _ in range(4):
        gn.run(graph=True)
        objs.append(gn.objective())
    assert objs[-1] < 0.5 * objs[0], objs
    assert all(np.isfinite(objs))


def test_spiral_iteration_graph_matches_eager_and_lowers_the_objective(setup):
    # the same iteration on a spiral trajectory (spiral J·v / Jᴴ·v, an addition to the reference)
    cb, ctx, start, seq, _, coils, _ = setup
    rng = np.random.default_rng(23)
    truth, _, _, _, _ = _problem()
    traj = cb.SpiralTrajectory.from_dict(ctx, W.spiral(rng, 60, 40, 22.4, 4e-6))
    p_true = cb.TissueParameters.from_soa(ctx, truth)
    y = cb.magnetization_to_signal(ctx, cb.simulate_magnetization(ctx, p_true, seq), p_true, traj, coils).to_numpy()
    eager = _gn(cb, ctx, start, seq, traj, coils, y, cg_iterations=3)
    graph = _gn(cb, ctx, start, seq, traj, coils, y, cg_iterations=3)
    objs = []
    for it in range(3):
        eager.run(graph=False)
        graph.run(graph=True)
        ctx.synchronize()
        for name in ("parameters", "gradient", "step", "scalars"):
            assert np.array_equal(eager.array(name).to_numpy(), graph.array(name).to_numpy()), (it, name)
        objs.append(graph.objective())
    assert objs[-1] < objs[0], objs



@pytest.mark.parametrize("kind", ["fisp", "pssfp"])
def test_exact_derivative_iteration(setup, kind):
    # delta = 0: the iteration takes m, ∂m/∂T1, ∂m/∂T2 from one tangent pass
    cb, ctx, start, seq, traj, coils, y = setup
    if kind == "pssfp":
        rng = np.random.default_rng(24)
        seq = cb.pSSFPSequence.from_dict(ctx, W.pssfp_sequence(rng, 60, nrf=5, nz=6))
        truth, _, _, _, _ = _problem()
        p_true = cb.TissueParameters.from_soa(ctx, truth)
        y = cb.magnetization_to_signal(ctx, cb.simulate_magnetization(ctx, p_true, seq), p_true, traj, coils,
                                       method="MatmulFast").to_numpy()
    eager = _gn(cb, ctx, start, seq, traj, coils, y, cg_iterations=3, delta=0.0)
    graph = _gn(cb, ctx, start, seq, traj, coils, y, cg_iterations=3, delta=0.0)
    tangents = cb.simulate_magnetization_tangents(ctx, cb.TissueParameters.from_soa(ctx, start), seq)
    objs = []
    for it in range(3):
        eager.run(graph=False)
        graph.run(graph=True)
        ctx.synchronize()
        if it == 0:
            for name, key in (("echos", "echos"), ("dT1", "T1"), ("dT2", "T2")):
                assert np.array_equal(graph.array(name).to_numpy(), tangents[key].to_numpy()), name
        for name in ("parameters", "echos", "dT1", "dT2", "signal", "gradient", "step", "scalars"):
            assert np.array_equal(eager.array(name).to_numpy(), graph.array(name).to_numpy()), (it, name)
        objs.append(graph.objective())
    assert objs[-1] < 0.5 * objs[0], objs


@pytest.mark.parametrize("graph", [True, False])
def test_line_search_never_raises_the_objective(graph):
    # the 64x64 FISP workload (400 TRs, 8 states, one coil), T1 and T2 started up to a factor 1.6
    # off: every iteration's objective is at most the previous one, and the estimate moves by the
    # step length the iteration reports (1, ½ or 0)
    import compas_b200 as cb

    ctx = cb.Context(0)
    w = W.fisp_small()
    rng = np.random.default_rng(31)
    truth = w["params"]
    start = truth.copy()
    start[0] *= rng.uniform(0.6, 1.6, truth.shape[1])
    start[1] *= rng.uniform(0.6, 1.6, truth.shape[1])
    start = start.astype(np.float32)
    seq = cb.FispSequence.from_dict(ctx, w["seq"])
    traj = cb.CartesianTrajectory.from_dict(ctx, w["traj"])
    p_true = cb.TissueParameters.from_soa(ctx, truth)
    y = cb.magnetization_to_signal(ctx, cb.simulate_magnetization(ctx, p_true, seq), p_true, traj, w["coils"]).to_numpy()
    gn = _gn(cb, ctx, start, seq, traj, w["coils"], y, cg_iterations=3)
    objs, lengths = [], []
    for _ in range(6):
        p0 = gn.array("parameters").to_numpy()
        gn.run(graph=graph)
        objs.append(gn.objective())
        t = gn.step_length()
        lengths.append(t)
        assert t in (0.0, 0.5, 1.0)
        step = gn.array("step").to_numpy().astype(np.float64)
        p1 = gn.array("parameters").to_numpy()
        c = np.clip(1.0 + t * step[:2], 0.5, 2.0)
        np.testing.assert_allclose(p1[0], p0[0] * c[0], rtol=1e-6)
        np.testing.assert_allclose(p1[1], p0[1] * c[1], rtol=1e-6)
        np.testing.assert_allclose(p1[4], p0[4] + t * step[2], rtol=1e-6, atol=1e-7)
        if t > 0:  # the taken trial's objective is the next iteration's starting objective
            assert float(gn.array("scalars").to_numpy()[6]) <= objs[-1]
    assert all(b <= a for a, b in zip(objs, objs[1:])), objs
    assert objs[-1] < objs[0], (objs, lengths)
