"""GPU parity of the forward-mode tangents (compas_b200_simulate_magnetization_tangents).

The reference computes ∂m/∂T1 and ∂m/∂T2 by forward differences with an absolute step
(src/simulate/derivative.cu:11-62); the tangent kernels compute the Δ → 0 limit of that quotient in
the same pass as the value. The oracle is the FP64 central difference of the oracle simulation
(relative step 1e-4, truncation error ~1e-8 relative). Tolerance: 1e-5 relative L2, the FP32 bound
of the simulations themselves.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5


@pytest.fixture(scope="module")
def cb():
    import compas_b200

    compas_b200.library()
    return compas_b200


@pytest.fixture(scope="module")
def ctx(cb):
    return cb.Context(0)


def _fisp(cb, ctx, w):
    return cb.TissueParameters.from_soa(ctx, w["params"]), cb.FispSequence.from_dict(ctx, w["seq"])


def _check_tangents(cb, oracle, got, p, seqd, sim, value_ref, vidx=None):
    for name, field in (("T1", 0), ("T2", 1)):
        ref = oracle.derivative_central(sim, p, seqd, field, vidx=vidx)
        g = got[name].to_numpy() if vidx is None else got[name].to_numpy()[:, vidx]
        assert oracle.rel_l2(g, ref) < TOL_FP32, name
    e = got["echos"].to_numpy() if vidx is None else got["echos"].to_numpy()[:, vidx]
    assert oracle.rel_l2(e, value_ref) < TOL_FP32


@pytest.mark.parametrize("max_state", [1, 2, 5, 8, 13, 25, 40])
def test_fisp_tangents_every_layout(cb, ctx, oracle, workloads, max_state):
    w = workloads.tiny(n_side=6, ntr=37, P=3, max_state=max_state, seed=max_state)
    params, seq = _fisp(cb, ctx, w)
    value = cb.simulate_magnetization(ctx, params, seq).to_numpy()
    ref_value = oracle.fisp(w["params"], w["seq"])
    ref = {f: oracle.derivative_central(oracle.fisp, w["params"], w["seq"], i) for i, f in enumerate(("T1", "T2"))}
    tried = 0
    try:
        for i, (k, g) in enumerate(cb.fisp_tangent_configs()):
            if k * g < max_state:
                continue
            cb.set_fisp_tangent_launch(i)
            got = cb.simulate_magnetization_tangents(ctx, params, seq)
            # same recurrence as the value kernel; the compiler may contract a different
            # multiply-add, so equal to FP32 rounding rather than bit for bit
            assert oracle.rel_l2(got["echos"].to_numpy(), value) < 1e-6, (k, g)
            for f in ("T1", "T2"):
                assert oracle.rel_l2(got[f].to_numpy(), ref[f]) < TOL_FP32, (k, g, f)
            tried += 1
    finally:
        cb.set_fisp_tangent_launch(-1)
    assert tried > 0
    assert oracle.rel_l2(value, ref_value) < TOL_FP32


@pytest.mark.parametrize("phase", [0.0, 0.3])
def test_fisp_packed_tangents_match_scalar_bits(cb, ctx, workloads, phase):
    # the two-wide tangent layouts run the scalar tangent update's operations on pairs of states
    # (with real phases, phase 0, in the form without the d_re products): m, ∂m/∂T1 and ∂m/∂T2 are
    # the bits of the scalar tangent layout of the same shape (up to the sign of exact zeros)
    rng = np.random.default_rng(23)
    ntr, P = 47, 3
    rf = workloads.smooth_flip_train(rng, ntr) * np.exp(1j * phase * rng.uniform(-1, 1, ntr))
    slices = workloads.gaussian_slice_profile(P, ntr)
    p = workloads.tissue(rng, 9, 22.4)
    params = cb.TissueParameters.from_soa(ctx, p)
    configs = [tuple(c) for c in cb.fisp_tangent_configs()]
    tried = 0
    try:
        for i, c in enumerate(configs):
            if not cb.fisp_tangent_config_packed(i):
                continue
            j = next(n for n, d in enumerate(configs) if d == c and not cb.fisp_tangent_config_packed(n))
            # N = K·(G-1) + 1 puts state N-1 in the first slot of the last lane: the packed layout
            # runs its slot-0 truncation form there, the scalar one its bit tests
            for N in sorted({c[0] * c[1], c[0] * c[1] - 3, c[0] * (c[1] - 1) + 1}):
                seq = cb.FispSequence.from_dict(ctx, workloads.fisp_sequence(rf, slices, 8.7e-3, 4.35e-3, 25e-3, N))
                cb.set_fisp_tangent_launch(i)
                packed = cb.simulate_magnetization_tangents(ctx, params, seq)
                packed = {k: packed[k].to_numpy() for k in ("echos", "T1", "T2")}
                cb.set_fisp_tangent_launch(j)
                scalar = cb.simulate_magnetization_tangents(ctx, params, seq)
                for k in ("echos", "T1", "T2"):
                    assert np.array_equal(packed[k], scalar[k].to_numpy()), (c, N, k, phase)
                tried += 1
    finally:
        cb.set_fisp_tangent_launch(-1)
    assert tried >= 10


def test_fisp_tangents_repetitions_undersampling(cb, ctx, oracle, workloads):
    # repetitions carry the state (and its tangents) through the wait TW; the C ABI's FISP
    # sequence always has the inversion prepulse and wait spoiling (bindings.cpp:151-174)
    w = workloads.tiny(n_side=5, ntr=23, P=4, max_state=9, seed=3)
    w["seq"]["reps"], w["seq"]["uf"], w["seq"]["TW"] = 3, 2, 0.05
    params, seq = _fisp(cb, ctx, w)
    got = cb.simulate_magnetization_tangents(ctx, params, seq)
    assert got["T1"].shape == (46, 25)
    _check_tangents(cb, oracle, got, w["params"], w["seq"], oracle.fisp, oracle.fisp(w["params"], w["seq"]))
    w["seq"]["reps"], w["seq"]["uf"], w["seq"]["TW"] = 2, 1, 0.0
    params, seq = _fisp(cb, ctx, w)
    got = cb.simulate_magnetization_tangents(ctx, params, seq)
    _check_tangents(cb, oracle, got, w["params"], w["seq"], oracle.fisp, oracle.fisp(w["params"], w["seq"]))


def test_fisp_tangents_mrstat_sampled(cb, ctx, oracle, workloads):
    # the 224² MR-STAT slice (25 states, 35 positions, 1120 TRs), checked on 64 voxels
    w = workloads.mrstat()
    params, seq = _fisp(cb, ctx, w)
    got = cb.simulate_magnetization_tangents(ctx, params, seq)
    value = cb.simulate_magnetization(ctx, params, seq).to_numpy()
    assert oracle.rel_l2(got["echos"].to_numpy(), value) < 1e-6
    idx = np.sort(np.random.default_rng(12).choice(50176, 64, replace=False))
    _check_tangents(cb, oracle, got, w["params"], w["seq"], oracle.fisp,
                    oracle.fisp(w["params"], w["seq"], vidx=idx), vidx=idx)


def test_fisp_tangents_are_the_limit_of_the_reference_difference(cb, ctx, workloads):
    # the reference's forward difference approaches the tangent as its step Δ shrinks. For T2
    # (10-500 ms) the O(Δ) truncation dominates and the error falls ~10× from Δ = 1e-3 to 1e-4;
    # for T1 (0.1-4 s) FP32 cancellation already sets the floor at Δ = 1e-4 (a few 1e-3), the
    # error the tangents avoid. At the reference's default Δ = 1e-4 both are within 1 %.
    w = workloads.tiny(n_side=5, ntr=31, P=2, max_state=6)
    params, seq = _fisp(cb, ctx, w)
    got = cb.simulate_magnetization_tangents(ctx, params, seq)
    echos = cb.simulate_magnetization(ctx, params, seq)
    for f, field in (("T1", 0), ("T2", 1)):
        t = got[f].to_numpy()
        err = {}
        for delta in (1e-3, 1e-4):
            fd = cb.simulate_magnetization_derivative(ctx, field, echos, params, seq, delta).to_numpy()
            err[delta] = np.linalg.norm(fd - t) / np.linalg.norm(t)
        assert err[1e-4] < 1e-2, (f, err)
        if f == "T2":
            assert err[1e-4] < err[1e-3] / 3, err


@pytest.mark.parametrize("nz", [1, 5, 35])
def test_pssfp_tangents_every_layout(cb, ctx, oracle, workloads, nz):
    rng = np.random.default_rng(nz + 50)
    seqd = workloads.pssfp_sequence(rng, 21, nrf=7, nz=nz)
    p = workloads.tissue(rng, 5, 20.0)
    params = cb.TissueParameters.from_soa(ctx, p)
    seq = cb.pSSFPSequence.from_dict(ctx, seqd)
    ref = {f: oracle.derivative_central(oracle.pssfp, p, seqd, i) for i, f in enumerate(("T1", "T2"))}
    tried = 0
    try:
        for i, (zt, gz) in enumerate(cb.pssfp_configs()):
            if zt * gz < nz:
                continue
            cb.set_pssfp_launch(i)
            got = cb.simulate_magnetization_tangents(ctx, params, seq)
            value = cb.simulate_magnetization(ctx, params, seq).to_numpy()
            assert oracle.rel_l2(got["echos"].to_numpy(), value) < 1e-6, (zt, gz)
            for f in ("T1", "T2"):
                assert oracle.rel_l2(got[f].to_numpy(), ref[f]) < TOL_FP32, (zt, gz, f)
            tried += 1
    finally:
        cb.set_pssfp_launch(-1)
    assert tried > 0


@pytest.mark.parametrize("scale,phase", [(1, 0.0), (3, 0.0), (1, 0.4)])
def test_pssfp_packed_tangents_match_scalar_bits(cb, ctx, workloads, scale, phase):
    # the two-wide tangent kernel runs the scalar tangent update's operations on pairs of isochromats:
    # m, ∂m/∂T1 and ∂m/∂T2 are the bits of the scalar layout with as many isochromats per lane (at 3x
    # the flip angles and 20x the off-resonance, some pairs take the sincos branch; phase 0: the
    # real-RF form)
    rng = np.random.default_rng(30 + scale)
    seqd = workloads.pssfp_sequence(rng, 15, nrf=5, nz=3)
    seqd["rf"] = (seqd["rf"] * scale * np.exp(1j * phase * rng.uniform(-1, 1, len(seqd["rf"])))).astype(np.complex64)
    p = workloads.tissue(rng, 5, 20.0)
    p[3] *= 1 if scale == 1 else 20
    params = cb.TissueParameters.from_soa(ctx, p)
    seq = cb.pSSFPSequence.from_dict(ctx, seqd)
    configs = cb.pssfp_configs()
    pairs = [(i, j) for i, c in enumerate(configs) if cb.pssfp_config_packed(i) and c[0] * c[1] >= 3
             for j, d in enumerate(configs) if not cb.pssfp_config_packed(j) and tuple(d) == tuple(c)]
    assert len(pairs) >= 3
    try:
        for i, j in pairs:
            cb.set_pssfp_launch(i)
            packed = cb.simulate_magnetization_tangents(ctx, params, seq)
            packed = {k: packed[k].to_numpy() for k in ("echos", "T1", "T2")}
            cb.set_pssfp_launch(j)
            scalar = cb.simulate_magnetization_tangents(ctx, params, seq)
            for k in ("echos", "T1", "T2"):
                assert np.array_equal(packed[k], scalar[k].to_numpy()), (configs[i], k)
    finally:
        cb.set_pssfp_launch(-1)


def test_pssfp_tangents_large_rotations(cb, ctx, oracle, workloads):
    # 3× the flip angles and 20× the off-resonance: the sincos branch of the rotation
    rng = np.random.default_rng(4)
    seqd = workloads.pssfp_sequence(rng, 17, nrf=3, nz=9)
    seqd["rf"] = (seqd["rf"] * 3).astype(np.complex64)
    p = workloads.tissue(rng, 4, 20.0)
    p[3] *= 20
    params = cb.TissueParameters.from_soa(ctx, p)
    got = cb.simulate_magnetization_tangents(ctx, params, cb.pSSFPSequence.from_dict(ctx, seqd))
    _check_tangents(cb, oracle, got, p, seqd, oracle.pssfp, oracle.pssfp(p, seqd))


def test_tangents_reject_bad_sequence(cb, ctx, workloads):
    w = workloads.tiny()
    params = cb.TissueParameters.from_soa(ctx, w["params"])
    with pytest.raises(cb.CompasError):
        cb.simulate_magnetization_tangents(ctx, params, params)
