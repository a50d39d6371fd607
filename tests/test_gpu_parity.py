"""GPU parity tests: every operation runs on cuda:0 through the C ABI
(libcompas_b200.so) and is compared with the CPU oracle on the same seeded inputs.

Tolerances (relative L2 against the FP64 oracle):
  * simulation (FISP EPG, pSSFP) and every plain-FP32 product:      1e-5
  * split-BF16 tensor-core products (MatmulFast/Low, GemmFast/Low): 1e-4
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5
TOL_BF16X3 = 1e-4
PLAIN_SIGNAL = ["Naive", "Direct", "MatmulPedantic", "Matmul"]
TC_SIGNAL = ["MatmulFast", "MatmulLow"]
PLAIN_JAC = ["Naive", "Direct", "Gemm"]
TC_JAC = ["GemmFast", "GemmLow"]


@pytest.fixture(scope="module")
def cb():
    import compas_b200

    compas_b200.library()
    return compas_b200


@pytest.fixture(scope="module")
def ctx(cb):
    return cb.Context(0)


def _upload(cb, ctx, w):
    params = cb.TissueParameters.from_soa(ctx, w["params"])
    seq = cb.FispSequence.from_dict(ctx, w["seq"]) if "seq" in w else None
    traj = cb.trajectory_from_dict(ctx, w["traj"])
    return params, seq, traj


# ------------------------------------------------------------------------------------------------
# FISP EPG
# ------------------------------------------------------------------------------------------------

@pytest.mark.parametrize("max_state", [1, 2, 5, 8, 13, 25])
def test_fisp_every_layout(cb, ctx, oracle, workloads, max_state):
    w = workloads.tiny(n_side=7, ntr=41, P=3, max_state=max_state)
    params, seq, _ = _upload(cb, ctx, w)
    ref = oracle.fisp(w["params"], w["seq"])
    tried = 0
    try:
        for i, (k, g) in enumerate(cb.fisp_configs()):
            if k * g < max_state:
                continue
            for warps in (1, 2, 3):
                cb.set_fisp_launch(i, warps)
                got = cb.simulate_magnetization(ctx, params, seq).to_numpy()
                assert oracle.rel_l2(got, ref) < TOL_FP32, (k, g, warps)
                tried += 1
    finally:
        cb.set_fisp_launch(-1, -1)
    assert tried > 0


def test_fisp_large_state_counts(cb, ctx, oracle, workloads):
    for n in (40, 64, 100, 128):
        w = workloads.tiny(n_side=5, ntr=150, P=2, max_state=n, seed=n)
        params, seq, _ = _upload(cb, ctx, w)
        got = cb.simulate_magnetization(ctx, params, seq).to_numpy()
        assert oracle.rel_l2(got, oracle.fisp(w["params"], w["seq"])) < TOL_FP32, n


def test_fisp_repetitions_undersampling(cb, ctx, oracle, workloads):
    w = workloads.tiny(n_side=6, ntr=29, P=5, max_state=7)
    w["seq"]["reps"], w["seq"]["uf"], w["seq"]["TW"] = 3, 4, 0.05
    params, seq, _ = _upload(cb, ctx, w)
    got = cb.simulate_magnetization(ctx, params, seq).to_numpy()
    assert got.shape == (29 * 4, 36)
    assert np.array_equal(got[0::4], got[3::4])
    assert oracle.rel_l2(got, oracle.fisp(w["params"], w["seq"])) < TOL_FP32


def test_fisp_small_config_full(cb, ctx, oracle, workloads):
    w = workloads.fisp_small()
    params, seq, _ = _upload(cb, ctx, w)
    got = cb.simulate_magnetization(ctx, params, seq).to_numpy()
    ref = oracle.fisp(w["params"], w["seq"])
    assert oracle.rel_l2(got, ref) < TOL_FP32
    # FP32 twin of the reference's arithmetic sits in the same band
    idx = np.arange(0, 4096, 41)
    twin = oracle.fisp(w["params"], w["seq"], vidx=idx, dtype="f32")
    assert oracle.rel_l2(got[:, idx], twin) < TOL_FP32


def test_fisp_mrstat_scale_sampled(cb, ctx, oracle, workloads):
    w = workloads.mrstat()
    params, seq, _ = _upload(cb, ctx, w)
    got = cb.simulate_magnetization(ctx, params, seq).to_numpy()
    assert got.shape == (1120, 50176) and np.isfinite(got).all()
    idx = np.sort(np.random.default_rng(11).choice(50176, 512, replace=False))
    ref = oracle.fisp(w["params"], w["seq"], vidx=idx)
    assert oracle.rel_l2(got[:, idx], ref) < TOL_FP32


def test_fisp_deterministic(cb, ctx, workloads):
    w = workloads.tiny(n_side=8, ntr=70, P=6, max_state=9)
    params, seq, _ = _upload(cb, ctx, w)
    a = cb.simulate_magnetization(ctx, params, seq).to_numpy()
    b = cb.simulate_magnetization(ctx, params, seq).to_numpy()
    assert np.array_equal(a, b)


@pytest.mark.parametrize("phase", [0.0, 0.3])
def test_fisp_packed_layouts_match_scalar_bits(cb, ctx, workloads, phase):
    # a packed layout runs the scalar update's operations on pairs of states. With real RF phases
    # (phase 0: a real flip train and real slice profiles) it runs the form without the products of
    # the coefficient d_re = sin φ·sin α·E1, which is then zero. Either way the echoes are the bits of
    # the scalar layout (up to the sign of exact zeros, which array_equal ignores).
    rng = np.random.default_rng(21)
    ntr, P = 57, 4
    rf = workloads.smooth_flip_train(rng, ntr) * np.exp(1j * phase * rng.uniform(-1, 1, ntr))
    slices = workloads.gaussian_slice_profile(P, ntr)
    p = workloads.tissue(rng, 9, 22.4)
    p[3] = rng.uniform(-30, 30, p.shape[1])  # off-resonance: complex relaxation factors
    params = cb.TissueParameters.from_soa(ctx, p)
    configs = [tuple(c) for c in cb.fisp_configs()]
    tried = 0
    try:
        for i, (k, g) in enumerate(configs):
            if not cb.fisp_config_packed(i):
                continue
            scalar_ks = {c[0] for n, c in enumerate(configs) if c[1] == 1 and not cb.fisp_config_packed(n)}
            twin = (k, 1) if k in scalar_ks else (k - 1, 1)  # 26 states packed, 25 scalar
            j = next(n for n, c in enumerate(configs) if c == twin and not cb.fisp_config_packed(n))
            for N in sorted({twin[0], twin[0] - 1}):
                seq = cb.FispSequence.from_dict(ctx, workloads.fisp_sequence(rf, slices, 8.7e-3, 4.35e-3, 25e-3, N))
                cb.set_fisp_launch(i, 4)
                packed = cb.simulate_magnetization(ctx, params, seq).to_numpy()
                cb.set_fisp_launch(j, 4)
                scalar = cb.simulate_magnetization(ctx, params, seq).to_numpy()
                assert np.array_equal(packed, scalar), (k, N, phase)
                tried += 1
    finally:
        cb.set_fisp_launch(-1, -1)
    assert tried >= 10


@pytest.mark.parametrize("inversion,wait_spoil", [(0, 1), (1, 0), (0, 0)])
def test_fisp_sequence_flags(cb, ctx, oracle, workloads, inversion, wait_spoil):
    # the C++ sequence's inversion prepulse and wait spoiling, off (compas_b200_make_fisp_sequence_ex),
    # with repetitions so that the wait and the next repetition's start matter
    w = workloads.tiny(n_side=6, ntr=31, P=3, max_state=9, seed=5)
    w["seq"].update(reps=3, TW=0.04, inversion=inversion, wait_spoil=wait_spoil)
    params, seq, _ = _upload(cb, ctx, w)
    got = cb.simulate_magnetization(ctx, params, seq).to_numpy()
    ref = oracle.fisp(w["params"], w["seq"])
    assert oracle.rel_l2(got, ref) < TOL_FP32
    both = oracle.fisp(w["params"], dict(w["seq"], inversion=1, wait_spoil=1))
    if not inversion:
        assert oracle.rel_l2(ref, both) > 1e-3  # the case differs from the C ABI's default sequence
    # (with the inversion, which spoils, the wait spoiling changes nothing: F states do not feed Z
    # without RF)
    tan = cb.simulate_magnetization_tangents(ctx, params, seq)
    assert oracle.rel_l2(tan["echos"].to_numpy(), got) < 1e-6
    for f, field in (("T1", 0), ("T2", 1)):
        d = oracle.derivative_central(oracle.fisp, w["params"], w["seq"], field)
        assert oracle.rel_l2(tan[f].to_numpy(), d) < TOL_FP32, f


def test_fisp_rejects_bad_state_count(cb, ctx, workloads):
    w = workloads.tiny()
    with pytest.raises(cb.CompasError):
        cb.FispSequence.from_dict(ctx, dict(w["seq"], max_state=129))
    # context still usable afterwards
    params, seq, _ = _upload(cb, ctx, w)
    assert np.isfinite(cb.simulate_magnetization(ctx, params, seq).to_numpy()).all()


# ------------------------------------------------------------------------------------------------
# against the reference's own kernels
# ------------------------------------------------------------------------------------------------

@pytest.mark.parametrize("kind", ["fisp", "pssfp"])
def test_simulation_matches_reference_kernels(cb, ctx, ref_simulations, oracle, kind):
    # golden echoes of the reference's FISP / pSSFP kernels (run on the CPU in FP32); both FP32
    # results lie within 1e-5 of the FP64 oracle, so they agree to 2e-5. FISP cases without the
    # inversion prepulse or the wait spoiling (which the reference's C ABI always sets) are built
    # through compas_b200_make_fisp_sequence_ex.
    tried, flagless = 0, 0
    for i, (p, seq, echos) in enumerate(ref_simulations[kind]):
        s = (cb.FispSequence if kind == "fisp" else cb.pSSFPSequence).from_dict(ctx, seq)
        got = cb.simulate_magnetization(ctx, cb.TissueParameters.from_soa(ctx, p), s).to_numpy()
        assert oracle.rel_l2(got, echos) < 2e-5, (kind, i)
        tried += 1
        flagless += kind == "fisp" and not (seq["inversion"] and seq["wait_spoil"])
    assert tried >= 3
    if kind == "fisp":
        assert flagless >= 1


def test_operators_match_reference_kernels(cb, ctx, ref_simulations, oracle):
    # phase encoding, every signal method, every Jacobian method, the residual and the spiral signal
    # against the outputs of the reference's own naive kernels (FP32 on the CPU, within 3e-7 of the
    # FP64 oracle): the plain FP32 methods to 1e-5 and the split-BF16 ones to 1e-4, plus that 3e-7
    c = ref_simulations["cartesian"]
    params = cb.TissueParameters.from_soa(ctx, c["params"])
    traj = cb.trajectory_from_dict(ctx, c["traj"])
    got = cb.phase_encoding(ctx, c["echos"], params, traj).to_numpy()
    assert oracle.rel_l2(got, c["phase_encoded"]) < TOL_FP32
    for m in PLAIN_SIGNAL + TC_SIGNAL:
        got = cb.magnetization_to_signal(ctx, c["echos"], params, traj, c["coils"], method=m).to_numpy()
        assert oracle.rel_l2(got, c["signal"]) < (TOL_FP32 if m in PLAIN_SIGNAL else TOL_BF16X3), m
    d = {"T1": c["dT1"], "T2": c["dT2"]}
    for m in PLAIN_JAC + TC_JAC:
        tol = TOL_FP32 if m in PLAIN_JAC else TOL_BF16X3
        jv = cb.compute_jacobian(ctx, c["echos"], d, params, traj, c["coils"], c["v"], method=m).to_numpy()
        assert oracle.rel_l2(jv, c["jv"]) < tol, ("J·v", m)
        jhv = cb.compute_jacobian_hermitian(ctx, c["echos"], d, params, traj, c["coils"], c["u"], method=m).to_numpy()
        assert oracle.rel_l2(jhv, c["jhv"]) < tol, ("Jᴴ·v", m)
    obj, diff = cb.compute_residual(ctx, c["signal"].astype(np.complex64), c["rhs"])
    assert oracle.rel_l2(diff.to_numpy(), c["residual"]) < TOL_FP32
    assert abs(obj - c["objective"]) < TOL_FP32 * c["objective"]
    s = ref_simulations["spiral"]
    params = cb.TissueParameters.from_soa(ctx, s["params"])
    traj = cb.trajectory_from_dict(ctx, s["traj"])
    for m in ("Direct", "MatmulFast"):
        got = cb.magnetization_to_signal(ctx, s["echos"], params, traj, s["coils"], method=m).to_numpy()
        assert oracle.rel_l2(got, s["signal"]) < (TOL_FP32 if m == "Direct" else TOL_BF16X3), ("spiral", m)


# ------------------------------------------------------------------------------------------------
# pSSFP
# ------------------------------------------------------------------------------------------------

@pytest.mark.parametrize("nz", [1, 5, 35])
def test_pssfp_every_layout(cb, ctx, oracle, workloads, nz):
    rng = np.random.default_rng(nz)
    seq = workloads.pssfp_sequence(rng, 23, nrf=7, nz=nz)
    p = workloads.tissue(rng, 5, 20.0)
    params = cb.TissueParameters.from_soa(ctx, p)
    s = cb.pSSFPSequence.from_dict(ctx, seq)
    ref = oracle.pssfp(p, seq)
    tried = 0
    try:
        for i, (zt, gz) in enumerate(cb.pssfp_configs()):
            if zt * gz < nz:
                continue
            cb.set_pssfp_launch(i)
            got = cb.simulate_magnetization(ctx, params, s).to_numpy()
            assert oracle.rel_l2(got, ref) < TOL_FP32, (zt, gz)
            tried += 1
    finally:
        cb.set_pssfp_launch(-1)
    assert tried > 0


def test_pssfp_large_rotations(cb, ctx, oracle, workloads):
    # flip angles of 120° per TR and strong off-resonance exercise the sincos branch
    rng = np.random.default_rng(4)
    seq = workloads.pssfp_sequence(rng, 17, nrf=3, nz=9)
    seq["rf"] = (seq["rf"] * 3).astype(np.complex64)
    p = workloads.tissue(rng, 4, 20.0)
    p[3] *= 20
    got = cb.simulate_magnetization(ctx, cb.TissueParameters.from_soa(ctx, p), cb.pSSFPSequence.from_dict(ctx, seq))
    assert oracle.rel_l2(got.to_numpy(), oracle.pssfp(p, seq)) < TOL_FP32


@pytest.mark.parametrize("scale,phase", [(1, 0.0), (3, 0.0), (1, 0.4)])
def test_pssfp_packed_layouts_match_scalar_bits(cb, ctx, workloads, scale, phase):
    # a two-wide layout runs the scalar update's operations on pairs of isochromats and sums them in
    # the scalar order: the same bits as the scalar layout with as many isochromats per lane; at 3x
    # the flip angles (and 20x the off-resonance) some pairs take the sincos branch. With a real RF
    # train (phase 0) the packed layouts run their real-RF form, without the products of the zero
    # axis component a_y: still the scalar bits (up to the sign of exact zeros)
    rng = np.random.default_rng(12 + scale)
    seq = workloads.pssfp_sequence(rng, 19, nrf=5, nz=3)
    seq["rf"] = (seq["rf"] * scale * np.exp(1j * phase * rng.uniform(-1, 1, len(seq["rf"])))).astype(np.complex64)
    p = workloads.tissue(rng, 5, 20.0)
    p[3] *= 1 if scale == 1 else 20
    params = cb.TissueParameters.from_soa(ctx, p)
    s = cb.pSSFPSequence.from_dict(ctx, seq)
    configs = cb.pssfp_configs()
    pairs = [(i, j) for i, c in enumerate(configs) if cb.pssfp_config_packed(i) and c[0] * c[1] >= 3
             for j, d in enumerate(configs) if not cb.pssfp_config_packed(j) and tuple(d) == tuple(c)]
    assert len(pairs) >= 3
    try:
        for i, j in pairs:
            cb.set_pssfp_launch(i)
            packed = cb.simulate_magnetization(ctx, params, s).to_numpy()
            cb.set_pssfp_launch(j)
            scalar = cb.simulate_magnetization(ctx, params, s).to_numpy()
            assert np.array_equal(packed, scalar), configs[i]
    finally:
        cb.set_pssfp_launch(-1)


# ------------------------------------------------------------------------------------------------
# signal
# ------------------------------------------------------------------------------------------------

@pytest.mark.parametrize("method", PLAIN_SIGNAL + TC_SIGNAL)
def test_signal_cartesian_methods(cb, ctx, oracle, workloads, method):
    w = workloads.tiny(n_side=11, ntr=45, ns=33, nc=3)
    params, _, traj = _upload(cb, ctx, w)
    echo = workloads.cn(np.random.default_rng(2), (45, 121))
    got = cb.magnetization_to_signal(ctx, echo, params, traj, w["coils"], method=method).to_numpy()
    ref = oracle.signal_cartesian(echo, w["params"], w["traj"], w["coils"])
    tol = TOL_BF16X3 if method in TC_SIGNAL else TOL_FP32
    assert oracle.rel_l2(got, ref) < tol


@pytest.mark.parametrize("low", [0, 1])
def test_signal_cartesian_reference_entry_point(cb, ctx, oracle, workloads, low):
    w = workloads.fisp_small()
    params, seq, traj = _upload(cb, ctx, w)
    echos = cb.simulate_magnetization(ctx, params, seq)
    sig = cb.magnetization_to_signal(ctx, echos, params, traj, w["coils"], low_precision=bool(low)).to_numpy()
    ref = oracle.signal_cartesian(echos.to_numpy(), w["params"], w["traj"], w["coils"])
    assert oracle.rel_l2(sig, ref) < TOL_BF16X3


@pytest.mark.parametrize("method", ["Direct", "MatmulFast"])
def test_signal_mrstat_scale_sampled(cb, ctx, oracle, workloads, method):
    w = workloads.mrstat()
    params, seq, traj = _upload(cb, ctx, w)
    rng = np.random.default_rng(5)
    echo = cb.simulate_magnetization(ctx, params, seq)
    sig = cb.magnetization_to_signal(ctx, echo, params, traj, w["coils"], method=method).to_numpy()
    ent = np.stack([rng.integers(0, 4, 192), rng.integers(0, 1120, 192), rng.integers(0, 224, 192)], 1)
    ref = oracle.signal_cartesian(echo.to_numpy(), w["params"], w["traj"], w["coils"], entries=ent)
    got = sig[ent[:, 0], ent[:, 1], ent[:, 2]]
    tol = TOL_BF16X3 if method == "MatmulFast" else TOL_FP32
    assert oracle.rel_l2(got, ref) < tol


@pytest.mark.parametrize("method", ["MatmulFast", "Direct"])
def test_signal_spiral_long_readouts(cb, ctx, oracle, workloads, method):
    # 1100 samples = 9 sample tiles of the tensor-core kernel (one W warp covers tiles 0 and 8)
    rng = np.random.default_rng(31)
    p = workloads.tissue(rng, 7, 22.4)
    traj = workloads.spiral(rng, 5, 1100, 22.4, 4e-6)
    coils = workloads.cn(rng, (3, 49))
    echo = workloads.cn(rng, (5, 49))
    got = cb.magnetization_to_signal(ctx, echo, cb.TissueParameters.from_soa(ctx, p), cb.trajectory_from_dict(ctx, traj),
                                     coils, method=method).to_numpy()
    ref = oracle.signal_spiral(echo, p, traj, coils)
    assert oracle.rel_l2(got, ref) < (TOL_FP32 if method == "Direct" else TOL_BF16X3)


def test_signal_spiral_readout_chunks_bitwise(cb, ctx, oracle, workloads, monkeypatch):
    # the tensor-core kernel runs the readouts in chunks bounded by the size of its per-voxel table;
    # a tiny budget (one readout per chunk) gives the same bits as one chunk
    rng = np.random.default_rng(32)
    p = workloads.tissue(rng, 9, 22.4)
    traj = workloads.spiral(rng, 6, 300, 22.4, 4e-6)
    coils = workloads.cn(rng, (4, 81))
    echo = workloads.cn(rng, (6, 81))
    args = (echo, cb.TissueParameters.from_soa(ctx, p), cb.trajectory_from_dict(ctx, traj), coils)
    whole = cb.magnetization_to_signal(ctx, *args, method="MatmulFast").to_numpy()
    monkeypatch.setenv("COMPAS_B200_SPIRAL_TABLE_BYTES", "1")
    chunked = cb.magnetization_to_signal(ctx, *args, method="MatmulFast").to_numpy()
    assert np.array_equal(whole, chunked)
    assert oracle.rel_l2(chunked, oracle.signal_spiral(echo, p, traj, coils)) < TOL_BF16X3


@pytest.mark.parametrize("nc", [1, 3, 11, 20])
@pytest.mark.parametrize("method", [None, "MatmulFast", "Direct"])
def test_signal_spiral(cb, ctx, oracle, workloads, method, nc):
    # None: the reference's spiral C-ABI entry point (split-BF16 tensor cores here, like the
    # Cartesian entry point with low_precision = 0); 300 samples = 3 ragged sample tiles; 3/11/20
    # coils = one 8-coil group, one 16-coil group, two 16-coil groups
    rng = np.random.default_rng(8 + nc)
    p = workloads.tissue(rng, 9, 22.4)
    traj = workloads.spiral(rng, 13, 300, 22.4, 4e-6)
    coils = workloads.cn(rng, (nc, 81))
    echo = workloads.cn(rng, (13, 81))
    params = cb.TissueParameters.from_soa(ctx, p)
    t = cb.trajectory_from_dict(ctx, traj)
    got = cb.magnetization_to_signal(ctx, echo, params, t, coils, method=method).to_numpy()
    ref = oracle.signal_spiral(echo, p, traj, coils)
    tol = TOL_FP32 if method == "Direct" else TOL_BF16X3
    assert oracle.rel_l2(got, ref) < tol


# ------------------------------------------------------------------------------------------------
# Jacobian products
# ------------------------------------------------------------------------------------------------

def _jac_case(workloads, rng, n_side=9, nr=37, ns=29, nc=3):
    p = workloads.tissue(rng, n_side, 22.4)
    nv = n_side * n_side
    traj = workloads.cartesian(nr, ns, 22.4, 5e-6, nr)
    coils = workloads.cn(rng, (nc, nv))
    e, d1, d2 = (workloads.cn(rng, (nr, nv)) for _ in range(3))
    return p, traj, coils, e, d1, d2


@pytest.mark.parametrize("method", PLAIN_JAC + TC_JAC)
def test_jacobian(cb, ctx, oracle, workloads, method):
    rng = np.random.default_rng(21)
    p, traj, coils, e, d1, d2 = _jac_case(workloads, rng)
    v = workloads.cn(rng, (4, p.shape[1]))
    params = cb.TissueParameters.from_soa(ctx, p)
    t = cb.trajectory_from_dict(ctx, traj)
    got = cb.compute_jacobian(ctx, e, {"T1": d1, "T2": d2}, params, t, coils, v, method=method).to_numpy()
    ref = oracle.jacobian(e, d1, d2, p, traj, coils, v)
    assert oracle.rel_l2(got, ref) < (TOL_BF16X3 if method in TC_JAC else TOL_FP32)


@pytest.mark.parametrize("nr", [257, 400, 743])
def test_cartesian_ragged_readout_counts(cb, ctx, oracle, workloads, nr):
    # readout counts that do not fill whole 256-readout tiles: the tensor-core contractions take
    # the fewest tiles, ceil(R / ceil(R / 256)) readouts each rounded up to 16 (743: 3 tiles of 256,
    # the last holding 231 readouts); split-BF16 signal and J·v against the FP64 oracle
    rng = np.random.default_rng(nr)
    p, traj, coils, e, d1, d2 = _jac_case(workloads, rng, nr=nr)
    params = cb.TissueParameters.from_soa(ctx, p)
    t = cb.trajectory_from_dict(ctx, traj)
    sig = cb.magnetization_to_signal(ctx, e, params, t, coils, method="MatmulFast").to_numpy()
    assert oracle.rel_l2(sig, oracle.signal_cartesian(e, p, traj, coils)) < TOL_BF16X3
    v = workloads.cn(rng, (4, p.shape[1]))
    jv = cb.compute_jacobian(ctx, e, {"T1": d1, "T2": d2}, params, t, coils, v, method="GemmFast").to_numpy()
    assert oracle.rel_l2(jv, oracle.jacobian(e, d1, d2, p, traj, coils, v)) < TOL_BF16X3


@pytest.mark.parametrize("method", PLAIN_JAC + TC_JAC)
@pytest.mark.parametrize("nc", [1, 5])
def test_jacobian_hermitian(cb, ctx, oracle, workloads, method, nc):
    rng = np.random.default_rng(22 + nc)
    p, traj, coils, e, d1, d2 = _jac_case(workloads, rng, nc=nc)
    u = workloads.cn(rng, (nc, traj["nr"], traj["ns"]))
    params = cb.TissueParameters.from_soa(ctx, p)
    t = cb.trajectory_from_dict(ctx, traj)
    got = cb.compute_jacobian_hermitian(ctx, e, {"T1": d1, "T2": d2}, params, t, coils, u, method=method).to_numpy()
    ref = oracle.jacobian_hermitian(e, d1, d2, p, traj, coils, u)
    assert oracle.rel_l2(got, ref) < (TOL_BF16X3 if method in TC_JAC else TOL_FP32)


def test_jacobian_adjointness_on_gpu(cb, ctx, workloads):
    rng = np.random.default_rng(31)
    p, traj, coils, e, d1, d2 = _jac_case(workloads, rng, n_side=13, nr=50, ns=40, nc=4)
    v = workloads.cn(rng, (4, p.shape[1]))
    u = workloads.cn(rng, (4, 50, 40))
    params = cb.TissueParameters.from_soa(ctx, p)
    t = cb.trajectory_from_dict(ctx, traj)
    for m in ("Direct", "GemmFast"):
        jv = cb.compute_jacobian(ctx, e, {"T1": d1, "T2": d2}, params, t, coils, v, method=m).to_numpy()
        jhu = cb.compute_jacobian_hermitian(ctx, e, {"T1": d1, "T2": d2}, params, t, coils, u, method=m).to_numpy()
        lhs = np.vdot(u.astype(complex), jv.astype(complex))
        rhs = np.vdot(jhu.astype(complex), v.astype(complex))
        assert abs(lhs - rhs) / abs(lhs) < (1e-5 if m == "Direct" else 1e-4), m


# ------------------------------------------------------------------------------------------------
# phase encoding, residual, derivatives, edge cases
# ------------------------------------------------------------------------------------------------

def test_phase_encoding(cb, ctx, oracle, workloads):
    w = workloads.fisp_small()
    params, _, traj = _upload(cb, ctx, w)
    echo = workloads.cn(np.random.default_rng(3), (400, 4096))
    got = cb.phase_encoding(ctx, echo, params, traj).to_numpy()
    assert oracle.rel_l2(got, oracle.phase_encoding(echo, w["params"], w["traj"]["k_start"])) < TOL_FP32
    # an odd voxel count: the elements are the same bits as in the full array
    odd = 4095
    p_odd = cb.TissueParameters.from_soa(ctx, np.ascontiguousarray(w["params"][:, :odd]))
    got_odd = cb.phase_encoding(ctx, np.ascontiguousarray(echo[:, :odd]), p_odd, traj).to_numpy()
    assert np.array_equal(got_odd, got[:, :odd])


def test_residual(cb, ctx, oracle):
    rng = np.random.default_rng(12)
    a = (rng.standard_normal((3, 70, 33)) + 1j * rng.standard_normal((3, 70, 33))).astype(np.complex64)
    b = (rng.standard_normal((3, 70, 33)) + 1j * rng.standard_normal((3, 70, 33))).astype(np.complex64)
    obj, d = cb.compute_residual(ctx, a, b)
    obj_ref, d_ref = oracle.residual(a, b)
    assert np.allclose(d.to_numpy(), d_ref, atol=1e-6)
    assert abs(obj - obj_ref) / obj_ref < 1e-5


@pytest.mark.parametrize("kind", ["fisp", "pssfp"])
def test_derivative(cb, ctx, oracle, workloads, kind):
    rng = np.random.default_rng(40)
    if kind == "fisp":
        w = workloads.tiny(n_side=5, ntr=31, P=2, max_state=6)
        seqd, sim = w["seq"], oracle.fisp
        p = w["params"]
        seq = cb.FispSequence.from_dict(ctx, seqd)
    else:
        seqd = workloads.pssfp_sequence(rng, 19, nrf=5, nz=6)
        p = workloads.tissue(rng, 5, 20.0)
        seq, sim = cb.pSSFPSequence.from_dict(ctx, seqd), oracle.pssfp
    params = cb.TissueParameters.from_soa(ctx, p)
    echos = cb.simulate_magnetization(ctx, params, seq)
    delta = 1e-3
    for field in (0, 1):
        got = cb.simulate_magnetization_derivative(ctx, field, echos, params, seq, delta).to_numpy()
        q = p.copy()
        q[field] = (p[field].astype(np.float32) + np.float32(delta)).astype(np.float32)
        ref = (sim(q, seqd) - sim(p, seqd)) / np.float32(delta)
        # FP32 forward differences: the GPU and oracle echoes differ by ~1e-7 relative, amplified by 1/Δ
        assert oracle.rel_l2(got, ref) < 5e-3, field


def test_single_voxel_single_readout(cb, ctx, oracle, workloads):
    w = workloads.tiny(n_side=1, ntr=1, ns=1, nc=1, P=1, max_state=1)
    params, seq, traj = _upload(cb, ctx, w)
    e = cb.simulate_magnetization(ctx, params, seq)
    assert oracle.rel_l2(e.to_numpy(), oracle.fisp(w["params"], w["seq"])) < TOL_FP32
    for m in ("Direct", "MatmulFast"):
        s = cb.magnetization_to_signal(ctx, e, params, traj, w["coils"], method=m).to_numpy()
        ref = oracle.signal_cartesian(e.to_numpy(), w["params"], w["traj"], w["coils"])
        assert oracle.rel_l2(s, ref) < TOL_BF16X3


def test_shape_mismatch_raises(cb, ctx, workloads):
    w = workloads.tiny()
    params, _, traj = _upload(cb, ctx, w)
    with pytest.raises(cb.CompasError):
        cb.magnetization_to_signal(ctx, np.zeros((3, 3), np.complex64), params, traj, w["coils"])


def test_empty_voxel_set(cb, ctx, workloads):
    # zero voxels: every operation returns correctly shaped empty or all-zero results (the
    # products are sums over voxels) without launching a kernel over an empty grid
    w = workloads.tiny(n_side=4, ntr=11, ns=6, nc=2, P=2, max_state=5)
    empty = np.zeros((9, 0), np.float32)
    params = cb.TissueParameters.from_soa(ctx, empty)
    seq = cb.FispSequence.from_dict(ctx, w["seq"])
    traj = cb.trajectory_from_dict(ctx, w["traj"])
    coils = np.zeros((2, 0), np.complex64)
    e = cb.simulate_magnetization(ctx, params, seq)
    assert e.to_numpy().shape == (11, 0)
    rng = np.random.default_rng(2)
    ps = cb.pSSFPSequence.from_dict(ctx, workloads.pssfp_sequence(rng, 9, nrf=3, nz=5))
    assert cb.simulate_magnetization(ctx, params, ps).to_numpy().shape == (9, 0)
    for seqx, nr in ((seq, 11), (ps, 9)):
        t = cb.simulate_magnetization_tangents(ctx, params, seqx)
        assert all(t[k].to_numpy().shape == (nr, 0) for k in ("echos", "T1", "T2"))
    d = {"T1": e, "T2": e}
    for m in PLAIN_SIGNAL + TC_SIGNAL:
        s = cb.magnetization_to_signal(ctx, e, params, traj, coils, method=m).to_numpy()
        assert s.shape == (2, 11, 6) and not s.any(), m
    for m in PLAIN_JAC + TC_JAC:
        jv = cb.compute_jacobian(ctx, e, d, params, traj, coils, np.zeros((4, 0), np.complex64), method=m)
        assert jv.to_numpy().shape == (2, 11, 6) and not jv.to_numpy().any(), m
        u = workloads.cn(rng, (2, 11, 6))
        jh = cb.compute_jacobian_hermitian(ctx, e, d, params, traj, coils, u, method=m)
        assert jh.to_numpy().shape == (4, 0), m
    st = workloads.spiral(rng, 11, 20, 22.4, 4e-6)
    s = cb.magnetization_to_signal(ctx, e, params, cb.trajectory_from_dict(ctx, st), coils).to_numpy()
    assert s.shape == (2, 11, 20) and not s.any()
