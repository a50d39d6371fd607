"""CPU tests of the oracle itself: pinned against the reference's own complex
arithmetic (golden vectors), analytic known answers and structural identities.
No GPU, no product code."""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).parent / "golden" / "ref_complex_ops.json"


def _ulp_close(a, b, ulps=4):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    tol = ulps * np.spacing(np.maximum(np.abs(a), np.abs(b)).astype(np.float32))
    return np.all(np.abs(a - b) <= tol + 1e-30)


# ---------------------------------------------------------------------------------------------
# golden vectors from compas-toolkit include/compas/core/complex_type.h (host build)
# ---------------------------------------------------------------------------------------------

@pytest.mark.parametrize("op,name,nin", [(0, "exp", 2), (1, "pow", 3), (2, "fma", 6), (3, "mul", 4)])
def test_twin_complex_ops_match_reference(oracle, op, name, nin):
    g = np.array(json.loads(GOLDEN.read_text())[name], np.float32)
    got = oracle.cx_eval_f32(op, g[:, :nin])
    want = g[:, nin:nin + 2]
    # same formulas, same FP32 libm calls: within a few ulp (sin/cos of |x|~60 rad amplify by |x|)
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-3)
    assert rel.max() < 2e-5, (name, rel.max())
    if name in ("fma", "mul"):
        assert _ulp_close(got, want, 2)


# ---------------------------------------------------------------------------------------------
# FISP / EPG
# ---------------------------------------------------------------------------------------------

def _one_voxel(T1=0.8, T2=0.06, B1=1.0, B0=0.0, rho=1.0, x=0.0, y=0.0, z=0.0):
    p = np.zeros((9, 1), np.float32)
    p[:, 0] = [T1, T2, B1, B0, np.real(rho), np.imag(rho), x, y, z]
    return p


@pytest.mark.parametrize("kind", ["fisp", "pssfp"])
def test_oracle_matches_reference_kernels(oracle, ref_simulations, kind):
    # echoes of the reference's own FISP / pSSFP kernels (run on the CPU, FP32): the FP64 oracle
    # agrees to FP32 rounding, the FP32 twin (the reference's arithmetic order) to ~1e-7
    sim = oracle.fisp if kind == "fisp" else oracle.pssfp
    for i, (p, seq, echos) in enumerate(ref_simulations[kind]):
        assert oracle.rel_l2(sim(p, seq), echos) < 1e-5, (kind, i)
        assert oracle.rel_l2(sim(p, seq, dtype="f32"), echos) < 1e-6, (kind, i)


def test_oracle_operators_match_reference_kernels(oracle, ref_simulations):
    # phase encoding, the naive Cartesian signal, J·v, Jᴴ·v, the residual and the spiral signal of
    # the reference's kernels (FP32 on the CPU) against the FP64 oracle: FP32 rounding only
    c = ref_simulations["cartesian"]
    p, t = c["params"], c["traj"]
    assert oracle.rel_l2(oracle.phase_encoding(c["echos"], p, t["k_start"]), c["phase_encoded"]) < 1e-6
    assert oracle.rel_l2(oracle.signal_cartesian(c["echos"], p, t, c["coils"]), c["signal"]) < 1e-6
    assert oracle.rel_l2(oracle.signal_cartesian(c["echos"], p, t, c["coils"], dtype="f32"), c["signal"]) < 1e-7
    jv = oracle.jacobian(c["echos"], c["dT1"], c["dT2"], p, t, c["coils"], c["v"])
    assert oracle.rel_l2(jv, c["jv"]) < 1e-6
    jhv = oracle.jacobian_hermitian(c["echos"], c["dT1"], c["dT2"], p, t, c["coils"], c["u"])
    assert oracle.rel_l2(jhv, c["jhv"]) < 1e-6
    obj, diff = oracle.residual(c["signal"].astype(np.complex64), c["rhs"])
    assert oracle.rel_l2(diff, c["residual"]) < 1e-6 and abs(obj - c["objective"]) < 1e-6 * obj
    s = ref_simulations["spiral"]
    assert oracle.rel_l2(oracle.signal_spiral(s["echos"], s["params"], s["traj"], s["coils"]), s["signal"]) < 1e-6


def test_reference_kernel_library_matches_oracle(oracle, workloads):
    # oracle/_ref/libref_kernels.so (the reference's simulate_fisp and naive Cartesian signal built
    # for the host; the CPU baseline of bench.py) against the FP64 oracle on a threaded run
    if oracle.ref_kernels() is None:
        pytest.skip("oracle/_ref/libref_kernels.so not built (no reference tree at build time)")
    w = workloads.tiny(n_side=6, ntr=29, P=3, max_state=25, seed=5)
    w["seq"]["reps"], w["seq"]["uf"], w["seq"]["TW"] = 2, 2, 0.02
    idx = np.array([0, 5, 17, 35])
    ref = oracle.fisp(w["params"], w["seq"], vidx=idx)
    assert oracle.rel_l2(oracle.ref_fisp(w["params"], w["seq"], vidx=idx, nthreads=3), ref) < 1e-5
    assert oracle.rel_l2(oracle.ref_fisp(w["params"], w["seq"], nthreads=4)[:, idx], ref) < 1e-5
    echo = workloads.cn(np.random.default_rng(6), (29, 36))
    ent = np.array([[0, 0, 0], [2, 13, 6], [1, 28, 3]])
    got = oracle.ref_signal_cartesian(echo, w["params"], w["traj"], w["coils"], ent, nthreads=2)
    want = oracle.signal_cartesian(echo, w["params"], w["traj"], w["coils"], entries=ent)
    assert oracle.rel_l2(got, want) < 1e-5


def test_fisp_zero_rf_gives_zero_echo(oracle, workloads):
    seq = workloads.fisp_sequence(np.zeros(20), np.ones((2, 20)), 8e-3, 4e-3, 20e-3, 6)
    e = oracle.fisp(_one_voxel(), seq)
    assert np.all(e == 0)


def test_fisp_single_hard_pulse_known_answer(oracle, workloads):
    # N=1, no inversion, one 90° pulse with phase φ: F+0 = -i e^{iφ} sinα · Z0, then decay to TE
    # (epg.cuh:73-81 convention R13 = (sinφ sinα, -cosφ sinα)).
    phi = 0.3
    TE, T2, B0 = 4e-3, 0.05, 7.0
    seq = workloads.fisp_sequence(np.array([90.0 * np.exp(1j * phi)]), np.ones((1, 1)), 8e-3, TE, 20e-3, 1)
    seq["inversion"] = 0
    e = oracle.fisp(_one_voxel(T2=T2, B0=B0), seq)[0, 0]
    f = lambda q: float(np.float32(q))  # inputs are stored as float32
    rf = complex(seq["rf"][0])
    want = -1j * (rf / abs(rf)) * np.exp(-f(TE) / f(T2)) * np.exp(2j * np.pi * f(B0) * f(TE))
    assert abs(e - want) < 1e-12


def test_fisp_relaxation_after_inversion(oracle, workloads):
    # one tiny-flip readout after inversion: Z0 = 1 - 2 e^{-TI/T1}; F+0 ≈ -i sinα Z0 e^{-TE/T2}
    T1, T2, TI, TE = 1.1, 0.09, 0.4, 3e-3
    a = 1e-3
    seq = workloads.fisp_sequence(np.array([a]), np.ones((1, 1)), 8e-3, TE, TI, 3)
    e = oracle.fisp(_one_voxel(T1=T1, T2=T2), seq)[0, 0]
    f = lambda q: float(np.float32(q))
    Z0 = 1 - 2 * np.exp(-f(TI) / f(T1))
    want = -1j * np.sin(np.deg2rad(f(a))) * Z0 * np.exp(-f(TE) / f(T2))
    assert abs(e - want) < 1e-9


def test_derivative_central_known_answer(oracle, workloads):
    # the readout above, e = -i sinα (1 - 2 e^{-TI/T1}) e^{-TE/T2}, differentiated in closed form:
    # ∂e/∂T1 = -i sinα (-2 e^{-TI/T1} TI/T1²) e^{-TE/T2},  ∂e/∂T2 = e·TE/T2²
    T1, T2, TI, TE, a = 1.1, 0.09, 0.4, 3e-3, 1e-3
    seq = workloads.fisp_sequence(np.array([a]), np.ones((1, 1)), 8e-3, TE, TI, 3)
    p = _one_voxel(T1=T1, T2=T2)
    f = lambda q: float(np.float32(q))
    sa, E2 = np.sin(np.deg2rad(f(a))), np.exp(-f(TE) / f(T2))
    e = -1j * sa * (1 - 2 * np.exp(-f(TI) / f(T1))) * E2
    d1 = -1j * sa * (-2 * np.exp(-f(TI) / f(T1)) * f(TI) / f(T1) ** 2) * E2
    d2 = e * f(TE) / f(T2) ** 2
    got1 = oracle.derivative_central(oracle.fisp, p, seq, 0)[0, 0]
    got2 = oracle.derivative_central(oracle.fisp, p, seq, 1)[0, 0]
    # O(step²) truncation at a relative step of 1e-4
    assert abs(got1 - d1) < 1e-7 * abs(d1) and abs(got2 - d2) < 1e-7 * abs(d2)


@pytest.mark.parametrize("kind", ["fisp", "pssfp"])
def test_derivative_central_converges(oracle, workloads, kind):
    # central differences at two steps agree to O(step²): the FP64 derivative oracle has converged
    rng = np.random.default_rng(9)
    if kind == "fisp":
        w = workloads.tiny(n_side=3, ntr=31, P=2, max_state=6)
        p, seqd, sim = w["params"], w["seq"], oracle.fisp
    else:
        seqd = workloads.pssfp_sequence(rng, 19, nrf=5, nz=6)
        p, sim = workloads.tissue(rng, 3, 20.0), oracle.pssfp
    for field in (0, 1):
        coarse = oracle.derivative_central(sim, p, seqd, field, rel_step=1e-3)
        fine = oracle.derivative_central(sim, p, seqd, field, rel_step=1e-4)
        assert oracle.rel_l2(coarse, fine) < 1e-5, field


def test_fisp_b0_conjugate_symmetry(oracle, workloads):
    # real RF: the EPG evolution under -B0 is D·conj(evolution under +B0) with D = diag(-1,-1,1)
    w = workloads.tiny()
    seq = dict(w["seq"])
    seq["rf"] = np.abs(seq["rf"]).astype(np.complex64)
    seq["slices"] = np.abs(seq["slices"]).astype(np.complex64)
    p = w["params"].copy()
    q = p.copy()
    q[3] = -q[3]
    e1 = oracle.fisp(p, seq)
    e2 = oracle.fisp(q, seq)
    assert np.abs(e2 + np.conj(e1)).max() < 1e-12


def _textbook_epg(T1, T2, B1, B0, seq):
    """Independent EPG (Weigel 2015 convention) in numpy: explicit 3x3 rotation T(α,φ),
    relaxation, gradient shift with F̃0 = conj(F̃-0). Single voxel, full control flow."""
    N = seq["max_state"]
    nTR = len(seq["rf"])
    out = np.zeros(nTR * seq["uf"], complex)
    for pos in range(seq["slices"].shape[0]):
        F = np.zeros((3, N), complex)
        F[2, 0] = 1
        for rep in range(seq["reps"]):
            if seq["inversion"]:
                F[2] *= -1
                F[0:2] = 0
                F[:2] *= np.exp(-seq["TI"] / T2)
                F[2] *= np.exp(-seq["TI"] / T1)
                F[2, 0] += 1 - np.exp(-seq["TI"] / T1)
            for t in range(nTR):
                rf = complex(seq["slices"][pos, t]) * complex(seq["rf"][t])
                a = np.deg2rad(abs(rf)) * B1
                ph = np.angle(rf)
                Tm = np.array([
                    [np.cos(a / 2) ** 2, np.exp(2j * ph) * np.sin(a / 2) ** 2, -1j * np.exp(1j * ph) * np.sin(a)],
                    [np.exp(-2j * ph) * np.sin(a / 2) ** 2, np.cos(a / 2) ** 2, 1j * np.exp(-1j * ph) * np.sin(a)],
                    [-0.5j * np.exp(-1j * ph) * np.sin(a), 0.5j * np.exp(1j * ph) * np.sin(a), np.cos(a)]])
                F = Tm @ F
                for half, dtt in enumerate((seq["TE"], seq["TR"] - seq["TE"])):
                    r = np.exp(2j * np.pi * B0 * dtt)
                    F[0] *= np.exp(-dtt / T2) * r
                    F[1] *= np.exp(-dtt / T2) * np.conj(r)
                    F[2] *= np.exp(-dtt / T1)
                    F[2, 0] += 1 - np.exp(-dtt / T1)
                    if half == 0 and rep == seq["reps"] - 1:
                        for q in range(seq["uf"]):
                            out[t * seq["uf"] + q] += F[0, 0]
                # dephasing gradient: F- down, F+ up, F+0 = conj(F-0), truncate at N-1
                F[1, :-1] = F[1, 1:]
                F[1, N - 1] = 0
                F[0, 1:] = F[0, :-1].copy()
                F[0, 0] = np.conj(F[1, 0])
            F[0:2] = 0
    return out


def test_fisp_matches_independent_textbook_epg(oracle, workloads):
    w = workloads.tiny(max_state=4)
    seq = dict(w["seq"])
    seq["uf"] = 2
    for key in ("TR", "TE", "TI"):
        seq[key] = float(np.float32(seq[key]))  # the oracle receives float32 scalars
    p = w["params"]
    e = oracle.fisp(p, seq)
    for v in range(0, p.shape[1], 7):
        ref = _textbook_epg(*[float(p[i, v]) for i in range(4)], seq)
        assert np.abs(e[:, v] - ref).max() < 1e-10


def test_fisp_twin_close_to_f64(oracle, workloads):
    w = workloads.fisp_small()
    idx = np.arange(0, w["params"].shape[1], 97)
    e64 = oracle.fisp(w["params"], w["seq"], vidx=idx)
    e32 = oracle.fisp(w["params"], w["seq"], vidx=idx, dtype="f32")
    assert oracle.rel_l2(e32, e64) < 1e-5


def test_fisp_repetitions_and_undersampling(oracle, workloads):
    w = workloads.tiny()
    seq = dict(w["seq"])
    seq["reps"], seq["uf"] = 3, 3
    e = oracle.fisp(w["params"], seq)
    assert e.shape[0] == len(seq["rf"]) * 3
    assert np.array_equal(e[0::3], e[1::3]) and np.array_equal(e[0::3], e[2::3])
    seq1 = dict(seq)
    seq1["reps"] = 1
    assert oracle.rel_l2(oracle.fisp(w["params"], seq1), e) > 1e-6  # repetitions change the steady state


# ---------------------------------------------------------------------------------------------
# pSSFP
# ---------------------------------------------------------------------------------------------

def test_pssfp_zero_rf_zero_echo(oracle, workloads):
    rng = np.random.default_rng(0)
    seq = workloads.pssfp_sequence(rng, 10, nrf=5, nz=4)
    seq["rf"] = np.zeros(10, np.complex64)
    e = oracle.pssfp(_one_voxel(B0=3.0), seq)
    assert np.all(np.abs(e) < 1e-15)


def test_pssfp_twin_close_to_f64(oracle, workloads):
    rng = np.random.default_rng(1)
    seq = workloads.pssfp_sequence(rng, 60, nrf=15, nz=35)
    p = workloads.tissue(rng, 4, 20.0)
    e64 = oracle.pssfp(p, seq)
    e32 = oracle.pssfp(p, seq, dtype="f32")
    assert oracle.rel_l2(e32, e64) < 1e-5


# ---------------------------------------------------------------------------------------------
# signal / Jacobian
# ---------------------------------------------------------------------------------------------

def test_signal_single_voxel_closed_form(oracle, workloads):
    T2, B0, x, y = 0.07, 11.0, 3.1, -2.0
    rho = 0.7 * np.exp(0.4j)
    p = _one_voxel(T2=T2, B0=B0, rho=rho, x=x, y=y)
    traj = workloads.cartesian(3, 9, 20.0, 1e-5, 3)
    echo = np.array([[0.3 + 0.1j], [0.2 - 0.5j], [-0.1 + 0.2j]], np.complex64)
    coils = np.array([[0.9 - 0.2j]], np.complex64)
    s = oracle.signal_cartesian(echo, p, traj, coils)
    dt, ns, dk = float(np.float32(traj["dt"])), traj["ns"], float(np.float32(traj["dk"]))
    R2 = 1 / np.float64(np.float32(T2))
    p64 = p.astype(np.float64)[:, 0]
    theta = dk * p64[6] + dt * 2 * np.pi * p64[3]
    for r in range(3):
        A = complex(echo[r, 0]) * complex(np.complex64(rho)) * np.exp(
            -0.5 * ns * dt * (-R2 + 2j * np.pi * p64[3]) + 1j * (-0.5 * ns * dk) * p64[6])
        k = np.arange(ns)
        want = complex(coils[0, 0]) * A * np.exp(k * (-dt * R2 + 1j * theta))
        assert np.abs(s[0, r] - want).max() < 1e-12


def _small_j(workloads, rng, nc=2, n_side=5, nr=6, ns=7):
    p = workloads.tissue(rng, n_side, 20.0)
    nv = n_side * n_side
    traj = workloads.cartesian(nr, ns, 20.0, 1e-5, nr)
    coils = workloads.cn(rng, (nc, nv))
    echo, d1, d2 = (workloads.cn(rng, (nr, nv)) for _ in range(3))
    return p, traj, coils, echo, d1, d2


def test_jacobian_adjointness(oracle, workloads):
    rng = np.random.default_rng(5)
    p, traj, coils, echo, d1, d2 = _small_j(workloads, rng)
    nv = p.shape[1]
    v = workloads.cn(rng, (4, nv))
    u = workloads.cn(rng, (coils.shape[0], traj["nr"], traj["ns"]))
    Jv = oracle.jacobian(echo, d1, d2, p, traj, coils, v)
    JHu = oracle.jacobian_hermitian(echo, d1, d2, p, traj, coils, u)
    lhs = np.vdot(u.astype(np.complex128), Jv)
    rhs = np.vdot(JHu, v.astype(np.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_jacobian_matches_finite_difference_of_signal(oracle, workloads):
    # analytic echo model m(T1,T2) with exact derivatives; J·v must equal the directional
    # derivative of the Cartesian signal (T-scaled T1/T2 columns, product_kernels.cuh:56-60)
    rng = np.random.default_rng(9)
    n_side, nr, ns, nc = 4, 5, 6, 2
    p = workloads.tissue(rng, n_side, 20.0).astype(np.float64)
    nv = n_side ** 2
    traj = workloads.cartesian(nr, ns, 20.0, 1e-5, nr)
    coils = workloads.cn(rng, (nc, nv))
    tr = np.linspace(0.01, 0.5, nr)[:, None]

    def model(T1, T2):
        m = (1 - 2 * np.exp(-tr / T1)) * np.exp(-0.004 / T2) * np.exp(1j * tr * 3)
        d1 = (-2 * np.exp(-tr / T1) * tr / T1 ** 2) * np.exp(-0.004 / T2) * np.exp(1j * tr * 3)
        d2 = (1 - 2 * np.exp(-tr / T1)) * np.exp(-0.004 / T2) * (0.004 / T2 ** 2) * np.exp(1j * tr * 3)
        return m, d1, d2

    m, d1, d2 = model(p[0], p[1])
    v = rng.standard_normal((4, nv))  # real directions: δT1 = h v0 T1, δT2 = h v1 T2, δρ = h (v2 + i v3)
    Jv = oracle.jacobian(m, d1, d2, p.astype(np.float32), traj, coils, v.astype(np.complex64))

    def sig(h):
        q = p.copy()
        q[0] = p[0] * (1 + h * v[0])
        q[1] = p[1] * (1 + h * v[1])
        q[4] = p[4] + h * v[2]
        q[5] = p[5] + h * v[3]
        mm, _, _ = model(q[0], q[1])
        return oracle.signal_cartesian(mm, q.astype(np.float32), traj, coils)

    # float32 parameter storage limits h; central difference with h=1e-3 and a loose bound
    h = 1e-3
    fd = (sig(h) - sig(-h)) / (2 * h)
    assert oracle.rel_l2(Jv, fd) < 2e-3


def test_cartesian_model_matches_signal_and_jacobian(oracle, workloads):
    # the FP64 model used for the finite-difference checks at full size: for a real Δk it is the
    # reference's naive Cartesian signal, and its central difference along v is the oracle's J·v
    rng = np.random.default_rng(19)
    p, traj, coils, echo, d1, d2 = _small_j(workloads, rng)
    nc, nr, ns = coils.shape[0], traj["nr"], traj["ns"]
    ent = np.array([(c, r, k) for c in range(nc) for r in range(nr) for k in range(ns)])
    q = p.astype(np.float64)
    rows = {r: echo[r].astype(np.complex128) for r in range(nr)}
    model = oracle.cartesian_model_entries(rows, q[1], q[3], q[6], q[7], q[4] + 1j * q[5], coils, traj, ent)
    sig = oracle.signal_cartesian(echo, p, traj, coils, entries=ent)
    assert oracle.rel_l2(model, sig) < 1e-12
    v = workloads.cn(rng, (4, p.shape[1]))
    fd = oracle.jacobian_fd_entries(echo, d1, d2, p, traj, coils, v, ent)
    assert oracle.rel_l2(fd, oracle.jacobian(echo, d1, d2, p, traj, coils, v, entries=ent)) < 1e-7


def _small_spiral_j(workloads, rng, n_side=4, nr=5, ns=7, nc=2):
    p = workloads.tissue(rng, n_side, 20.0)
    nv = n_side * n_side
    traj = workloads.spiral(rng, nr, ns, 20.0, 4e-6)
    coils = workloads.cn(rng, (nc, nv))
    echo, d1, d2 = (workloads.cn(rng, (nr, nv)) for _ in range(3))
    return p, traj, coils, echo, d1, d2


def test_spiral_jacobian_adjointness(oracle, workloads):
    # the spiral products have no counterpart in the reference; Jᴴ must be the exact adjoint of J
    rng = np.random.default_rng(15)
    p, traj, coils, echo, d1, d2 = _small_spiral_j(workloads, rng)
    nv = p.shape[1]
    v = workloads.cn(rng, (4, nv))
    u = workloads.cn(rng, (coils.shape[0], traj["nr"], traj["ns"]))
    Jv = oracle.spiral_jacobian(echo, d1, d2, p, traj, coils, v)
    JHu = oracle.spiral_jacobian_hermitian(echo, d1, d2, p, traj, coils, u)
    lhs = np.vdot(u.astype(np.complex128), Jv)
    rhs = np.vdot(JHu, v.astype(np.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_spiral_jacobian_matches_finite_difference_of_spiral_signal(oracle, workloads):
    # J·v on a spiral equals the directional derivative of the reference's spiral signal model
    # (rewind exp((S/2)Δt R2), z^k = exp(k(-Δt R2 + iΘ))) with the T-scaled columns
    rng = np.random.default_rng(19)
    n_side, nr, ns, nc = 4, 5, 6, 2
    p = workloads.tissue(rng, n_side, 20.0).astype(np.float64)
    nv = n_side ** 2
    traj = workloads.spiral(rng, nr, ns, 20.0, 4e-6)
    coils = workloads.cn(rng, (nc, nv))
    tr = np.linspace(0.01, 0.5, nr)[:, None]

    def model(T1, T2):
        m = (1 - 2 * np.exp(-tr / T1)) * np.exp(-0.004 / T2) * np.exp(1j * tr * 3)
        d1 = (-2 * np.exp(-tr / T1) * tr / T1 ** 2) * np.exp(-0.004 / T2) * np.exp(1j * tr * 3)
        d2 = (1 - 2 * np.exp(-tr / T1)) * np.exp(-0.004 / T2) * (0.004 / T2 ** 2) * np.exp(1j * tr * 3)
        return m, d1, d2

    m, d1, d2 = model(p[0], p[1])
    v = rng.standard_normal((4, nv))
    Jv = oracle.spiral_jacobian(m, d1, d2, p.astype(np.float32), traj, coils, v.astype(np.complex64))

    def sig(h):
        q = p.copy()
        q[0] = p[0] * (1 + h * v[0])
        q[1] = p[1] * (1 + h * v[1])
        q[4] = p[4] + h * v[2]
        q[5] = p[5] + h * v[3]
        mm, _, _ = model(q[0], q[1])
        return oracle.signal_spiral(mm, q.astype(np.float32), traj, coils)

    h = 1e-3
    fd = (sig(h) - sig(-h)) / (2 * h)
    assert oracle.rel_l2(Jv, fd) < 2e-3


def test_residual(oracle):
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((2, 3, 4)) + 1j * rng.standard_normal((2, 3, 4))).astype(np.complex64)
    b = (rng.standard_normal((2, 3, 4)) + 1j * rng.standard_normal((2, 3, 4))).astype(np.complex64)
    obj, d = oracle.residual(a, b)
    assert np.allclose(d, a.astype(complex) - b)
    assert abs(obj - np.sum(np.abs(a.astype(complex) - b) ** 2)) < 1e-9
