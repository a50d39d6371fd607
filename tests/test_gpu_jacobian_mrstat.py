"""J·v and Jᴴ·v at the MR-STAT Jacobian size: 224² = 50176 voxels, Cartesian 1120 readouts × 224
samples, 8 coils, random echoes and ∂echoes, v ~ CN(0,1) [4][V] and residual ~ CN(0,1) [8][1120][224]
(workloads.jacobian_inputs), through the C ABI.

The FP64 oracle cannot evaluate whole products of this size in a test, so each check samples:
  * J·v on 256 random (coil, readout, sample) entries, each summed over all 50176 voxels in FP64;
  * Jᴴ·v on 512 random voxels, each summed over all coils, readouts and samples in FP64;
  * J·v against an FP64 central difference of the forward model at a relative step h = 1e-4;
  * ⟨u, J·v⟩ = ⟨Jᴴ·u, v⟩ over the full arrays (a size-independent property).
Tolerances (relative L2): split-BF16 tensor-core methods 1e-4, plain FP32 methods 1e-5. The split-BF16
kernels bound the number of K16 steps one tensor-core accumulator sums (≤ 512 per voxel split), which
is what keeps them inside 1e-4 at K = 50176 voxels (J·v) and 8 × 1120 readouts (Jᴴ·v).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"GemmFast": 1e-4, None: 1e-4, "Direct": 1e-5}


@pytest.fixture(scope="module")
def cb():
    import compas_b200

    compas_b200.library()
    return compas_b200


@pytest.fixture(scope="module")
def ctx(cb):
    return cb.Context(0)


@pytest.fixture(scope="module")
def case(cb, ctx, workloads):
    w = workloads.jacobian_inputs()
    params = cb.TissueParameters.from_soa(ctx, w["params"])
    traj = cb.CartesianTrajectory.from_dict(ctx, w["traj"])
    arr = {k: cb.CompasArray.from_numpy(ctx, w[k]) for k in ("echo", "dT1", "dT2", "v", "r", "coils")}
    return w, params, traj, arr


def _jv(cb, ctx, case, method, v=None):
    w, params, traj, arr = case
    d = {"T1": arr["dT1"], "T2": arr["dT2"]}
    return cb.compute_jacobian(ctx, arr["echo"], d, params, traj, arr["coils"], arr["v"] if v is None else v,
                               method=method).to_numpy()


def _jhv(cb, ctx, case, method):
    w, params, traj, arr = case
    d = {"T1": arr["dT1"], "T2": arr["dT2"]}
    return cb.compute_jacobian_hermitian(ctx, arr["echo"], d, params, traj, arr["coils"], arr["r"],
                                         method=method).to_numpy()


def _entries(seed, n=256):
    rng = np.random.default_rng(seed)
    return np.stack([rng.integers(0, 8, n), rng.integers(0, 1120, n), rng.integers(0, 224, n)], 1)


@pytest.fixture(scope="module")
def jv_ref(case, oracle):
    w = case[0]
    ent = _entries(17)
    return ent, oracle.jacobian(w["echo"], w["dT1"], w["dT2"], w["params"], w["traj"], w["coils"], w["v"], entries=ent)


@pytest.mark.parametrize("method", [None, "GemmFast", "Direct"])
def test_jv_mrstat_sampled_fp64(cb, ctx, oracle, case, jv_ref, method):
    # None: the reference's C-ABI entry point with low_precision = 0 (split-BF16 here)
    ent, ref = jv_ref
    got = _jv(cb, ctx, case, method)
    assert got.shape == (8, 1120, 224) and np.isfinite(got).all()
    assert oracle.rel_l2(got[ent[:, 0], ent[:, 1], ent[:, 2]], ref) < TOL[method], method


@pytest.mark.parametrize("method", [None, "GemmFast", "Direct"])
def test_jhv_mrstat_sampled_fp64(cb, ctx, oracle, case, method):
    w = case[0]
    idx = np.sort(np.random.default_rng(18).choice(50176, 512, replace=False))
    got = _jhv(cb, ctx, case, method)
    assert got.shape == (4, 50176) and np.isfinite(got).all()
    ref = oracle.jacobian_hermitian(w["echo"], w["dT1"], w["dT2"], w["params"], w["traj"], w["coils"], w["r"],
                                    vidx=idx)
    assert oracle.rel_l2(got[:, idx], ref) < TOL[method], method


def test_jv_mrstat_matches_finite_difference(cb, ctx, oracle, case, jv_ref):
    # J·v is the directional derivative of the forward model s = Σ_v C·ρ·m·E_k(T2) along v (T1 and
    # T2 stepped relatively, ρ absolutely, echoes linearised): FP64 central difference, h = 1e-4
    w = case[0]
    ent = _entries(23, 96)
    fd = oracle.jacobian_fd_entries(w["echo"], w["dT1"], w["dT2"], w["params"], w["traj"], w["coils"], w["v"], ent,
                                    h=1e-4)
    ref = oracle.jacobian(w["echo"], w["dT1"], w["dT2"], w["params"], w["traj"], w["coils"], w["v"], entries=ent)
    assert oracle.rel_l2(ref, fd) < 1e-7  # the oracle's J·v is that derivative
    for method in ("GemmFast", "Direct"):
        got = _jv(cb, ctx, case, method)
        assert oracle.rel_l2(got[ent[:, 0], ent[:, 1], ent[:, 2]], fd) < TOL[method], method


@pytest.mark.parametrize("method", ["GemmFast", "Direct"])
def test_adjointness_mrstat(cb, ctx, case, method):
    # each side carries the product's own error (≤ TOL relative L2); an inner product with a random
    # vector does not average that error down, so the bound is a few times TOL
    w = case[0]
    jv = _jv(cb, ctx, case, method).astype(np.complex128)
    jhu = _jhv(cb, ctx, case, method).astype(np.complex128)
    lhs = np.vdot(w["r"].astype(np.complex128), jv)
    rhs = np.vdot(jhu, w["v"].astype(np.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 5 * TOL[method], method
