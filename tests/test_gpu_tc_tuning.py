"""Tensor-core contractions under the launches the autotuner can choose.

The readout tile of the Cartesian signal / J·v kernel and the split count of every contraction
change only how the work is distributed over CTAs and the FP32 order in which split partial sums
are added. Every accepted (tile, splits) must therefore meet the split-BF16 tolerance (relative L2
1e-4) against the FP64 oracle. Cases: 9000 voxels, Cartesian 480 readouts x 45 samples (readout
tiles 48, 96, 160 and 240 all cover 480 rows exactly; one split accumulates 282 stages of the signal
or 563 of J·v, i.e. folds its TMEM accumulator into the running sum 2 or 4 times), spiral 70
interleaves x 150 samples (at least 3 voxel splits for the signal and 5 for J·v, from the
512-K16-step accumulation bound of that kernel), 3 coils.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_BF16X3 = 1e-4
NV, NC = 9000, 3


@pytest.fixture(scope="module")
def cb():
    import compas_b200

    compas_b200.library()
    yield compas_b200
    for kind in compas_b200.TC_KINDS:
        compas_b200.set_tc_launch(kind, 0, 0)


@pytest.fixture(scope="module")
def ctx(cb):
    return cb.Context(0)


@pytest.fixture(scope="module")
def case(workloads):
    rng = np.random.default_rng(77)
    p = workloads.tissue_voxels(rng, NV, 22.4)
    cart = workloads.cartesian(480, 45, 22.4, 5e-6, 45)
    spir = workloads.spiral(rng, 70, 150, 22.4, 4e-6)
    coils = workloads.cn(rng, (NC, NV))
    out = {"p": p, "coils": coils}
    for name, traj in (("cartesian", cart), ("spiral", spir)):
        R = traj["nr"]
        out[name] = {"traj": traj, "echo": workloads.cn(rng, (R, NV)) * 0.1,
                     "dT1": workloads.cn(rng, (R, NV)) * 0.05, "dT2": workloads.cn(rng, (R, NV)) * 0.5,
                     "r": workloads.cn(rng, (NC, R, traj["ns"]))}
    out["v"] = workloads.cn(rng, (4, NV))
    out["entries"] = {name: np.stack([rng.integers(0, NC, 256), rng.integers(0, out[name]["traj"]["nr"], 256),
                                      rng.integers(0, out[name]["traj"]["ns"], 256)], 1)
                      for name in ("cartesian", "spiral")}
    out["vidx"] = np.sort(rng.choice(NV, 256, replace=False))
    return out


@pytest.fixture(scope="module")
def workloads():
    import workloads as w

    return w


def _run(cb, ctx, case, kind):
    geo = "cartesian" if kind.startswith("cartesian") else "spiral"
    c = case[geo]
    params = cb.TissueParameters.from_soa(ctx, case["p"])
    traj = cb.trajectory_from_dict(ctx, c["traj"])
    d = {"T1": c["dT1"], "T2": c["dT2"]}
    if kind.endswith("signal"):
        return cb.magnetization_to_signal(ctx, c["echo"], params, traj, case["coils"], method="MatmulFast").to_numpy()
    if kind.endswith("jacobian"):
        return cb.compute_jacobian(ctx, c["echo"], d, params, traj, case["coils"], case["v"],
                                   method="GemmFast").to_numpy()
    return cb.compute_jacobian_hermitian(ctx, c["echo"], d, params, traj, case["coils"], c["r"],
                                         method="GemmFast").to_numpy()


def _oracle(oracle, case, kind):
    geo = "cartesian" if kind.startswith("cartesian") else "spiral"
    c = case[geo]
    args = (c["echo"], c["dT1"], c["dT2"], case["p"], c["traj"], case["coils"])
    ent = case["entries"][geo]
    if kind == "cartesian_signal":
        return oracle.signal_cartesian(c["echo"], case["p"], c["traj"], case["coils"], entries=ent)
    if kind == "spiral_signal":
        return oracle.signal_spiral(c["echo"], case["p"], c["traj"], case["coils"], entries=ent)
    if kind == "cartesian_jacobian":
        return oracle.jacobian(*args, case["v"], entries=ent)
    if kind == "spiral_jacobian":
        return oracle.spiral_jacobian(*args, case["v"], entries=ent)
    if kind == "cartesian_hermitian":
        return oracle.jacobian_hermitian(*args, c["r"], vidx=case["vidx"])
    return oracle.spiral_jacobian_hermitian(*args, c["r"], vidx=case["vidx"])


def _pick(case, kind, got):
    if kind.endswith("hermitian"):
        return got[:, case["vidx"]]
    ent = case["entries"]["cartesian" if kind.startswith("cartesian") else "spiral"]
    return got[ent[:, 0], ent[:, 1], ent[:, 2]]


# (kind, [(tile, splits), ...]): one split or the accuracy minimum, in between, and near the cap of 64
# (57 and 63 are the counts that 64 requested splits round to at 9000 voxels: whole voxel stages of
# 32 (signal) or 16 (J·v) voxels per split, every split non-empty)
LAUNCHES = [
    ("cartesian_signal", [(48, 1), (96, 7), (160, 57), (240, 2)]),
    ("cartesian_jacobian", [(48, 1), (160, 11), (240, 63), (96, 3)]),
    ("cartesian_hermitian", [(0, 1), (0, 5), (0, 23)]),  # 3 coils x 480 readouts = 23 tiles of 64 pairs
    ("spiral_signal", [(0, 3), (0, 10), (0, 57)]),
    ("spiral_jacobian", [(0, 5), (0, 13), (0, 63)]),
    ("spiral_hermitian", [(0, 1), (0, 9), (0, 70)]),  # one split per readout at 70
]


@pytest.mark.parametrize("kind,launches", LAUNCHES, ids=[k for k, _ in LAUNCHES])
def test_every_tuned_launch_keeps_parity(cb, ctx, oracle, case, kind, launches):
    geo = "cartesian" if kind.startswith("cartesian") else "spiral"
    t = case[geo]["traj"]
    ref = _oracle(oracle, case, kind)
    cb.set_tc_launch(kind, 0, 0)
    base = _pick(case, kind, _run(cb, ctx, case, kind))
    assert oracle.rel_l2(base, ref) < TOL_BF16X3
    try:
        for tile, splits in launches:
            cb.set_tc_launch(kind, tile, splits)
            assert cb.tc_launch_choice(kind, NV, t["nr"], t["ns"], NC) == (tile, splits)
            got = _pick(case, kind, _run(cb, ctx, case, kind))
            err = oracle.rel_l2(got, ref)
            assert err < TOL_BF16X3, (tile, splits, err)
    finally:
        cb.set_tc_launch(kind, 0, 0)
