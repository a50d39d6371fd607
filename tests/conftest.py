import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "compas-toolkit_b200"
for p in (str(PKG), str(ROOT / "oracle"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    # gpu tests are selected with -m gpu; without a device they are skipped, not failed
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    import oracle as o

    o.lib()
    return o


@pytest.fixture(scope="session")
def workloads():
    import workloads as w

    return w


@pytest.fixture(scope="session")
def ref_simulations():
    """Seeded cases computed by the reference's own kernels on the CPU
    (tests/golden/ref_simulations.json, made by tests/golden/make_golden.py). "fisp" / "pssfp":
    lists of (params float32 [9][nv], sequence dict in the oracle's / workloads' format, echoes
    complex128 [nreadouts][nv]); "cartesian" / "spiral": one dict each with the inputs (complex64,
    the library's layouts) and the reference's outputs (complex128)."""
    import json

    import numpy as np

    data = json.loads((ROOT / "tests" / "golden" / "ref_simulations.json").read_text())

    def cx(a):
        a = np.asarray(a, np.float64)
        return a[0::2] + 1j * a[1::2]

    out = {"fisp": [], "pssfp": [], "cartesian": None, "spiral": None}
    for c in data["fisp"]:
        nv, ntr, P = c["nv"], c["nTR"], c["P"]
        seq = {"rf": cx(c["rf"]).astype(np.complex64),
               "slices": cx(c["slices"]).reshape(P, ntr).astype(np.complex64),
               "TR": c["TR"], "TE": c["TE"], "TI": c["TI"], "TW": c["TW"], "max_state": c["max_state"],
               "uf": c["uf"], "reps": c["reps"], "inversion": c["inversion"], "wait_spoil": c["wait_spoil"]}
        out["fisp"].append((np.array(c["params"], np.float32).reshape(9, nv), seq,
                            cx(c["echos"]).reshape(ntr * c["uf"], nv)))
    for c in data["pssfp"]:
        nv, ntr = c["nv"], c["nTR"]
        seq = {"rf": cx(c["rf"]).astype(np.complex64), "TR": c["TR"],
               "gdtrf": cx(c["gamma_dt_RF"]).astype(np.complex64), "dt": tuple(c["dt"]),
               "gz": tuple(c["gamma_dt_GRz"]), "z": np.array(c["z"], np.float32)}
        out["pssfp"].append((np.array(c["params"], np.float32).reshape(9, nv), seq,
                             cx(c["echos"]).reshape(ntr, nv)))
    # Cartesian and spiral operator cases: inputs in the library's / oracle's layouts, complex64
    c = data["cartesian"]
    nv, R, S, C = c["nv"], c["R"], c["S"], c["C"]
    f32 = lambda key, *shape: cx(c[key]).reshape(shape).astype(np.complex64)  # noqa: E731
    out["cartesian"] = {
        "params": np.array(c["params"], np.float32).reshape(9, nv),
        "traj": {"kind": "cartesian", "nr": R, "ns": S, "dt": c["dt"], "k_start": f32("k_start", R),
                 "dk": c["dk"]},
        "echos": f32("echos", R, nv), "dT1": f32("dT1", R, nv), "dT2": f32("dT2", R, nv),
        "coils": f32("coils", C, nv), "v": f32("v", 4, nv), "u": f32("u", C, R, S), "rhs": f32("rhs", C, R, S),
        "phase_encoded": cx(c["phase_encoded"]).reshape(R, nv), "signal": cx(c["signal"]).reshape(C, R, S),
        "jv": cx(c["jv"]).reshape(C, R, S), "jhv": cx(c["jhv"]).reshape(4, nv),
        "residual": cx(c["residual"]).reshape(C, R, S), "objective": float(c["objective"])}
    c = data["spiral"]
    nv, R, S, C = c["nv"], c["R"], c["S"], c["C"]
    out["spiral"] = {
        "params": np.array(c["params"], np.float32).reshape(9, nv),
        "traj": {"kind": "spiral", "nr": R, "ns": S, "dt": c["dt"], "k_start": f32("k_start", R),
                 "dk": f32("delta_k", R)},
        "echos": f32("echos", R, nv), "coils": f32("coils", C, nv), "signal": cx(c["signal"]).reshape(C, R, S)}
    return out
