"""J·v and Jᴴ·v on spiral trajectories (an addition: the reference's Jacobians accept Cartesian
trajectories only). The GPU kernels are checked against the oracle's derivation from the spiral
signal model (itself pinned by adjointness and finite differences in test_oracle.py) within the FP32
tolerance (FP32 kernels) or the split-BF16 tolerance (tensor-core J·v and Jᴴ·v), through the C-ABI entry
points, which dispatch on the trajectory type; plus adjointness on the GPU. Sizes cross the kernels' tile boundaries: samples
past one 1024-sample block and 64-sample chunks, coil counts 1, 3, 5 and 9 (coil groups of 1, 4, 8
and 8+1), enough readouts for the Jᴴ·v readout splits."""
import numpy as np
import pytest

import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5
TOL_BF16X3 = 1e-4


def _case(seed, nv, nr, ns, nc):
    rng = np.random.default_rng(seed)
    p = W.tissue_voxels(rng, nv, 22.4)
    traj = W.spiral(rng, nr, ns, 22.4, 4e-6)
    coils = W.gaussian_coils(nc, p, 22.4) if nc > 1 else np.ones((1, nv), np.complex64)
    echo = W.cn(rng, (nr, nv)) * 0.1
    d1 = W.cn(rng, (nr, nv)) * 0.05
    d2 = W.cn(rng, (nr, nv)) * 0.5
    v = W.cn(rng, (4, nv))
    u = W.cn(rng, (nc, nr, ns))
    return p, traj, coils, echo, d1, d2, v, u


@pytest.fixture(scope="module")
def ctx():
    import compas_b200 as cb

    return cb.Context(0)


@pytest.mark.parametrize("method", ["Direct", "GemmFast"])
@pytest.mark.parametrize("nc,ns", [(1, 1100), (3, 150), (5, 70), (9, 130), (18, 40)])
def test_spiral_jacobian_matches_oracle(ctx, oracle, nc, ns, method):
    # Direct: FP32 SIMT kernel; GemmFast: split-BF16 tensor-core kernel (the C-ABI entry point's choice)
    import compas_b200 as cb

    p, traj_d, coils, echo, d1, d2, v, u = _case(40 + nc, 150, 9, ns, nc)
    params = cb.TissueParameters.from_soa(ctx, p)
    traj = cb.SpiralTrajectory.from_dict(ctx, traj_d)
    d = {"T1": d1, "T2": d2}
    got = cb.compute_jacobian(ctx, echo, d, params, traj, coils, v, method=method).to_numpy()
    ref = oracle.spiral_jacobian(echo, d1, d2, p, traj_d, coils, v)
    assert oracle.rel_l2(got, ref) < (TOL_FP32 if method == "Direct" else TOL_BF16X3)
    if method == "GemmFast":
        via_abi = cb.compute_jacobian(ctx, echo, d, params, traj, coils, v).to_numpy()
        assert np.array_equal(via_abi, got)


@pytest.mark.parametrize("method", ["Direct", "GemmFast"])
@pytest.mark.parametrize("nc,nr,ns", [(1, 33, 100), (3, 12, 130), (9, 40, 70), (2, 5, 1100)])
def test_spiral_jacobian_hermitian_matches_oracle(ctx, oracle, nc, nr, ns, method):
    # Direct: FP32 kernel; GemmFast: split-BF16 tensor-core kernel (readouts of at most 1024 samples,
    # coil groups of at most 8: 9 coils = 5 + 4; 1100 samples take the FP32 kernel)
    import compas_b200 as cb

    p, traj_d, coils, echo, d1, d2, v, u = _case(60 + nc, 290, nr, ns, nc)
    params = cb.TissueParameters.from_soa(ctx, p)
    traj = cb.SpiralTrajectory.from_dict(ctx, traj_d)
    d = {"T1": d1, "T2": d2}
    got = cb.compute_jacobian_hermitian(ctx, echo, d, params, traj, coils, u, method=method).to_numpy()
    ref = oracle.spiral_jacobian_hermitian(echo, d1, d2, p, traj_d, coils, u)
    assert oracle.rel_l2(got, ref) < (TOL_FP32 if method == "Direct" else TOL_BF16X3)
    if method == "GemmFast":
        # the reference's entry point (low_precision = 0) takes the same split-BF16 kernel
        via_abi = cb.compute_jacobian_hermitian(ctx, echo, d, params, traj, coils, u).to_numpy()
        assert np.array_equal(via_abi, got)


def test_spiral_jacobian_hermitian_readout_chunks_bitwise(ctx, oracle, monkeypatch):
    # the tensor-core Jᴴ·v runs the readouts in chunks bounded by its per-voxel table; one readout
    # per chunk changes only the order in which readouts are summed (FP32 rounding)
    import compas_b200 as cb

    p, traj_d, coils, echo, d1, d2, v, u = _case(71, 300, 7, 200, 3)
    params = cb.TissueParameters.from_soa(ctx, p)
    traj = cb.SpiralTrajectory.from_dict(ctx, traj_d)
    d = {"T1": d1, "T2": d2}
    whole = cb.compute_jacobian_hermitian(ctx, echo, d, params, traj, coils, u, method="GemmFast").to_numpy()
    monkeypatch.setenv("COMPAS_B200_SPIRAL_TABLE_BYTES", "1")
    chunked = cb.compute_jacobian_hermitian(ctx, echo, d, params, traj, coils, u, method="GemmFast").to_numpy()
    assert oracle.rel_l2(chunked, whole) < 1e-6
    ref = oracle.spiral_jacobian_hermitian(echo, d1, d2, p, traj_d, coils, u)
    assert oracle.rel_l2(chunked, ref) < TOL_BF16X3


def test_spiral_adjointness_on_gpu(ctx):
    import compas_b200 as cb

    p, traj_d, coils, echo, d1, d2, v, u = _case(77, 400, 16, 200, 4)
    params = cb.TissueParameters.from_soa(ctx, p)
    traj = cb.SpiralTrajectory.from_dict(ctx, traj_d)
    d = {"T1": d1, "T2": d2}
    for method, tol in (("Direct", 1e-5), ("GemmFast", 1e-4)):
        Jv = cb.compute_jacobian(ctx, echo, d, params, traj, coils, v, method=method).to_numpy().astype(np.complex128)
        JHu = cb.compute_jacobian_hermitian(ctx, echo, d, params, traj, coils, u, method=method)
        JHu = JHu.to_numpy().astype(np.complex128)
        lhs = np.vdot(u.astype(np.complex128), Jv)
        rhs = np.vdot(JHu, v.astype(np.complex128))
        assert abs(lhs - rhs) / abs(lhs) < tol
