"""Failure detection on the GPU, without a GPU fault.

Kernels never trap: a bounded device-side wait that gives up records STATUS_WAIT_TIMEOUT in the
status word of the context (or serving slot) it was launched through, returns, and the host raises
CompasError at the next synchronisation — the reference traps on the device instead
(include/compas/core/assertion.h:24, COMPAS_CHECK → CompasException at 35-44). Here the wait is made
to run out on a barrier that nothing completes (compas_b200_wait_probe), and bad inputs come in
through the C ABI. Every case checks that the context stays usable afterwards.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb():
    import compas_b200

    compas_b200.library()
    return compas_b200


@pytest.fixture(scope="module")
def ctx(cb):
    return cb.Context(0)


def _still_usable(cb, ctx, oracle, workloads):
    w = workloads.tiny(n_side=5, ntr=17, P=2, max_state=4)
    p = cb.TissueParameters.from_soa(ctx, w["params"])
    got = cb.simulate_magnetization(ctx, p, cb.FispSequence.from_dict(ctx, w["seq"])).to_numpy()
    assert oracle.rel_l2(got, oracle.fisp(w["params"], w["seq"])) < 1e-5


def test_wait_timeout_is_reported_and_cleared(cb, ctx, oracle, workloads):
    cb.wait_probe(ctx, 2_000_000)  # ~1 ms of SM cycles, then the wait gives up
    with pytest.raises(cb.CompasError, match="bounded device-side wait gave up"):
        ctx.synchronize()
    ctx.synchronize()  # the report cleared the status word
    _still_usable(cb, ctx, oracle, workloads)


def test_serving_failure_stays_in_its_batch(cb, ctx, workloads):
    # two slots, one request per batch: the batch of the injected request fails, the batch of the
    # other request (on the other slot, with its own status word) completes with the same result
    # as on an engine that saw no failure
    d = workloads.serve_requests(seed=5, n=2, vmin=2000, vmax=3000, cmin=2, cmax=3)[0]
    p, s, t, _ = cb.job_from_dict(ctx, d)
    coils, data = cb.CompasArray.from_numpy(ctx, d["coils"]), cb.CompasArray.from_numpy(ctx, d["data"])
    clean = cb.ServeEngine(ctx, memory_budget_gb=8.0, max_inflight_batches=2, max_batch_requests=1)
    ref = clean.submit(p, s, t, coils, data)
    ref_obj = clean.wait(ref)["objective"]
    ref_grad = clean.result(ref, "gradient").to_numpy()
    clean.release(ref)
    eng = cb.ServeEngine(ctx, memory_budget_gb=8.0, max_inflight_batches=2, max_batch_requests=1)
    bad = eng.submit(p, s, t, coils, data, inject_wait_timeout=True)
    good = eng.submit(p, s, t, coils, data)
    with pytest.raises(cb.CompasError, match="bounded device-side wait gave up|reported an error"):
        eng.wait(bad)
    res = eng.wait(good)
    assert res["objective"] == ref_obj
    assert np.array_equal(eng.result(good, "gradient").to_numpy(), ref_grad)
    after = eng.submit(p, s, t, coils, data)  # the failed slot serves again
    assert eng.wait(after)["objective"] == ref_obj
    st = eng.stats()
    assert st["failed"] == 1 and st["completed"] == 2
    for k in (bad, good, after):
        eng.release(k)
    ctx.synchronize()  # the slot's error never reached the device-wide word


def test_ncoils_mismatch_is_a_clean_error(cb, ctx, oracle, workloads):
    # the C-ABI products take the coil count and the coil array separately (bindings.cpp)
    w = workloads.tiny(n_side=4, ntr=9, ns=5, nc=2)
    params = cb.TissueParameters.from_soa(ctx, w["params"])
    traj = cb.trajectory_from_dict(ctx, w["traj"])
    e = cb.CompasArray.from_numpy(ctx, workloads.cn(np.random.default_rng(0), (9, 16)))
    c = cb.CompasArray.from_numpy(ctx, w["coils"])
    v = cb.CompasArray.from_numpy(ctx, workloads.cn(np.random.default_rng(1), (4, 16)))
    u = cb.CompasArray.from_numpy(ctx, workloads.cn(np.random.default_rng(2), (2, 9, 5)))
    lib = cb.library()
    calls = [lambda: lib.compas_magnetization_to_signal_cartesian(ctx.ptr, 3, e.ptr, params.ptr, c.ptr, traj.ptr, 0),
             lambda: lib.compas_compute_jacobian(ctx.ptr, 3, e.ptr, e.ptr, e.ptr, params.ptr, c.ptr, traj.ptr, v.ptr, 0),
             lambda: lib.compas_compute_jacobian_hermitian(ctx.ptr, 1, e.ptr, e.ptr, e.ptr, params.ptr, traj.ptr, c.ptr,
                                                           u.ptr, 0)]
    for call in calls:
        assert not call()
        assert "ncoils does not match" in lib.compas_last_error().decode()
    _still_usable(cb, ctx, oracle, workloads)


def test_max_state_above_128_is_a_clean_error(cb, ctx, oracle, workloads):
    w = workloads.tiny()
    for n in (0, 129):
        with pytest.raises(cb.CompasError, match="max_state"):
            cb.FispSequence.from_dict(ctx, dict(w["seq"], max_state=n))
    _still_usable(cb, ctx, oracle, workloads)


@pytest.mark.parametrize("bad", [np.nan, 0.0, -0.05])
def test_bad_T2_stays_in_its_voxel(cb, ctx, workloads, bad):
    # no validation of tissue values, as in the reference (tissue.cpp): a NaN or non-positive T2
    # gives non-finite or meaningless echoes for that voxel only; every other voxel's echoes are
    # the same bits as without it. Signal and products sum over voxels, so they carry the NaN on.
    w = workloads.tiny(n_side=6, ntr=21, P=3, max_state=6)
    seq = cb.FispSequence.from_dict(ctx, w["seq"])
    clean = cb.simulate_magnetization(ctx, cb.TissueParameters.from_soa(ctx, w["params"]), seq).to_numpy()
    p = w["params"].copy()
    p[1, 7] = bad
    got = cb.simulate_magnetization(ctx, cb.TissueParameters.from_soa(ctx, p), seq).to_numpy()
    others = np.arange(36) != 7
    assert np.array_equal(got[:, others], clean[:, others])
    if np.isnan(bad):
        assert np.isnan(got[:, 7]).all()
        sig = cb.magnetization_to_signal(ctx, got, cb.TissueParameters.from_soa(ctx, p), cb.trajectory_from_dict(ctx, w["traj"]),
                                         w["coils"], method="Direct").to_numpy()
        assert np.isnan(sig).all()
