"""Continuous-batching serving engine (compas_b200_make_server / _submit / _wait).

A request is simulate -> signal -> residual against measured data and the gradient Jᴴ·r with
forward-difference derivatives (Cartesian or spiral). The tests submit a mix of
FISP/pSSFP, Cartesian/spiral requests of different sizes from several threads while batches are
running, and check that every result (objective, residual, gradient) is bit-identical to the
same request computed alone through the one-request operations; that requests larger than the
memory budget fail cleanly while a small budget still serves everything (one batch at a time);
and that a repeated echo_key reuses resident echoes with unchanged results.
"""
import threading
import time

import numpy as np
import pytest

import workloads as W

pytestmark = pytest.mark.gpu


def _requests(seed=31, n=10):
    jobs = W.batch_jobs(seed=seed, njobs=n, vmin=200, vmax=2000, ntr_min=20, ntr_max=60, cmax=5, ns_spiral=80,
                        P=5, nz=9, nrf=5)
    rng = np.random.default_rng(seed)
    for j in jobs:
        c, r, s = j["ncoils"], j["traj"]["nr"], j["traj"]["ns"]
        j["data"] = W.cn(rng, (c, r, s)) * 0.05
    return jobs


def _alone(cb, ctx, objs, d):
    """The request through the one-request operations."""
    params, seq, traj, coils = objs
    echos = cb.simulate_magnetization(ctx, params, seq)
    s = cb.magnetization_to_signal(ctx, echos, params, traj, coils, method="MatmulFast")
    obj, diff = cb.compute_residual(ctx, d["data"], s)
    out = {"objective": obj, "residual": diff.to_numpy()}
    dd = cb.simulate_magnetization_derivatives(ctx, echos, params, seq)
    out["gradient"] = cb.compute_jacobian_hermitian(ctx, echos, dd, params, traj, coils, diff,
                                                    method="GemmFast").to_numpy()
    return out


@pytest.fixture(scope="module")
def env():
    import compas_b200 as cb

    ctx = cb.Context(0)
    dicts = _requests()
    objs = [cb.job_from_dict(ctx, d) for d in dicts]
    coils = [cb.CompasArray.from_numpy(ctx, d["coils"]) for d in dicts]
    data = [cb.CompasArray.from_numpy(ctx, d["data"]) for d in dicts]
    objs = [(p, s, t, c) for (p, s, t, _), c in zip(objs, coils)]
    alone = [_alone(cb, ctx, o, d) for o, d in zip(objs, dicts)]
    return cb, ctx, dicts, objs, data, alone


def _check_same(cb, eng, ticket, ref, key):
    info = eng.wait(ticket)
    assert info["objective"] == ref["objective"], key
    assert np.array_equal(eng.result(ticket, "residual").to_numpy(), ref["residual"]), key
    assert np.array_equal(eng.result(ticket, "gradient").to_numpy(), ref["gradient"]), key
    return info


def test_mixed_requests_from_threads_match_alone_bitwise(env):
    cb, ctx, dicts, objs, data, alone = env
    eng = cb.ServeEngine(ctx, memory_budget_gb=8.0, max_inflight_batches=3, max_batch_requests=3)
    tickets = [None] * len(dicts)

    def client(idx):
        for i in idx:
            p, s, t, c = objs[i]
            tickets[i] = eng.submit(p, s, t, c, data[i])
            time.sleep(0.002 * (i % 3))

    threads = [threading.Thread(target=client, args=(list(range(k, len(dicts), 3)),)) for k in range(3)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    batches = set()
    for i, d in enumerate(dicts):
        info = _check_same(cb, eng, tickets[i], alone[i], i)
        batches.add(info["batch"])
        assert info["latency_ms"] >= info["device_ms"] >= 0
        eng.release(tickets[i])
    st = eng.stats()
    assert st["completed"] == len(dicts) and st["failed"] == 0
    assert st["batches"] == len(batches) >= 2
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_budget_admission_and_oversized_request(env):
    cb, ctx, dicts, objs, data, alone = env
    # a small budget: fewer requests admitted at once, the peak footprint within it, same results
    eng = cb.ServeEngine(ctx, memory_budget_gb=0.02, max_inflight_batches=4, max_batch_requests=8)
    ts = [eng.submit(*objs[i], data[i]) for i in range(4)]
    for i, t in enumerate(ts):
        _check_same(cb, eng, t, alone[i], i)
        eng.release(t)
    st = eng.stats()
    assert st["peak_bytes"] <= 0.02 * 2 ** 30
    # a request larger than the whole budget fails with a clear error
    tiny = cb.ServeEngine(ctx, memory_budget_gb=1e-4)
    t = tiny.submit(*objs[0], data[0])
    with pytest.raises(cb.CompasError, match="more device memory than the serving budget"):
        tiny.wait(t)


def test_echo_key_reuses_resident_echoes(env):
    cb, ctx, dicts, objs, data, alone = env
    i = next(k for k, d in enumerate(dicts) if d["traj"]["kind"] == "cartesian")
    eng = cb.ServeEngine(ctx, memory_budget_gb=4.0, echo_cache_gb=1.0)
    t1 = eng.submit(*objs[i], data[i], echo_key=77)
    _check_same(cb, eng, t1, alone[i], "first")
    t2 = eng.submit(*objs[i], data[i], echo_key=77)
    _check_same(cb, eng, t2, alone[i], "cached")
    assert eng.stats()["echo_cache_hits"] == 1


def test_exact_derivative_requests_match_alone_bitwise(env):
    # delta = 0: each request's simulation is one tangent pass (the exact ∂/∂T1, ∂/∂T2); the
    # residual and gradient equal the one-request operations with simulate_magnetization_tangents
    cb, ctx, dicts, objs, data, _ = env
    ref = []
    for (params, seq, traj, coils), d in zip(objs, dicts):
        t = cb.simulate_magnetization_tangents(ctx, params, seq)
        s = cb.magnetization_to_signal(ctx, t["echos"], params, traj, coils, method="MatmulFast")
        obj, diff = cb.compute_residual(ctx, d["data"], s)
        g = cb.compute_jacobian_hermitian(ctx, t["echos"], {"T1": t["T1"], "T2": t["T2"]}, params, traj, coils,
                                          diff, method="GemmFast").to_numpy()
        ref.append({"objective": obj, "residual": diff.to_numpy(), "gradient": g})
    eng = cb.ServeEngine(ctx, memory_budget_gb=8.0, max_inflight_batches=2, max_batch_requests=4, delta=0.0)
    tickets = [eng.submit(*objs[i], data[i]) for i in range(len(dicts))]
    for i, t in enumerate(tickets):
        _check_same(cb, eng, t, ref[i], i)
        eng.release(t)
    assert eng.stats()["failed"] == 0
