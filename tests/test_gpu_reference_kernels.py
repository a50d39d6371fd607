"""The reference's own kernels built for the B200 ("reference kernels, re-hosted":
oracle/_ref/libref_gpu.so from its unmodified src/simulate, src/trajectories, src/jacobian and
src/utils kernel headers with its CUDA flags and launch shapes, and its cuBLAS calls for the default
MatmulFast / GemmFast products; see oracle/ref_gpu*.cu). These tests check that the re-hosted build
agrees with the FP64 oracle, the reference's kernels run on the CPU (golden fixtures) and this
library, so that its timing in bench.py is a fair baseline. The reference builds with
--use_fast_math (__expf, __sincosf, rhypotf), so its echoes are within 1e-4 of FP64, not 1e-5; its
default products run in TF32 (10-bit mantissa), within 2e-3.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(oracle):
    if oracle.ref_gpu() is None:
        pytest.skip("oracle/_ref/libref_gpu.so not built (no reference tree at build time)")
    return oracle


def test_reference_fisp_on_gpu(ref, ref_simulations, workloads):
    import compas_b200 as cb
    import torch

    ctx = cb.Context(0)
    cases = [(p, s) for p, s, _ in ref_simulations["fisp"] if s["inversion"] and s["wait_spoil"]]
    for n in (5, 25, 40):
        w = workloads.tiny(n_side=7, ntr=41, P=3, max_state=n, seed=n)
        cases.append((w["params"], w["seq"]))
    for i, (p, seq) in enumerate(cases):
        got = ref.ref_gpu_fisp(p, seq)
        torch.cuda.synchronize()
        assert ref.ref_gpu_out_of_bounds() == 0
        got = got.cpu().numpy()
        assert ref.rel_l2(got, ref.fisp(p, seq)) < 1e-4, i
        mine = cb.simulate_magnetization(ctx, cb.TissueParameters.from_soa(ctx, p),
                                         cb.FispSequence.from_dict(ctx, seq)).to_numpy()
        assert ref.rel_l2(mine, got) < 1e-4, i


def test_reference_pssfp_on_gpu(ref, ref_simulations, workloads):
    import compas_b200 as cb
    import torch

    ctx = cb.Context(0)
    rng = np.random.default_rng(31)
    cases = [(p, s) for p, s, _ in ref_simulations["pssfp"]]
    cases.append((workloads.tissue(rng, 6, 20.0), workloads.pssfp_sequence(rng, 23, nrf=15, nz=35)))
    for i, (p, seq) in enumerate(cases):
        got = ref.ref_gpu_pssfp(p, seq)
        torch.cuda.synchronize()
        assert ref.ref_gpu_out_of_bounds() == 0
        got = got.cpu().numpy()
        assert ref.rel_l2(got, ref.pssfp(p, seq)) < 1e-4, i
        mine = cb.simulate_magnetization(ctx, cb.TissueParameters.from_soa(ctx, p),
                                         cb.pSSFPSequence.from_dict(ctx, seq)).to_numpy()
        assert ref.rel_l2(mine, got) < 1e-4, i


def test_reference_products_on_gpu(ref, ref_simulations, workloads):
    # the C ABI's default product paths of the reference (MatmulFast, GemmFast: TF32 cuBLAS)
    import compas_b200 as cb

    ctx = cb.Context(0)
    c = ref_simulations["cartesian"]
    rng = np.random.default_rng(5)
    w = workloads.tiny(n_side=9, ntr=37, ns=29, nc=3, seed=5)
    big = {"params": w["params"], "traj": w["traj"], "coils": w["coils"], "echos": workloads.cn(rng, (37, 81)),
           "dT1": workloads.cn(rng, (37, 81)), "dT2": workloads.cn(rng, (37, 81)), "v": workloads.cn(rng, (4, 81)),
           "u": workloads.cn(rng, (3, 37, 29))}
    for case in (c, big):
        p, t = case["params"], case["traj"]
        sig = ref.ref_gpu_signal_cartesian(p, case["echos"], t, case["coils"]).cpu().numpy()
        jv = ref.ref_gpu_jacobian(p, case["echos"], case["dT1"], case["dT2"], t, case["coils"], case["v"]).cpu().numpy()
        jhv = ref.ref_gpu_jacobian(p, case["echos"], case["dT1"], case["dT2"], t, case["coils"], case["u"],
                                   hermitian=True).cpu().numpy()
        assert ref.ref_gpu_out_of_bounds() == 0
        assert ref.rel_l2(sig, ref.signal_cartesian(case["echos"], p, t, case["coils"])) < 2e-3
        assert ref.rel_l2(jv, ref.jacobian(case["echos"], case["dT1"], case["dT2"], p, t, case["coils"],
                                           case["v"])) < 2e-3
        assert ref.rel_l2(jhv, ref.jacobian_hermitian(case["echos"], case["dT1"], case["dT2"], p, t, case["coils"],
                                                      case["u"])) < 2e-3
        params = cb.TissueParameters.from_soa(ctx, p)
        traj = cb.trajectory_from_dict(ctx, t)
        mine = cb.magnetization_to_signal(ctx, case["echos"], params, traj, case["coils"], method="MatmulFast")
        assert ref.rel_l2(mine.to_numpy(), sig) < 2e-3


def test_reference_spiral_signal_on_gpu(ref, ref_simulations, workloads):
    import compas_b200 as cb

    ctx = cb.Context(0)
    rng = np.random.default_rng(8)
    s = ref_simulations["spiral"]
    p = workloads.tissue(rng, 9, 22.4)
    big = {"params": p, "traj": workloads.spiral(rng, 13, 300, 22.4, 4e-6), "coils": workloads.cn(rng, (3, 81)),
           "echos": workloads.cn(rng, (13, 81))}
    for case in (s, big):
        got = ref.ref_gpu_signal_spiral(case["params"], case["echos"], case["traj"], case["coils"]).cpu().numpy()
        assert ref.ref_gpu_out_of_bounds() == 0
        want = ref.signal_spiral(case["echos"], case["params"], case["traj"], case["coils"])
        assert ref.rel_l2(got, want) < 1e-4
        params = cb.TissueParameters.from_soa(ctx, case["params"])
        mine = cb.magnetization_to_signal(ctx, case["echos"], params, cb.trajectory_from_dict(ctx, case["traj"]),
                                          case["coils"], method="MatmulFast").to_numpy()
        assert ref.rel_l2(mine, got) < 2e-4
