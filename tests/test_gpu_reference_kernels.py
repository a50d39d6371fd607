"""The reference's own FISP and pSSFP kernels built for the B200 ("reference kernels, re-hosted":
oracle/_ref/libref_gpu.so from the unmodified src/simulate/*_kernels.cuh with the reference's CUDA
flags and launch shapes; see oracle/ref_gpu.cu). These tests check that the re-hosted build
reproduces the reference's kernels as run on the CPU (the golden fixtures) and agrees with this
library, so that its timing in bench.py is a fair baseline. The reference builds with
--use_fast_math (__expf, __sincosf, rhypotf), so its echoes are within 1e-4 of FP64, not 1e-5.
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
        assert ref.ref_gpu().ref_gpu_out_of_bounds() == 0
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
        assert ref.ref_gpu().ref_gpu_out_of_bounds() == 0
        got = got.cpu().numpy()
        assert ref.rel_l2(got, ref.pssfp(p, seq)) < 1e-4, i
        mine = cb.simulate_magnetization(ctx, cb.TissueParameters.from_soa(ctx, p),
                                         cb.pSSFPSequence.from_dict(ctx, seq)).to_numpy()
        assert ref.rel_l2(mine, got) < 1e-4, i
