"""Regenerate the golden fixtures from the reference's own code.

Builds oracle/_ref/ref_golden and oracle/_ref/ref_sim (oracle/Makefile target `ref`, which
compiles oracle/ref_golden.cpp and oracle/ref_sim.cpp against the reference's include and src
trees: the directory named by COMPAS_REFERENCE, by default /root/reference) and stores their JSON
output next to this script:
  * ref_complex_ops.json  — complex_type.h primitives (FP32);
  * ref_simulations.json  — inputs and outputs of seeded FISP, pSSFP, Cartesian (phase encoding,
                            signal, J·v, Jᴴ·v, residual) and spiral (signal) cases from the
                            reference's kernels run one thread at a time on the CPU.
Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]


def main() -> int:
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    out = subprocess.run([str(ROOT / "oracle" / "_ref" / "ref_golden")], check=True, capture_output=True, text=True)
    data = json.loads(out.stdout)
    data["_source"] = ("compas-toolkit include/compas/core/complex_type.h (exp :106-114, pow :153-161, "
                       "fma :174-178, operator* :220-223), FP32, host build by oracle/Makefile `ref`")
    (Path(__file__).parent / "ref_complex_ops.json").write_text(json.dumps(data, indent=0))
    print("wrote", {k: len(v) for k, v in data.items() if isinstance(v, list)})

    out = subprocess.run([str(ROOT / "oracle" / "_ref" / "ref_sim")], check=True, capture_output=True, text=True)
    sims = json.loads(out.stdout)
    sims["_source"] = ("compas-toolkit src/simulate/fisp_kernels.cuh (simulate_fisp, expand_undersampled_echos), "
                       "src/simulate/pssfp_kernels.cuh (simulate_pssfp) with src/operators/epg.cuh and "
                       "isochromat.cuh; src/trajectories/phase_encoding_kernels.cuh, signal_kernels.cuh "
                       "(sum_signal_cartesian_naive; prepare_readout_echos, prepare_sample_decay_spiral, "
                       "sum_signal_spiral), src/jacobian/product_kernels.cuh (jacobian_product_naive), "
                       "hermitian_kernels.cuh (jacobian_hermitian_product_naive), src/utils/residual_kernels.cuh; "
                       "FP32, one-thread launches on the host (oracle/ref_sim.cpp, ref_sim_hermitian.cpp); "
                       "fast-math intrinsics replaced by libm")
    (Path(__file__).parent / "ref_simulations.json").write_text(json.dumps(sims))
    print("wrote", sorted(k for k in sims if not k.startswith("_")))
    return 0


if __name__ == "__main__":
    sys.exit(main())
