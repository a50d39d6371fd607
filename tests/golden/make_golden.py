"""Regenerate tests/golden/ref_complex_ops.json from the reference's own code.

Builds oracle/_ref/ref_golden (oracle/Makefile target `ref`, which compiles
oracle/ref_golden.cpp against the reference's include tree, by default
/root/reference/include) and stores its JSON output next to this script.
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
    return 0


if __name__ == "__main__":
    sys.exit(main())
