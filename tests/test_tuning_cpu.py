"""Launch-layout selection: built-in choice, autotuner table (COMPAS_B200_TUNING) and overrides.

The choice is host logic only, so it runs without a GPU. Each case runs in a fresh interpreter
because the library reads the tuning table once per process.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "compas-toolkit_b200"

PROBE = """
import json, sys
sys.path.insert(0, {pkg!r})
import compas_b200 as cb
out = {{"fisp": [cb.fisp_launch_choice(*s) for s in [(25, 50176, 35), (25, 4096, 1), (8, 4096, 1)]],
       "pssfp": [cb.pssfp_launch_choice(*s) for s in [(35, 16384), (5, 4096)]],
       "fisp_configs": cb.fisp_configs(), "pssfp_configs": cb.pssfp_configs(),
       "fisp_packed": [cb.fisp_config_packed(i) for i in range(len(cb.fisp_configs()))],
       "pssfp_packed": [cb.pssfp_config_packed(i) for i in range(len(cb.pssfp_configs()))]}}
cb.set_fisp_launch(0, 2)
out["override_uncovered"] = cb.fisp_launch_choice(25, 50176, 35)
ok = [i for i, (k, g) in enumerate(cb.fisp_configs()) if k * g >= 25][-1]
cb.set_fisp_launch(ok, 3)
out["override"] = cb.fisp_launch_choice(25, 50176, 35)
print(json.dumps(out))
"""


def _probe(env_extra=None):
    env = dict(os.environ)
    env.pop("COMPAS_B200_TUNING", None)
    env.update(env_extra or {})
    r = subprocess.run([sys.executable, "-c", PROBE.format(pkg=str(PKG))], capture_output=True, text=True, env=env,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_builtin_choice_covers_the_states():
    out = _probe()
    fc, pc = out["fisp_configs"], out["pssfp_configs"]
    for (cfg, warps), n in zip(out["fisp"], (25, 25, 8)):
        k, g = fc[cfg]
        assert k * g >= n and 1 <= warps <= 8
    # 25 states x 35 positions at 50176 voxels: one lane per voxel in the packed layout (12 pairs of
    # states, two states per two-wide instruction, and one unpaired state), 8 warps
    assert tuple(fc[out["fisp"][0][0]]) == (25, 1) and out["fisp_packed"][out["fisp"][0][0]]
    assert out["fisp"][0][1] == 8
    assert fc[out["fisp"][2][0]][1] == 4  # few voxel/position pairs: states split over 4 lanes
    for cfg, nz in zip(out["pssfp"], (35, 5)):
        zt, gz = pc[cfg]
        assert zt * gz >= nz
    # 35 z: the two-wide layout of 4 pairs and one unpaired isochromat on 4 lanes (36 slots); 5 z:
    # 1 pair on 4 lanes (8 slots)
    assert tuple(pc[out["pssfp"][0]]) == (9, 4) and out["pssfp_packed"][out["pssfp"][0]]
    assert tuple(pc[out["pssfp"][1]]) == (2, 4) and out["pssfp_packed"][out["pssfp"][1]]
    # an override that does not cover the states is ignored; a covering one wins
    assert out["override_uncovered"] == out["fisp"][0]
    assert out["override"][1] == 3


def test_tuning_table_is_used(tmp_path):
    base = _probe()
    fc, pc = base["fisp_configs"], base["pssfp_configs"]
    fisp_cfg = next(i for i, (k, g) in enumerate(fc) if (k, g) == (7, 4))
    pssfp_cfg = next(i for i, (z, g) in enumerate(pc) if (z, g) == (9, 4))
    table = tmp_path / "tuning.txt"
    table.write_text(f"# comment lines are ignored\nfisp 25 15 5 {fisp_cfg} 6\npssfp 35 14 {pssfp_cfg}\n"
                     f"fisp 25 12 0 0 1\n")  # layout 0 cannot hold 25 states: ignored
    out = _probe({"COMPAS_B200_TUNING": str(table)})
    assert out["fisp"][0] == [fisp_cfg, 6]
    assert out["fisp"][1] == base["fisp"][1]
    assert out["pssfp"][0] == pssfp_cfg
    assert out["pssfp"][1] == base["pssfp"][1]


TC_PROBE = """
import json, sys
sys.path.insert(0, {pkg!r})
import compas_b200 as cb
shape = (50176, 1120, 224, 4)  # voxels, readouts, samples per readout, coils
out = {{k: cb.tc_launch_choice(k, *shape) for k in cb.TC_KINDS}}
out["ragged"] = cb.tc_launch_choice("cartesian_signal", 50176, 1000, 224, 4)
cb.set_tc_launch("cartesian_signal", 112, 1)
out["override_min_splits"] = cb.tc_launch_choice("cartesian_signal", *shape)
cb.set_tc_launch("cartesian_hermitian", 0, 1000)
out["override_hermitian"] = cb.tc_launch_choice("cartesian_hermitian", *shape)
cb.set_tc_launch("spiral_jacobian", 0, 7)
out["override_spiral"] = cb.tc_launch_choice("spiral_jacobian", 50176, 760, 1000, 8)
errors = []
for bad in [("cartesian_signal", 17, 0), ("cartesian_signal", 272, 0), ("cartesian_signal", 0, -1), (6, 0, 0)]:
    try:
        cb.set_tc_launch(*bad)
    except cb.CompasError as e:
        errors.append(str(e))
out["errors"] = errors
print(json.dumps(out))
"""


def _tc_probe(env_extra=None):
    env = dict(os.environ)
    env.pop("COMPAS_B200_TUNING", None)
    env.update(env_extra or {})
    r = subprocess.run([sys.executable, "-c", TC_PROBE.format(pkg=str(PKG))], capture_output=True, text=True,
                       env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_tensor_core_builtin_choice_and_overrides():
    out = _tc_probe()
    # Cartesian: the fewest readout tiles of at most 256, then the least padding (5 tiles of 224
    # for 1120); voxel splits only to fill the GPU (the kernel bounds its accumulation length
    # itself), at most 64
    tile, splits = out["cartesian_signal"]
    assert tile == 224 and 1 <= splits <= 64
    tile, splits = out["cartesian_jacobian"]
    assert tile == 224 and 1 <= splits <= 64
    # 1000 readouts: 4 tiles of 256 (1024 rows), not the 7 tiles of 144 (1008 rows) that pad least
    assert out["ragged"][0] == 256
    assert out["cartesian_hermitian"][0] == 0 and out["cartesian_hermitian"][1] >= 1
    assert out["spiral_signal"][1] >= 13 and out["spiral_jacobian"][1] >= 25
    # a Cartesian override of one split is taken as it is; the spiral J·v kernel raises a split
    # count below its accuracy bound (ceil(V / 2048)) to it; Jᴴ·v splits are capped at one split
    # per 64-pair tile (4 coils x 1120 readouts = 70 tiles)
    assert out["override_min_splits"] == [112, 1]
    assert out["override_hermitian"] == [0, 70]
    assert out["override_spiral"] == [0, 25]
    assert len(out["errors"]) == 4


def test_tensor_core_tuning_table_is_used(tmp_path):
    base = _tc_probe()
    table = tmp_path / "tuning.txt"
    # kind 0 (Cartesian signal), log2 1120 = 10, log2 50176 = 15, log2 (4 x 224) = 9
    table.write_text("tc 0 10 15 9 160 20\n"
                     "tc 1 10 15 9 240 30\n"    # 240 pads 1120 readouts to 1200 > 17/16 x 1120: built-in tile
                     "tc 2 10 15 9 0 5\n"
                     "tc 0 10 15 9 17 4\n"      # invalid tile: the line is ignored (the first stays)
                     "tc 9 10 15 9 0 4\n")      # unknown kind: ignored
    out = _tc_probe({"COMPAS_B200_TUNING": str(table)})
    assert out["cartesian_signal"] == [160, 20]
    assert out["cartesian_jacobian"] == [224, 30]
    assert out["cartesian_hermitian"] == [0, 5]
    assert out["spiral_signal"] == base["spiral_signal"]
    assert out["ragged"] == base["ragged"]  # 1000 readouts: log2 class 9, no line
