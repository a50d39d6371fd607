"""CPU checks of the C-ABI library: it builds, loads without a GPU, exports every symbol
that include/compas_b200.h declares (the reference's 26 plus the additions), and fails
cleanly — with an error message, not a crash — when no device is present."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "compas_b200.h"

REFERENCE_SYMBOLS = [
    "compas_version", "compas_make_context", "compas_copy_context_for_device", "compas_destroy_context",
    "compas_destroy_object", "compas_synchronize", "compas_make_array_float", "compas_read_array_float",
    "compas_make_array_complex", "compas_read_array_complex", "compas_destroy_array",
    "compas_make_tissue_parameters", "compas_make_fisp_sequence", "compas_make_pssfp_sequence",
    "compas_make_cartesian_trajectory", "compas_make_spiral_trajectory", "compas_simulate_magnetization_fisp",
    "compas_simulate_magnetization_pssfp", "compas_magnetization_to_signal_cartesian",
    "compas_magnetization_to_signal_spiral", "compas_compute_jacobian", "compas_compute_jacobian_hermitian",
    "phase_encoding", "compas_compute_residual", "compas_simulate_magnetization_derivative_pssfp",
    "compas_simulate_magnetization_derivative_fisp",
]


def declared_symbols():
    text = HEADER.read_text()
    return re.findall(r"^COMPAS_API [^(]*?\b(\w+)\(", text, flags=re.M)


@pytest.fixture(scope="module")
def cb():
    import compas_b200

    compas_b200.library()
    return compas_b200


def test_header_declares_reference_abi():
    decl = declared_symbols()
    assert len(REFERENCE_SYMBOLS) == 26
    for s in REFERENCE_SYMBOLS:
        assert s in decl, s


def test_library_exports_every_declared_symbol(cb):
    lib = cb.library()
    for s in declared_symbols():
        assert hasattr(lib, s), f"{s} not exported"
    # the Python front-end binds exactly declared symbols
    assert set(cb.exported_symbols()) <= set(declared_symbols())


def test_version_and_layout_tables(cb):
    assert cb.version().startswith("compas-b200")
    fisp = cb.fisp_configs()
    assert fisp and all(k * g >= 1 for k, g in fisp)
    assert any(k * g >= 128 for k, g in fisp)  # max_state up to 128 is covered (src/simulate/fisp.cu:93-102)
    assert any(k * g >= 35 for k, g in cb.pssfp_configs())


def test_no_device_fails_cleanly(cb):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(cb.CompasError):
        cb.Context(0)
    # the thread-local error slot is set and the library stays usable
    assert cb.library().compas_last_error() is not None
    assert cb.version()


def test_null_handles_are_rejected(cb):
    lib = cb.library()
    assert lib.compas_simulate_magnetization_fisp(None, None, None) is None
    assert b"null" in lib.compas_last_error()
    assert lib.compas_make_fisp_sequence(None, None, 0.0, 0.0, 0.0, 4, 0.0, 1, 1) is None
    assert lib.compas_last_error() is not None


def test_null_handles_are_rejected_by_the_tangent_entry_points(cb):
    import ctypes as C

    lib = cb.library()
    outs = [C.c_void_p(), C.c_void_p(), C.c_void_p()]
    rc = lib.compas_b200_simulate_magnetization_tangents(None, None, None, C.byref(outs[0]), C.byref(outs[1]),
                                                        C.byref(outs[2]))
    assert rc == -1 and lib.compas_last_error() is not None
    assert not any(o.value for o in outs)
    assert lib.compas_b200_simulate_magnetization_tangents(None, None, None, None, None, None) == -1
    assert b"null" in lib.compas_last_error()
    assert lib.compas_b200_batch_derivative(None, 0, 0) is None
    assert b"null" in lib.compas_last_error()
    assert lib.compas_b200_make_batch_tangents(None, 0, None, None, None, None, 4, None) is None
    assert lib.compas_last_error() is not None


def test_voxel_shard_partition_through_the_c_abi():
    # the library's partition of a slice over ranks (host code: runs without a GPU)
    import ctypes as C

    import compas_b200 as cb

    lib = cb.library()
    b, e = C.c_int64(), C.c_int64()
    for nv in (0, 1, 5, 49, 50176, 200003):
        for world in (1, 2, 3, 7, 8):
            prev = 0
            for rank in range(world):
                assert lib.compas_b200_voxel_shard(nv, rank, world, C.byref(b), C.byref(e)) == 0
                assert b.value == prev and e.value >= b.value
                assert e.value - b.value in (nv // world, nv // world + 1)
                prev = e.value
            assert prev == nv
    for bad in ((10, 2, 2), (10, -1, 2), (10, 0, 0), (-1, 0, 1)):
        assert lib.compas_b200_voxel_shard(*bad, C.byref(b), C.byref(e)) == -1
        assert lib.compas_last_error()


def test_vector_value_type_on_the_host(tmp_path):
    # compas/vector.h (vector<T, N>, vfloat3, …) compiled by the host compiler: construction,
    # element names, layout, dot / norm / cross, elementwise arithmetic, map, comparisons
    import shutil
    import subprocess

    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "v.cpp"
    src.write_text(r"""
#include "compas/vector.h"
#include <cmath>
#include <cstdio>
using namespace compas;
int main() {
    vfloat3 a(1.f, 2.f, 2.f), b(0.f, 1.f, 0.f);
    vfloat3 c = cross(a, b);
    vdouble4 d(2.0);
    d += vdouble4(1.0, 2.0, 3.0, 4.0);
    d = 0.5 * (d * 2.0) - 1.0;
    ndint<5> n(7);
    auto m = a.map([](float x) { return int(x * 10); });
    vfloat2 big(3e30f, 4e30f);
    int ok = norm(a) == 3.f && dot(a, b) == 2.f && c.x == -2.f && c.y == 0.f && c.z == 1.f
        && sizeof(vfloat3) == 12 && alignof(vfloat2) == 8 && sizeof(vfloat4) == 16 && alignof(vfloat4) == 16
        && d[0] == 2.0 && d.w == 5.0 && n.size() == 5 && n[4] == 7 && m[1] == 20
        && a == vfloat3(1.f, 2.f, 2.f) && a != b && !(vfloat2(1.f) == vfloat3(1.f))
        && std::fabs(norm(big) - 5e30f) < 1e24f && std::isnan(norm(vfloat2(NAN, 1.f)));
    std::printf("%d\n", ok);
    return ok ? 0 : 1;
}
""")
    exe = tmp_path / "v"
    subprocess.run([cxx, "-std=c++17", "-I", str(ROOT / "compas-toolkit_b200" / "include"), str(src), "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)], capture_output=True, text=True).stdout.strip() == "1"
