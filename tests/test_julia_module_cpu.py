"""The Julia module shipped with the library (compas-toolkit_b200/julia/CompasToolkit.jl), checked as text.

Julia is not installed here, so the module is checked against the C ABI it binds rather than run:
  * it binds every one of the 26 symbols the reference's CompasToolkit.jl binds, and only symbols
    that include/compas_b200.h declares and libcompas_b200.so exports;
  * every @ccall passes as many arguments as the C declaration has parameters, each with a Julia
    type of the same kind (pointer, 32-bit integer, 64-bit integer, float), and returns the
    declared kind;
  * it defines the reference module's public names, passes the pSSFP slice positions as Float32
    (the type the library reads), and its brackets and blocks balance.
"""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
MODULE = ROOT / "compas-toolkit_b200" / "julia" / "CompasToolkit.jl"
HEADER = ROOT / "include" / "compas_b200.h"
LIB = ROOT / "compas-toolkit_b200" / "libcompas_b200.so"

# the symbols the reference's CompasToolkit.jl binds through @ccall LIBRARY.<name>
REFERENCE_SYMBOLS = {
    "compas_version", "compas_make_context", "compas_copy_context_for_device", "compas_destroy_context",
    "compas_destroy_object", "compas_synchronize", "compas_make_array_float", "compas_make_array_complex",
    "compas_read_array_float", "compas_read_array_complex", "compas_destroy_array",
    "compas_make_tissue_parameters", "compas_make_fisp_sequence", "compas_make_pssfp_sequence",
    "compas_make_cartesian_trajectory", "compas_make_spiral_trajectory", "compas_simulate_magnetization_fisp",
    "compas_simulate_magnetization_pssfp", "compas_simulate_magnetization_derivative_fisp",
    "compas_simulate_magnetization_derivative_pssfp", "compas_magnetization_to_signal_cartesian",
    "compas_magnetization_to_signal_spiral", "compas_compute_jacobian", "compas_compute_jacobian_hermitian",
    "phase_encoding", "compas_compute_residual",
}

# public names of the reference module (types, constructors, functions, the precision switch)
REFERENCE_API = [
    "version", "check_version", "Context", "init_context", "set_context", "get_context", "synchronize",
    "CompasArray", "TissueParameters", "FispSequence", "pSSFPSequence", "Trajectory", "CartesianTrajectory",
    "SpiralTrajectory", "simulate_magnetization", "simulate_magnetization_derivative",
    "simulate_magnetization_derivatives", "magnetization_to_signal", "compute_jacobian",
    "compute_jacobian_hermitian", "phase_encoding", "compute_residual", "LOW_PRECISION_MODE",
]


def _close(text, i, open_ch, close_ch):
    """index of the bracket closing the one at text[i]"""
    depth = 0
    for j in range(i, len(text)):
        if text[j] == open_ch:
            depth += 1
        elif text[j] == close_ch:
            depth -= 1
            if depth == 0:
                return j
    raise AssertionError(f"unbalanced {open_ch} at offset {i}")


def _split_top(s):
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        parts.append(cur)
    return [p.strip() for p in parts if p.strip()]


def _julia_type(expr):
    """the type after the last top-level '::' of `expr`"""
    depth, last = 0, -1
    for i in range(len(expr) - 1):
        ch = expr[i]
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        elif depth == 0 and expr[i:i + 2] == "::":
            last = i
    assert last >= 0, f"no type in {expr!r}"
    return expr[last + 2:].strip()


def _ccalls():
    src = MODULE.read_text()
    out = []
    for m in re.finditer(r"@ccall\s+LIBRARY\.(\w+)\(", src):
        open_at = m.end() - 1
        close_at = _close(src, open_at, "(", ")")
        args = _split_top(src[open_at + 1:close_at])
        rest = src[close_at + 1:]
        assert rest.startswith("::"), f"{m.group(1)}: no return type"
        ret = re.match(r"::(\w+(\{[^}]*\})?)", rest).group(1)
        out.append((m.group(1), [_julia_type(a) for a in args], ret))
    return out


def _declarations():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    decls = {}
    for m in re.finditer(r"COMPAS_API\s+([^;(]*?)\s*\b(\w+)\s*\(([^;]*?)\)\s*;", text, flags=re.S):
        ret, name, params = m.group(1), m.group(2), m.group(3).strip()
        plist = [] if params in ("", "void") else [" ".join(p.split()) for p in params.split(",")]
        decls[name] = (" ".join(ret.split()), plist)
    return decls


def _c_kind(decl):
    if "*" in decl:
        return "ptr"
    words = decl.replace("const", "").split()
    base = " ".join(words[:-1]) if len(words) > 1 else words[0]
    return {"int": "i32", "int32_t": "i32", "int64_t": "i64", "float": "f32", "void": "void"}[base]


def _julia_kind(t):
    if t.startswith("Ptr{") or t == "Cstring":
        return "ptr"
    return {"Int32": "i32", "Cint": "i32", "Int64": "i64", "Float32": "f32", "Cvoid": "void"}[t]


def test_binds_every_reference_symbol_and_only_declared_exported_ones():
    calls = _ccalls()
    names = {n for n, _, _ in calls}
    assert REFERENCE_SYMBOLS <= names, sorted(REFERENCE_SYMBOLS - names)
    decls = _declarations()
    assert names <= set(decls), sorted(names - set(decls))
    lib = ctypes.CDLL(str(LIB))
    for n in names:
        assert hasattr(lib, n), n


def test_every_ccall_matches_its_c_declaration():
    decls = _declarations()
    for name, jtypes, jret in _ccalls():
        cret, cparams = decls[name]
        assert len(jtypes) == len(cparams), (name, jtypes, cparams)
        for jt, cp in zip(jtypes, cparams):
            assert _julia_kind(jt) == _c_kind(cp), (name, jt, cp)
        ret_kind = "ptr" if "*" in cret else _c_kind(cret + " r")
        assert _julia_kind(jret) == ret_kind, (name, jret, cret)


def test_reference_api_names_and_the_pssfp_z_type():
    src = MODULE.read_text()
    for name in REFERENCE_API:
        pattern = rf"(function|struct|const|abstract type)\s+{re.escape(name)}\b|^{re.escape(name)}\(.*\)\s*(::\w+)?\s*="
        assert re.search(pattern, src, flags=re.M), name
    assert re.search(r"device_array\(z, Float32,", src)
    assert not re.search(r"\bz\b[^\n]*ComplexF32", src)


def _strip_strings_and_comments(src):
    src = re.sub(r'"""(.*?)"""', '""', src, flags=re.S)
    src = re.sub(r'"(\\.|[^"\\])*"', '""', src)
    return re.sub(r"#.*", "", src)


def test_brackets_and_blocks_balance():
    code = _strip_strings_and_comments(MODULE.read_text())
    for o, c in ("()", "[]", "{}"):
        assert code.count(o) == code.count(c), (o, code.count(o), code.count(c))
    opens = ends = 0
    for line in code.splitlines():
        s = line.strip()
        if re.match(r"abstract type .* end$", s):
            continue
        if re.match(r"(function|mutable struct|struct|module|if|for|while|let|begin|try)\b", s) or re.search(r"\bdo( \w+)?$", s):
            opens += 1
        if re.match(r"end\b", s):
            ends += 1
    assert opens == ends, (opens, ends)
