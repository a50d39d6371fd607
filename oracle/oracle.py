"""ctypes front-end of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker and the CPU baseline. Imported by
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference
legs of ``bench.py`` — never by the product package.

Arrays follow the reference's C++ row-major layouts (compas-toolkit
``include/compas/*``): tissue parameters float32 ``[9][V]`` (T1, T2, B1, B0,
rho_x, rho_y, x, y, z), echos complex ``[R][V]``, coils ``[C][V]``, signal
``[C][R][S]``, J·v input ``[4][V]``, Jᴴ·v input ``[C][R][S]``, output ``[4][V]``.
``dtype='f64'`` returns the FP64 truth, ``'f32'`` the FP32 reference twin.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None

_P, _I, _I64, _F = C.c_void_p, C.c_int, C.c_int64, C.c_float
_SIGS = {
    "oracle_fisp_f64": [_P, _I64, _P, _I64, _P, _P, _I, _I, _F, _F, _F, _F, _I, _I, _I, _I, _I, _P, _I],
    "oracle_fisp_f32": [_P, _I64, _P, _I64, _P, _P, _I, _I, _F, _F, _F, _F, _I, _I, _I, _I, _I, _P, _I],
    "oracle_pssfp_f64": [_P, _I64, _P, _I64, _P, _I, _P, _I, _F, _F, _F, _F, _F, _F, _P, _I, _P, _I],
    "oracle_pssfp_f32": [_P, _I64, _P, _I64, _P, _I, _P, _I, _F, _F, _F, _F, _F, _F, _P, _I, _P, _I],
    "oracle_phase_encoding_f64": [_P, _P, _I64, _I, _P, _P],
    "oracle_signal_cartesian_f64": [_P, _P, _I64, _I, _I, _F, _P, _F, _F, _P, _I, _P, _I64, _P, _I],
    "oracle_signal_cartesian_f32": [_P, _P, _I64, _I, _I, _F, _P, _F, _F, _P, _I, _P, _I64, _P, _I],
    "oracle_signal_spiral_f64": [_P, _P, _I64, _I, _I, _F, _P, _P, _P, _I, _P, _I64, _P, _I],
    "oracle_jacobian_f64": [_P, _P, _P, _P, _I64, _I, _I, _F, _F, _F, _P, _I, _P, _P, _I64, _P, _I],
    "oracle_jacobian_hermitian_f64": [_P, _P, _P, _P, _I64, _I, _I, _F, _F, _F, _P, _I, _P, _P, _I64, _P, _I],
    "oracle_spiral_jacobian_f64": [_P, _P, _P, _P, _I64, _I, _I, _F, _P, _P, _P, _I, _P, _P, _I64, _P, _I],
    "oracle_spiral_jacobian_hermitian_f64": [_P, _P, _P, _P, _I64, _I, _I, _F, _P, _P, _P, _I, _P, _P, _I64, _P,
                                             _I],
    "oracle_residual_f64": [_P, _P, _I64, _P],
    "oracle_cx_eval_f32": [_I, _P, _I64, _P],
    "oracle_max_threads": [],
}


def lib():
    global _LIB
    if _LIB is None:
        path = _HERE / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: run `make -C oracle` (or __graft_entry__.build())")
        L = C.CDLL(str(path))
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_double if name == "oracle_residual_f64" else C.c_int
        _LIB = L
    return _LIB


def nthreads_default() -> int:
    return int(os.environ.get("COMPAS_ORACLE_THREADS", os.cpu_count() or 1))


def _cf(a) -> np.ndarray:
    """complex array -> contiguous interleaved float32 view."""
    a = np.ascontiguousarray(a, dtype=np.complex64)
    return a.view(np.float32)


def _ff(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _ip(idx):
    if idx is None:
        return None, 0
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    return idx, len(idx)


def _iptr(idx):
    return None if idx is None else idx.ctypes.data


def _out(shape, dtype):
    if dtype == "f64":
        return np.zeros(shape + (2,), np.float64)
    return np.zeros(shape + (2,), np.float32)


def _as_complex(buf):
    return buf[..., 0] + 1j * buf[..., 1] if buf.dtype == np.float64 else (buf[..., 0] + 1j * buf[..., 1]).astype(np.complex64)


def fisp(params, seq, vidx=None, dtype="f64", nthreads=None):
    """simulate_magnetization(FISP): echos [nTR*uf][n]."""
    params = _ff(params)
    nv = params.shape[1]
    idx, nidx = _ip(vidx)
    n = nidx if idx is not None else nv
    rf = _cf(seq["rf"])
    slices = _cf(seq["slices"])
    nTR = len(seq["rf"])
    P = seq["slices"].shape[0]
    R = nTR * int(seq.get("uf", 1))
    out = _out((R, n), dtype)
    fn = lib().oracle_fisp_f64 if dtype == "f64" else lib().oracle_fisp_f32
    rc = fn(params.ctypes.data, C.c_int64(nv), _iptr(idx), C.c_int64(nidx), rf.ctypes.data, slices.ctypes.data,
            nTR, P, C.c_float(seq["TR"]), C.c_float(seq["TE"]), C.c_float(seq.get("TW", 0.0)),
            C.c_float(seq["TI"]), int(seq["max_state"]), int(seq.get("uf", 1)), int(seq.get("reps", 1)),
            int(seq.get("inversion", 1)), int(seq.get("wait_spoil", 1)), out.ctypes.data,
            nthreads or nthreads_default())
    if rc != 0:
        raise ValueError("oracle_fisp rejected its arguments")
    return _as_complex(out)


def pssfp(params, seq, vidx=None, dtype="f64", nthreads=None):
    """simulate_magnetization(pSSFP): echos [nTR][n]."""
    params = _ff(params)
    nv = params.shape[1]
    idx, nidx = _ip(vidx)
    n = nidx if idx is not None else nv
    rf = _cf(seq["rf"])
    g = _cf(seq["gdtrf"])
    z = _ff(seq["z"])
    nTR = len(seq["rf"])
    out = _out((nTR, n), dtype)
    fn = lib().oracle_pssfp_f64 if dtype == "f64" else lib().oracle_pssfp_f32
    dt, gz = seq["dt"], seq["gz"]
    rc = fn(params.ctypes.data, C.c_int64(nv), _iptr(idx), C.c_int64(nidx), rf.ctypes.data, nTR, g.ctypes.data,
            len(seq["gdtrf"]), C.c_float(dt[0]), C.c_float(dt[1]), C.c_float(dt[2]), C.c_float(gz[0]),
            C.c_float(gz[1]), C.c_float(gz[2]), z.ctypes.data, len(z), out.ctypes.data,
            nthreads or nthreads_default())
    if rc != 0:
        raise ValueError("oracle_pssfp rejected its arguments")
    return _as_complex(out)


def phase_encoding(echo, params, k_start):
    e, params, ks = _cf(echo), _ff(params), _cf(k_start)
    R, V = echo.shape
    out = np.zeros((R, V, 2), np.float64)
    lib().oracle_phase_encoding_f64(e.ctypes.data, params.ctypes.data, C.c_int64(V), R, ks.ctypes.data,
                                    out.ctypes.data)
    return _as_complex(out)


def _entries(entries):
    if entries is None:
        return None, 0
    e = np.ascontiguousarray(entries, dtype=np.int32).reshape(-1, 3)
    return e, len(e)


def signal_cartesian(echo, params, traj, coils, entries=None, dtype="f64", nthreads=None):
    e, params, ks, co = _cf(echo), _ff(params), _cf(traj["k_start"]), _cf(coils)
    R, V = echo.shape
    Cn = coils.shape[0]
    ent, nent = _entries(entries)
    shape = (nent,) if ent is not None else (Cn, traj["nr"], traj["ns"])
    out = _out(shape, dtype)
    dk = complex(traj["dk"])
    fn = lib().oracle_signal_cartesian_f64 if dtype == "f64" else lib().oracle_signal_cartesian_f32
    fn(e.ctypes.data, params.ctypes.data, C.c_int64(V), traj["nr"], traj["ns"], C.c_float(traj["dt"]),
       ks.ctypes.data, C.c_float(dk.real), C.c_float(dk.imag), co.ctypes.data, Cn,
       None if ent is None else ent.ctypes.data, C.c_int64(nent), out.ctypes.data, nthreads or nthreads_default())
    return _as_complex(out)


def signal_spiral(echo, params, traj, coils, entries=None, nthreads=None):
    e, params, ks, dk, co = _cf(echo), _ff(params), _cf(traj["k_start"]), _cf(traj["dk"]), _cf(coils)
    R, V = echo.shape
    Cn = coils.shape[0]
    ent, nent = _entries(entries)
    shape = (nent,) if ent is not None else (Cn, traj["nr"], traj["ns"])
    out = _out(shape, "f64")
    lib().oracle_signal_spiral_f64(e.ctypes.data, params.ctypes.data, C.c_int64(V), traj["nr"], traj["ns"],
                                   C.c_float(traj["dt"]), ks.ctypes.data, dk.ctypes.data, co.ctypes.data, Cn,
                                   None if ent is None else ent.ctypes.data, C.c_int64(nent), out.ctypes.data,
                                   nthreads or nthreads_default())
    return _as_complex(out)


def jacobian(echo, dT1, dT2, params, traj, coils, vec, entries=None, nthreads=None):
    e, d1, d2, params, co, ve = _cf(echo), _cf(dT1), _cf(dT2), _ff(params), _cf(coils), _cf(vec)
    R, V = echo.shape
    Cn = coils.shape[0]
    ent, nent = _entries(entries)
    shape = (nent,) if ent is not None else (Cn, traj["nr"], traj["ns"])
    out = _out(shape, "f64")
    dk = complex(traj["dk"])
    lib().oracle_jacobian_f64(e.ctypes.data, d1.ctypes.data, d2.ctypes.data, params.ctypes.data, C.c_int64(V),
                              traj["nr"], traj["ns"], C.c_float(traj["dt"]), C.c_float(dk.real),
                              C.c_float(dk.imag), co.ctypes.data, Cn, ve.ctypes.data,
                              None if ent is None else ent.ctypes.data, C.c_int64(nent), out.ctypes.data,
                              nthreads or nthreads_default())
    return _as_complex(out)


def jacobian_hermitian(echo, dT1, dT2, params, traj, coils, vec, vidx=None, nthreads=None):
    e, d1, d2, params, co, ve = _cf(echo), _cf(dT1), _cf(dT2), _ff(params), _cf(coils), _cf(vec)
    R, V = echo.shape
    Cn = coils.shape[0]
    idx, nidx = _ip(vidx)
    n = nidx if idx is not None else V
    out = _out((4, n), "f64")
    dk = complex(traj["dk"])
    lib().oracle_jacobian_hermitian_f64(e.ctypes.data, d1.ctypes.data, d2.ctypes.data, params.ctypes.data,
                                        C.c_int64(V), traj["nr"], traj["ns"], C.c_float(traj["dt"]),
                                        C.c_float(dk.real), C.c_float(dk.imag), co.ctypes.data, Cn,
                                        ve.ctypes.data, _iptr(idx), C.c_int64(nidx), out.ctypes.data,
                                        nthreads or nthreads_default())
    return _as_complex(out)


def spiral_jacobian(echo, dT1, dT2, params, traj, coils, vec, entries=None, nthreads=None):
    """J·v on a spiral trajectory (no counterpart in the reference; derived from its spiral signal)."""
    e, d1, d2, params, co, ve = _cf(echo), _cf(dT1), _cf(dT2), _ff(params), _cf(coils), _cf(vec)
    ks, dk = _cf(traj["k_start"]), _cf(traj["dk"])
    R, V = echo.shape
    Cn = coils.shape[0]
    ent, nent = _entries(entries)
    shape = (nent,) if ent is not None else (Cn, traj["nr"], traj["ns"])
    out = _out(shape, "f64")
    lib().oracle_spiral_jacobian_f64(e.ctypes.data, d1.ctypes.data, d2.ctypes.data, params.ctypes.data, C.c_int64(V),
                                     traj["nr"], traj["ns"], C.c_float(traj["dt"]), ks.ctypes.data, dk.ctypes.data,
                                     co.ctypes.data, Cn, ve.ctypes.data, None if ent is None else ent.ctypes.data,
                                     C.c_int64(nent), out.ctypes.data, nthreads or nthreads_default())
    return _as_complex(out)


def spiral_jacobian_hermitian(echo, dT1, dT2, params, traj, coils, vec, vidx=None, nthreads=None):
    """Jᴴ·v on a spiral trajectory: [4][n]."""
    e, d1, d2, params, co, ve = _cf(echo), _cf(dT1), _cf(dT2), _ff(params), _cf(coils), _cf(vec)
    ks, dk = _cf(traj["k_start"]), _cf(traj["dk"])
    R, V = echo.shape
    Cn = coils.shape[0]
    idx, nidx = _ip(vidx)
    n = nidx if idx is not None else V
    out = _out((4, n), "f64")
    lib().oracle_spiral_jacobian_hermitian_f64(e.ctypes.data, d1.ctypes.data, d2.ctypes.data, params.ctypes.data,
                                               C.c_int64(V), traj["nr"], traj["ns"], C.c_float(traj["dt"]),
                                               ks.ctypes.data, dk.ctypes.data, co.ctypes.data, Cn, ve.ctypes.data,
                                               _iptr(idx), C.c_int64(nidx), out.ctypes.data,
                                               nthreads or nthreads_default())
    return _as_complex(out)


def residual(lhs, rhs):
    a, b = _cf(lhs), _cf(rhs)
    n = lhs.size
    out = np.zeros(lhs.shape + (2,), np.float64)
    obj = lib().oracle_residual_f64(a.ctypes.data, b.ctypes.data, C.c_int64(n), out.ctypes.data)
    return float(obj), _as_complex(out)


def cx_eval_f32(op: int, packed: np.ndarray) -> np.ndarray:
    """Evaluate the FP32 twin's complex primitives (see oracle_capi.cpp)."""
    packed = _ff(packed)
    n = packed.shape[0]
    out = np.zeros((n, 2), np.float32)
    rc = lib().oracle_cx_eval_f32(op, packed.ctypes.data, C.c_int64(n), out.ctypes.data)
    if rc != 0:
        raise ValueError("unknown op")
    return out


_REF = None
_REF_PATH = _HERE / "_ref" / "libref_kernels.so"


def ref_kernels():
    """The reference's own FISP and Cartesian-signal kernels built for the host
    (oracle/_ref/libref_kernels.so, oracle/Makefile target `ref`), or None where they were not
    built (no reference tree at build time)."""
    global _REF
    if _REF is None and _REF_PATH.exists():
        L = C.CDLL(str(_REF_PATH))
        L.ref_fisp.argtypes = [_P, _I64, _P, _I64, _P, _P, _I, _I, _F, _F, _F, _F, _I, _I, _I, _I, _I, _P, _I]
        L.ref_fisp.restype = C.c_int
        L.ref_signal_cartesian_entries.argtypes = [_P, _P, _I64, _I, _I, _F, _P, _F, _P, _I, _P, _I64, _P, _I]
        L.ref_signal_cartesian_entries.restype = None
        _REF = L
    return _REF


_REF_GPU = {}
_REF_GPU_PATH = {False: _HERE / "_ref" / "libref_gpu.so", True: _HERE / "_ref" / "libref_gpu_unchecked.so"}


def ref_gpu(unchecked=False):
    """The reference's FISP and pSSFP kernels built for the B200 with its own CUDA flags
    (oracle/_ref/libref_gpu.so, "reference kernels, re-hosted"), or None where they were not built.
    Entry points take device pointers (ints) and a cudaStream_t. unchecked: the build without the
    stand-in views' index checks (libref_gpu_unchecked.so), for timing launches that the checked
    build has run without a flagged index."""
    if unchecked not in _REF_GPU and _REF_GPU_PATH[unchecked].exists():
        L = C.CDLL(str(_REF_GPU_PATH[unchecked]))
        L.ref_gpu_fisp.argtypes = [_P, _I, _P, _P, _I, _I, _F, _F, _F, _F, _I, _I, _I, _P, _P, _P]
        L.ref_gpu_fisp.restype = C.c_int
        L.ref_gpu_pssfp.argtypes = [_P, _I, _P, _I, _F, _P, _I, _P, _P, _P, _I, _P, _P]
        L.ref_gpu_pssfp.restype = C.c_int
        L.ref_gpu_signal_cartesian.argtypes = [_P, _I, _P, _P, _I, _I, _I, _F, _P, _F, _P, _P]
        L.ref_gpu_signal_cartesian.restype = None
        L.ref_gpu_signal_spiral.argtypes = [_P, _I, _P, _P, _I, _I, _I, _F, _P, _P, _P, _P]
        L.ref_gpu_signal_spiral.restype = None
        L.ref_gpu_jacobian.argtypes = [_P, _I, _P, _P, _P, _P, _I, _I, _I, _F, _P, _F, _P, _P, _P]
        L.ref_gpu_jacobian.restype = None
        L.ref_gpu_jacobian_hermitian.argtypes = [_P, _I, _P, _P, _P, _P, _I, _I, _I, _F, _P, _F, _P, _P, _P]
        L.ref_gpu_jacobian_hermitian.restype = None
        for name in ("ref_gpu_out_of_bounds", "ref_gpu_products_out_of_bounds", "ref_gpu_hermitian_out_of_bounds"):
            getattr(L, name).argtypes = []
            getattr(L, name).restype = C.c_int
        _REF_GPU[unchecked] = L
    return _REF_GPU.get(unchecked)


def ref_gpu_out_of_bounds() -> int:
    """1 when any view index of the re-hosted reference kernels was out of range (and clamped)."""
    L = ref_gpu()
    flags = [L.ref_gpu_out_of_bounds(), L.ref_gpu_products_out_of_bounds(), L.ref_gpu_hermitian_out_of_bounds()]
    return -1 if min(flags) < 0 else max(flags)


def _dev(a, dtype):
    import torch

    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda").to(dtype).contiguous()


def ref_gpu_signal_cartesian(params, echos, traj, coils, unchecked=False):
    """Signal [C][R][S] (torch complex64) of the reference's default Cartesian path (MatmulFast: its
    kernels plus TF32 cuBLAS) on torch's current stream."""
    import torch

    p, e, c = _dev(_ff(params), torch.float32), _dev(echos, torch.complex64), _dev(coils, torch.complex64)
    ks = _dev(traj["k_start"], torch.complex64)
    V, C_, R, S = p.shape[1], c.shape[0], traj["nr"], traj["ns"]
    out = torch.empty((C_, R, S), dtype=torch.complex64, device="cuda")
    ref_gpu(unchecked).ref_gpu_signal_cartesian(p.data_ptr(), V, e.data_ptr(), c.data_ptr(), C_, R, S, traj["dt"],
                                       ks.data_ptr(), float(complex(traj["dk"]).real), out.data_ptr(),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return out


def ref_gpu_signal_spiral(params, echos, traj, coils, unchecked=False):
    """Spiral signal [C][R][S] (torch complex64) of the reference's spiral kernels on torch's
    current stream."""
    import torch

    p, e, c = _dev(_ff(params), torch.float32), _dev(echos, torch.complex64), _dev(coils, torch.complex64)
    ks, dk = _dev(traj["k_start"], torch.complex64), _dev(traj["dk"], torch.complex64)
    V, C_, R, S = p.shape[1], c.shape[0], traj["nr"], traj["ns"]
    out = torch.empty((C_, R, S), dtype=torch.complex64, device="cuda")
    ref_gpu(unchecked).ref_gpu_signal_spiral(p.data_ptr(), V, e.data_ptr(), c.data_ptr(), C_, R, S, traj["dt"], ks.data_ptr(),
                                    dk.data_ptr(), out.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return out


def ref_gpu_jacobian(params, echos, dT1, dT2, traj, coils, vector, hermitian=False, unchecked=False):
    """J·v [C][R][S] (vector [4][V]) or, with hermitian, Jᴴ·v [4][V] (vector [C][R][S]) of the
    reference's default GemmFast paths (its kernels plus TF32 cuBLAS), torch complex64."""
    import torch

    p = _dev(_ff(params), torch.float32)
    e, d1, d2 = (_dev(x, torch.complex64) for x in (echos, dT1, dT2))
    c, v = _dev(coils, torch.complex64), _dev(vector, torch.complex64)
    ks = _dev(traj["k_start"], torch.complex64)
    V, C_, R, S = p.shape[1], c.shape[0], traj["nr"], traj["ns"]
    shape = (4, V) if hermitian else (C_, R, S)
    out = torch.empty(shape, dtype=torch.complex64, device="cuda")
    fn = ref_gpu(unchecked).ref_gpu_jacobian_hermitian if hermitian else ref_gpu(unchecked).ref_gpu_jacobian
    fn(p.data_ptr(), V, e.data_ptr(), d1.data_ptr(), d2.data_ptr(), c.data_ptr(), C_, R, S, traj["dt"], ks.data_ptr(),
       float(complex(traj["dk"]).real), v.data_ptr(), out.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return out


def ref_gpu_fisp(params, seq, unchecked=False):
    """FISP echoes [nTR*uf][nv] (torch complex64) from the re-hosted reference kernels, launched on
    torch's current CUDA stream (the inputs' temporaries are freed in that stream's order);
    `params` [9][nv] float32, `seq` a workloads-style dict."""
    import torch

    L = ref_gpu(unchecked)
    dev = torch.device("cuda")
    p = torch.as_tensor(_ff(params), device=dev)
    nv = p.shape[1]
    rf = torch.as_tensor(np.ascontiguousarray(seq["rf"], np.complex64), device=dev)
    sl = torch.as_tensor(np.ascontiguousarray(seq["slices"], np.complex64), device=dev)
    nTR, P, uf = rf.shape[0], sl.shape[0], int(seq.get("uf", 1))
    tr = torch.empty((nv, nTR), dtype=torch.complex64, device=dev)
    out = torch.empty((nTR * uf, nv), dtype=torch.complex64, device=dev)
    st = torch.cuda.current_stream()
    rc = L.ref_gpu_fisp(p.data_ptr(), nv, rf.data_ptr(), sl.data_ptr(), nTR, P, seq["TR"], seq["TE"],
                        seq.get("TW", 0.0), seq["TI"], int(seq["max_state"]), uf, int(seq.get("reps", 1)),
                        tr.data_ptr(), out.data_ptr(), C.c_void_p(st.cuda_stream))
    if rc != 0:
        raise ValueError("ref_gpu_fisp rejected its arguments")
    return out


def ref_gpu_pssfp(params, seq, unchecked=False):
    """pSSFP echoes [nTR][nv] (torch complex64) from the re-hosted reference kernels, on torch's
    current CUDA stream."""
    import torch

    L = ref_gpu(unchecked)
    dev = torch.device("cuda")
    p = torch.as_tensor(_ff(params), device=dev)
    nv = p.shape[1]
    rf = torch.as_tensor(np.ascontiguousarray(seq["rf"], np.complex64), device=dev)
    g = torch.as_tensor(np.ascontiguousarray(seq["gdtrf"], np.complex64), device=dev)
    z = torch.as_tensor(_ff(seq["z"]), device=dev)
    dt = (C.c_float * 3)(*seq["dt"])
    gz = (C.c_float * 3)(*seq["gz"])
    out = torch.empty((rf.shape[0], nv), dtype=torch.complex64, device=dev)
    st = torch.cuda.current_stream()
    rc = L.ref_gpu_pssfp(p.data_ptr(), nv, rf.data_ptr(), rf.shape[0], seq["TR"], g.data_ptr(), g.shape[0], dt, gz,
                         z.data_ptr(), z.shape[0], out.data_ptr(), C.c_void_p(st.cuda_stream))
    if rc != 0:
        raise ValueError("ref_gpu_pssfp rejected its arguments")
    return out


def ref_fisp(params, seq, vidx=None, nthreads=None):
    """Echoes [nTR*uf][n] from the reference's simulate_fisp kernel run on the host cores."""
    L = ref_kernels()
    params = _ff(params)
    nv = params.shape[1]
    idx, nidx = _ip(vidx)
    n = nidx if idx is not None else nv
    rf, slices = _cf(seq["rf"]), _cf(seq["slices"])
    nTR, P = len(seq["rf"]), seq["slices"].shape[0]
    out = np.zeros((nTR * int(seq.get("uf", 1)), n, 2), np.float32)
    rc = L.ref_fisp(params.ctypes.data, C.c_int64(nv), _iptr(idx), C.c_int64(n), rf.ctypes.data, slices.ctypes.data,
                    nTR, P, C.c_float(seq["TR"]), C.c_float(seq["TE"]), C.c_float(seq.get("TW", 0.0)),
                    C.c_float(seq["TI"]), int(seq["max_state"]), int(seq.get("uf", 1)), int(seq.get("reps", 1)),
                    int(seq.get("inversion", 1)), int(seq.get("wait_spoil", 1)), out.ctypes.data,
                    nthreads or nthreads_default())
    if rc != 0:
        raise ValueError("ref_fisp rejected its arguments")
    return _as_complex(out)


def ref_signal_cartesian(echo, params, traj, coils, entries, nthreads=None):
    """Signal entries (coil, readout, sample) from the reference's naive Cartesian kernel on the host."""
    L = ref_kernels()
    e, params, ks, co = _cf(echo), _ff(params), _cf(traj["k_start"]), _cf(coils)
    R, V = echo.shape
    ent = np.ascontiguousarray(entries, dtype=np.int32)
    out = np.zeros((len(ent), 2), np.float32)
    L.ref_signal_cartesian_entries(e.ctypes.data, params.ctypes.data, C.c_int64(V), traj["nr"], traj["ns"],
                                   C.c_float(traj["dt"]), ks.ctypes.data, C.c_float(complex(traj["dk"]).real),
                                   co.ctypes.data, coils.shape[0], ent.ctypes.data, C.c_int64(len(ent)),
                                   out.ctypes.data, nthreads or nthreads_default())
    return _as_complex(out)


def cartesian_model_entries(echo_rows, T2, B0, x, y, rho, coils, traj, entries):
    """FP64 numpy form of the Cartesian forward model that compute_jacobian differentiates,
    s[c][r][k] = Σ_v C[c][v]·ρ_v·m[r][v]·E_k(v), E_k = exp((k − S/2)(−Δt/T2 + iΘ)),
    Θ = Re Δk·x + Im Δk·y + 2πΔt·B0 (src/jacobian/product_kernels.cuh:42-63 with
    include/compas/trajectories/cartesian_view.cuh:65-80; for a real Δk it equals the signal of
    src/trajectories/signal_kernels.cuh's naive kernel). Every input is float64 / complex128, so a
    finite difference at a relative step of 1e-4 keeps about 12 digits: echo_rows maps each readout
    r that occurs in `entries` to its complex128 row m[r][:]; T2, B0, x, y float64 [V]; rho
    complex128 [V]; coils complex [C][V]. Returns complex128 [len(entries)]."""
    # Δt and Δk cross the C ABI as float32; round them as the library and the oracle see them
    S, dt = traj["ns"], float(np.float32(traj["dt"]))
    dk = complex(traj["dk"])
    dk = complex(float(np.float32(dk.real)), float(np.float32(dk.imag)))
    theta = dk.real * x + dk.imag * y + 2 * np.pi * dt * B0
    arg = -dt / T2 + 1j * theta
    co = np.asarray(coils, np.complex128)
    out = np.empty(len(entries), np.complex128)
    for i, (c, r, k) in enumerate(np.asarray(entries)):
        E = np.exp((float(k) - 0.5 * S) * arg)
        out[i] = np.sum(co[c] * rho * echo_rows[int(r)] * E)
    return out


def jacobian_fd_entries(echo, dT1, dT2, params, traj, coils, vec, entries, h=1e-4):
    """J·v at `entries` by an FP64 central difference of cartesian_model_entries along the direction
    that the Jacobian's columns are scaled for (product_kernels.cuh:56-60): T1 → T1·(1 + h·w0),
    T2 → T2·(1 + h·w1), ρ → ρ + h·(w2 + i·w3), with the echoes linearised,
    m → m + h·(w0·T1·∂m/∂T1 + w1·T2·∂m/∂T2). A complex v splits by linearity into
    J(Re v) + i·J(Im v), each a real direction. The truncation error is O(h²) ≈ 1e-8 relative."""
    p = np.asarray(params, np.float64)
    T1, T2, B0, x, y = p[0], p[1], p[3], p[6], p[7]
    rho = p[4] + 1j * p[5]
    rows = sorted({int(r) for r in np.asarray(entries)[:, 1]})
    m = {r: np.asarray(echo[r], np.complex128) for r in rows}
    m1 = {r: np.asarray(dT1[r], np.complex128) * T1 for r in rows}
    m2 = {r: np.asarray(dT2[r], np.complex128) * T2 for r in rows}
    vec = np.asarray(vec, np.complex128)

    def along(w):
        def at(s):
            mm = {r: m[r] + s * h * (w[0] * m1[r] + w[1] * m2[r]) for r in rows}
            return cartesian_model_entries(mm, T2 * (1 + s * h * w[1]), B0, x, y, rho + s * h * (w[2] + 1j * w[3]),
                                           coils, traj, entries)
        return (at(1.0) - at(-1.0)) / (2 * h)

    return along(vec.real) + 1j * along(vec.imag)


def derivative_central(simulate, params, seq, field: int, rel_step: float = 1e-4, vidx=None, **kw):
    """∂echo/∂params[field] by an FP64 central difference of an oracle simulation (`fisp` or
    `pssfp`) with a step of rel_step·|p| per voxel (voxels are independent, so all are stepped at
    once). The reference's derivative is the forward difference with an absolute step
    (src/simulate/derivative.cu:11-62, derivative_kernels.cuh:6-35); this is its Δ → 0 limit to
    O(step²), the quantity the tangent kernels compute. The stepped parameters are float32 (the
    oracle's input type), so the exact float32 difference of the two points divides."""
    p = _ff(params)
    step = np.maximum(np.abs(p[field]) * np.float32(rel_step), np.float32(1e-12)).astype(np.float32)
    hi, lo = p.copy(), p.copy()
    hi[field] = p[field] + step
    lo[field] = p[field] - step
    den = hi[field].astype(np.float64) - lo[field].astype(np.float64)
    if vidx is not None:
        den = den[np.asarray(vidx)]
    return (simulate(hi, seq, vidx=vidx, **kw) - simulate(lo, seq, vidx=vidx, **kw)) / den[None, :]


def rel_l2(x, ref) -> float:
    x = np.asarray(x, np.complex128)
    ref = np.asarray(ref, np.complex128)
    den = np.linalg.norm(ref.ravel())
    return float(np.linalg.norm((x - ref).ravel()) / (den if den > 0 else 1.0))
