"""Python front-end of libcompas_b200.so (the C ABI in include/compas_b200.h).

Mirrors the reference's Julia module (CompasToolkit.jl/src/CompasToolkit.jl): a
``Context``, device arrays (``CompasArray``), ``TissueParameters``,
``FispSequence`` / ``pSSFPSequence``, ``CartesianTrajectory`` / ``SpiralTrajectory``
and the operations ``simulate_magnetization``, ``simulate_magnetization_derivative(s)``,
``magnetization_to_signal``, ``compute_jacobian``, ``compute_jacobian_hermitian``,
``phase_encoding`` and ``compute_residual``. Every call goes through the C ABI
symbols the Julia module binds; arrays use the C++ row-major layout (slowest
dimension first), which is the reverse of the Julia view.

The GPU library is required: importing works without it, but every operation raises
``CompasError`` when libcompas_b200.so is missing — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

_HERE = Path(__file__).resolve().parent
LIBRARY_PATH = Path(os.environ.get("COMPAS_B200_LIBRARY", _HERE / "libcompas_b200.so"))

# enum values of the reference (compas/trajectories/signal.h:14-44, compas/jacobian/product.h:10)
SIGNAL_METHODS = {"Naive": 0, "Direct": 1, "MatmulPedantic": 2, "Matmul": 3, "MatmulFast": 4, "MatmulLow": 5}
JACOBIAN_METHODS = {"Naive": 0, "Direct": 1, "Gemm": 2, "GemmFast": 3, "GemmLow": 4}
FIELDS = {"T1": 0, "T2": 1, "B1": 2, "B0": 3, "rho_x": 4, "rho_y": 5, "x": 6, "y": 7, "z": 8}


class CompasError(RuntimeError):
    pass


_P, _I, _I32, _I64, _F = C.c_void_p, C.c_int, C.c_int32, C.c_int64, C.c_float
_SIGS = {
    "compas_version": ([], C.c_char_p),
    "compas_last_error": ([], C.c_char_p),
    "compas_make_context": ([], _P),
    "compas_copy_context_for_device": ([_P, _I], _P),
    "compas_destroy_context": ([_P], None),
    "compas_destroy_object": ([_P], None),
    "compas_synchronize": ([_P], None),
    "compas_make_array_float": ([_P, _P, _I, _P], _P),
    "compas_read_array_float": ([_P, _P, _P, _I64], None),
    "compas_make_array_complex": ([_P, _P, _I, _P], _P),
    "compas_read_array_complex": ([_P, _P, _P, _I64], None),
    "compas_destroy_array": ([_P], None),
    "compas_make_tissue_parameters": ([_P, _I] + [_P] * 9, _P),
    "compas_make_fisp_sequence": ([_P, _P, _F, _F, _F, _I, _F, _I, _I], _P),
    "compas_b200_make_fisp_sequence_ex": ([_P, _P, _F, _F, _F, _I, _F, _I, _I, _I, _I], _P),
    "compas_make_pssfp_sequence": ([_P, _F, _P, _F, _F, _F, _F, _F, _F, _P], _P),
    "compas_make_cartesian_trajectory": ([_I, _I, _F, _P, _F], _P),
    "compas_make_spiral_trajectory": ([_I, _I, _F, _P, _P], _P),
    "compas_simulate_magnetization_fisp": ([_P, _P, _P], _P),
    "compas_simulate_magnetization_pssfp": ([_P, _P, _P], _P),
    "compas_magnetization_to_signal_cartesian": ([_P, _I, _P, _P, _P, _P, _I32], _P),
    "compas_magnetization_to_signal_spiral": ([_P, _I, _P, _P, _P, _P], _P),
    "compas_compute_jacobian": ([_P, _I, _P, _P, _P, _P, _P, _P, _P, _I32], _P),
    "compas_compute_jacobian_hermitian": ([_P, _I, _P, _P, _P, _P, _P, _P, _P, _I32], _P),
    "phase_encoding": ([_P, _P, _P, _P], _P),
    "compas_compute_residual": ([_P, _P, _P, _P], _P),
    "compas_simulate_magnetization_derivative_pssfp": ([_P, _I, _P, _P, _F, _P], _P),
    "compas_simulate_magnetization_derivative_fisp": ([_P, _I, _P, _P, _F, _P], _P),
    "compas_b200_magnetization_to_signal": ([_P, _P, _P, _P, _P, _I], _P),
    "compas_b200_compute_jacobian": ([_P, _P, _P, _P, _P, _P, _P, _P, _I], _P),
    "compas_b200_compute_jacobian_hermitian": ([_P, _P, _P, _P, _P, _P, _P, _P, _I], _P),
    "compas_b200_context_stream": ([_P], _P),
    "compas_b200_array_device_ptr": ([_P], _P),
    "compas_b200_array_rank": ([_P], _I),
    "compas_b200_array_extent": ([_P, _I], _I64),
    "compas_b200_compute_residual_noalloc": ([_I, _P, _P, _P, _P, _I64, _P], _I),
    "compas_b200_launch_count": ([], C.c_uint64),
    "compas_b200_set_fisp_launch": ([_I, _I], None),
    "compas_b200_set_pssfp_launch": ([_I], None),
    "compas_b200_fisp_config_count": ([], _I),
    "compas_b200_fisp_config_info": ([_I, C.POINTER(C.c_int), C.POINTER(C.c_int)], _I),
    "compas_b200_fisp_config_packed": ([_I], _I),
    "compas_b200_pssfp_config_count": ([], _I),
    "compas_b200_pssfp_config_info": ([_I, C.POINTER(C.c_int), C.POINTER(C.c_int)], _I),
    "compas_b200_pssfp_config_packed": ([_I], _I),
    "compas_b200_fisp_launch_choice": ([_I, _I64, _I, C.POINTER(C.c_int), C.POINTER(C.c_int)], None),
    "compas_b200_pssfp_launch_choice": ([_I, _I64], _I),
    "compas_b200_set_tc_launch": ([_I, _I, _I], None),
    "compas_b200_tc_launch_choice": ([_I, _I, _I, _I, _I, _I, C.POINTER(C.c_int), C.POINTER(C.c_int)], _I),
    "compas_b200_simulate_magnetization_tangents": ([_P, _P, _P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)], _I),
    "compas_b200_set_fisp_tangent_launch": ([_I], None),
    "compas_b200_fisp_tangent_config_count": ([], _I),
    "compas_b200_fisp_tangent_config_info": ([_I, C.POINTER(C.c_int), C.POINTER(C.c_int)], _I),
    "compas_b200_fisp_tangent_config_packed": ([_I], _I),
    "compas_b200_make_batch": ([_P, _I, _P, _P, _P, _P, _I], _P),
    "compas_b200_make_batch_tangents": ([_P, _I, _P, _P, _P, _P, _I, _P], _P),
    "compas_b200_batch_derivative": ([_P, _I, _I], _P),
    "compas_b200_batch_run": ([_P], _I),
    "compas_b200_batch_echos": ([_P, _I], _P),
    "compas_b200_batch_signal": ([_P, _I], _P),
    "compas_b200_make_gauss_newton": ([_P, _P, _P, _P, _P, _P, _I, _F, _I], _P),
    "compas_b200_gauss_newton_run": ([_P, _I], _I),
    "compas_b200_gauss_newton_array": ([_P, _I], _P),
    "compas_b200_gauss_newton_graph_kernels": ([_P], _I),
    "compas_b200_make_server": ([_P, C.c_double, _I, _I, C.c_double, _I, _F], _P),
    "compas_b200_server_submit": ([_P, _P, _P, _P, _P, _P, C.c_uint64], _I64),
    "compas_b200_server_submit_flags": ([_P, _P, _P, _P, _P, _P, C.c_uint64, _I], _I64),
    "compas_b200_wait_probe": ([_P, _I64], _I),
    "compas_b200_gauss_newton_set_line_search": ([_P, _I], _I),
    "compas_b200_voxel_shard": ([_I64, _I, _I, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], _I),
    "compas_b200_compute_gemm": ([_P, _P, _P, _P, C.c_float, C.c_float, _I], _I),
    "compas_b200_compute_complex_gemm": ([_P, _P, _P, _P, C.c_float, C.c_float, _I], _I),
    "compas_b200_convert_complex_to_planar": ([_P, _P, _P], _I),
    "compas_b200_convert_planar_to_complex": ([_P, _P, _P], _I),
    "compas_b200_make_array_bfloat16": ([_P, _P, _I, C.POINTER(C.c_int64)], _P),
    "compas_b200_read_array_bfloat16": ([_P, _P, _P, _I64], None),
    "compas_b200_comm_unique_id": ([C.c_char_p, _I], _I),
    "compas_b200_make_communicator": ([_P, _I, _I, C.c_char_p], _P),
    "compas_b200_allreduce_sum": ([_P, _P, _P], _I),
    "compas_b200_magnetization_to_signal_sharded": ([_P, _P, _P, _P, _P, _P, _I], _P),
    "compas_b200_compute_jacobian_sharded": ([_P, _P, _P, _P, _P, _P, _P, _P, _P, _I], _P),
    "compas_b200_server_wait": ([_P, _I64, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)], _I),
    "compas_b200_server_result": ([_P, _I64, _I], _P),
    "compas_b200_server_release": ([_P, _I64], _I),
    "compas_b200_server_drain": ([_P], _I),
    "compas_b200_server_stats": ([_P, C.POINTER(C.c_double), _I], _I),
    "compas_b200_server_reset_stats": ([_P], None),
}

_LIB = None


def library() -> C.CDLL:
    """Load libcompas_b200.so (raises CompasError when it has not been built)."""
    global _LIB
    if _LIB is None:
        if not LIBRARY_PATH.exists():
            raise CompasError(f"{LIBRARY_PATH} not found: build it with __graft_entry__.build() "
                              "(make -C compas-toolkit_b200)")
        lib = C.CDLL(str(LIBRARY_PATH))
        for name, (args, res) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _LIB = lib
    return _LIB


def exported_symbols() -> list:
    return list(_SIGS)


def _check(result=None, what="compas call"):
    err = library().compas_last_error()
    if err is not None:
        raise CompasError(err.decode(errors="replace"))
    if result is None and what is not None and what.endswith("!"):
        raise CompasError(f"{what[:-1]} returned NULL")
    return result


def version() -> str:
    return library().compas_version().decode()


class Context:
    """A COMPAS context on one device (compas_make_context / compas_copy_context_for_device)."""

    def __init__(self, device: int = 0):
        lib = library()
        base = lib.compas_make_context()
        _check(base, "compas_make_context!")
        if device != 0:
            ptr = lib.compas_copy_context_for_device(base, device)
            lib.compas_destroy_context(base)
            _check(ptr, "compas_copy_context_for_device!")
            base = ptr
        self.ptr = base
        self.device = device

    def synchronize(self):
        library().compas_synchronize(self.ptr)
        _check()

    @property
    def stream(self) -> int:
        """cudaStream_t of this context (all its work is ordered on it)."""
        return library().compas_b200_context_stream(self.ptr) or 0

    def __del__(self):
        if getattr(self, "ptr", None) and _LIB is not None:
            _LIB.compas_destroy_context(self.ptr)
            self.ptr = None


class CompasArray:
    """Device array handle (float32 or complex64, rank 1-3), row-major like the C++ side."""

    def __init__(self, context: Context, ptr, dtype, shape):
        self.context = context
        self.ptr = ptr
        self.dtype = np.dtype(dtype)
        self.shape = tuple(int(s) for s in shape)

    @staticmethod
    def from_bfloat16(context: Context, arr) -> "CompasArray":
        """A bfloat16 device array from float values (rounded to the nearest bfloat16); its numpy
        side is the raw 16-bit patterns (dtype uint16, see bfloat16_bits / bfloat16_values)."""
        bits = bfloat16_bits(arr)
        if bits.ndim < 1 or bits.ndim > 3:
            raise CompasError("cannot support rank > 3")
        sizes = (C.c_int64 * bits.ndim)(*bits.shape)
        ptr = library().compas_b200_make_array_bfloat16(context.ptr, bits.ctypes.data, bits.ndim, sizes)
        _check(ptr, "compas_b200_make_array_bfloat16!")
        return CompasArray(context, ptr, np.uint16, bits.shape)

    @staticmethod
    def from_numpy(context: Context, arr) -> "CompasArray":
        arr = np.asarray(arr)
        if np.iscomplexobj(arr):
            a = np.ascontiguousarray(arr, dtype=np.complex64)
            fn = library().compas_make_array_complex
        else:
            a = np.ascontiguousarray(arr, dtype=np.float32)
            fn = library().compas_make_array_float
        if a.ndim < 1 or a.ndim > 3:
            raise CompasError("cannot support rank > 3")
        sizes = (C.c_int64 * a.ndim)(*a.shape)
        ptr = fn(context.ptr, a.ctypes.data, a.ndim, sizes)
        _check(ptr, "compas_make_array!")
        return CompasArray(context, ptr, a.dtype, a.shape)

    @property
    def size(self) -> int:
        return int(np.prod(self.shape)) if self.shape else 0

    @property
    def device_ptr(self) -> int:
        return library().compas_b200_array_device_ptr(self.ptr) or 0

    def to_numpy(self) -> np.ndarray:
        out = np.empty(self.shape, self.dtype)
        if self.dtype == np.uint16:
            library().compas_b200_read_array_bfloat16(self.context.ptr, self.ptr, out.ctypes.data, out.size)
            _check()
            return out
        fn = library().compas_read_array_complex if self.dtype == np.complex64 else library().compas_read_array_float
        fn(self.context.ptr, self.ptr, out.ctypes.data, out.size)
        _check()
        return out

    @property
    def __cuda_array_interface__(self) -> dict:
        """Zero-copy float32 view for CUDA-aware libraries (e.g. torch.as_tensor(arr, device="cuda"));
        the consumer orders its use after the context's stream, on which the array was produced."""
        # complex values are exposed as float32 pairs (trailing axis of 2): consumers differ in
        # their support of complex type strings
        shape = self.shape + (2,) if self.dtype == np.complex64 else self.shape
        return {"shape": shape, "typestr": "<f4", "data": (self.device_ptr, False), "version": 3,
                "strides": None, "stream": int(self.context.stream) or None}

    def read_into(self, out: np.ndarray) -> np.ndarray:
        """Blocking copy into a preallocated (e.g. pinned) host array of matching size/dtype."""
        assert out.dtype == self.dtype and out.size == self.size and out.flags.c_contiguous
        fn = library().compas_read_array_complex if self.dtype == np.complex64 else library().compas_read_array_float
        fn(self.context.ptr, self.ptr, out.ctypes.data, out.size)
        _check()
        return out

    collect = to_numpy

    def __del__(self):
        if getattr(self, "ptr", None) and _LIB is not None:
            _LIB.compas_destroy_array(self.ptr)
            self.ptr = None

    def __repr__(self):
        return f"CompasArray{{{self.dtype}}} of size {self.shape}"


def _arr(context, a, dtype=None) -> CompasArray:
    if isinstance(a, CompasArray):
        return a
    a = np.asarray(a)
    if dtype is not None:
        a = a.astype(dtype, copy=False)
    return CompasArray.from_numpy(context, a)


class _Object:
    def __init__(self, ptr, keep=()):
        _check(ptr, "constructor!")
        self.ptr = ptr
        self._keep = keep

    def __del__(self):
        if getattr(self, "ptr", None) and _LIB is not None:
            _LIB.compas_destroy_object(self.ptr)
            self.ptr = None


class TissueParameters(_Object):
    """compas_make_tissue_parameters; fields as host vectors of nvoxels floats."""

    def __init__(self, context: Context, nvoxels: int, T1, T2, B1, B0, rho_x, rho_y, x, y, z=None):
        cols = [np.ascontiguousarray(np.broadcast_to(np.asarray(c, np.float32), (nvoxels,)))
                for c in (T1, T2, B1, B0, rho_x, rho_y, x, y)]
        cols.append(np.zeros(nvoxels, np.float32) if z is None else
                    np.ascontiguousarray(np.broadcast_to(np.asarray(z, np.float32), (nvoxels,))))
        ptr = library().compas_make_tissue_parameters(context.ptr, int(nvoxels), *[c.ctypes.data for c in cols])
        super().__init__(ptr)
        self.nvoxels = int(nvoxels)

    @staticmethod
    def from_soa(context: Context, params: np.ndarray) -> "TissueParameters":
        p = np.asarray(params, np.float32)
        return TissueParameters(context, p.shape[1], *p)


class FispSequence(_Object):
    """compas_make_fisp_sequence: RF train [nTR] (deg, phase), slice profiles [npos][nTR]. Without the
    inversion prepulse or the wait spoiling (both on in the reference's C ABI) it is built by
    compas_b200_make_fisp_sequence_ex."""

    def __init__(self, context: Context, RF_train, slice_profiles, TR: float, TE: float, max_state: int, TI: float,
                 undersampling_factor: int = 1, repetitions: int = 1, TW: float = 0.0,
                 inversion_prepulse: bool = True, wait_spoiling: bool = True):
        rf = _arr(context, np.asarray(RF_train, np.complex64))
        sp = _arr(context, np.asarray(slice_profiles, np.complex64).reshape(-1, rf.shape[0]))
        if inversion_prepulse and wait_spoiling:
            ptr = library().compas_make_fisp_sequence(rf.ptr, sp.ptr, TR, TE, TW, int(max_state), TI,
                                                      int(undersampling_factor), int(repetitions))
        else:
            ptr = library().compas_b200_make_fisp_sequence_ex(rf.ptr, sp.ptr, TR, TE, TW, int(max_state), TI,
                                                              int(undersampling_factor), int(repetitions),
                                                              int(bool(inversion_prepulse)), int(bool(wait_spoiling)))
        super().__init__(ptr, (rf, sp))
        self.nreadouts = rf.shape[0] * int(undersampling_factor)
        self.max_state = int(max_state)
        self.npositions = sp.shape[0]

    @staticmethod
    def from_dict(context: Context, s: dict) -> "FispSequence":
        return FispSequence(context, s["rf"], s["slices"], s["TR"], s["TE"], s["max_state"], s["TI"],
                            s.get("uf", 1), s.get("reps", 1), s.get("TW", 0.0), bool(s.get("inversion", 1)),
                            bool(s.get("wait_spoil", 1)))


class pSSFPSequence(_Object):
    """compas_make_pssfp_sequence. `z` is passed as float32, which is what the C++ side reads
    (compas/sequences/pssfp.h: Array<float>); the reference's Julia wrapper converts it to
    ComplexF32 (CompasToolkit.jl), which does not match."""

    def __init__(self, context: Context, RF_train, TR: float, gamma_dt_RF, dt: Sequence[float],
                 gamma_dt_GRz: Sequence[float], z):
        rf = _arr(context, np.asarray(RF_train, np.complex64))
        g = _arr(context, np.asarray(gamma_dt_RF, np.complex64))
        zz = _arr(context, np.asarray(z, np.float32))
        ptr = library().compas_make_pssfp_sequence(rf.ptr, TR, g.ptr, dt[0], dt[1], dt[2], gamma_dt_GRz[0],
                                                   gamma_dt_GRz[1], gamma_dt_GRz[2], zz.ptr)
        super().__init__(ptr, (rf, g, zz))
        self.nreadouts = rf.shape[0]

    @staticmethod
    def from_dict(context: Context, s: dict) -> "pSSFPSequence":
        return pSSFPSequence(context, s["rf"], s["TR"], s["gdtrf"], s["dt"], s["gz"], s["z"])


class CartesianTrajectory(_Object):
    def __init__(self, context: Context, nreadouts: int, samples_per_readout: int, delta_t: float, k_start,
                 delta_k: float):
        ks = _arr(context, np.asarray(k_start, np.complex64))
        ptr = library().compas_make_cartesian_trajectory(int(nreadouts), int(samples_per_readout), delta_t, ks.ptr,
                                                         float(delta_k))
        super().__init__(ptr, (ks,))
        self.nreadouts, self.samples_per_readout = int(nreadouts), int(samples_per_readout)

    @staticmethod
    def from_dict(context: Context, t: dict) -> "CartesianTrajectory":
        return CartesianTrajectory(context, t["nr"], t["ns"], t["dt"], t["k_start"], t["dk"])


class SpiralTrajectory(_Object):
    def __init__(self, context: Context, nreadouts: int, samples_per_readout: int, delta_t: float, k_start, delta_k):
        ks = _arr(context, np.asarray(k_start, np.complex64))
        dk = _arr(context, np.asarray(delta_k, np.complex64))
        ptr = library().compas_make_spiral_trajectory(int(nreadouts), int(samples_per_readout), delta_t, ks.ptr,
                                                      dk.ptr)
        super().__init__(ptr, (ks, dk))
        self.nreadouts, self.samples_per_readout = int(nreadouts), int(samples_per_readout)

    @staticmethod
    def from_dict(context: Context, t: dict) -> "SpiralTrajectory":
        return SpiralTrajectory(context, t["nr"], t["ns"], t["dt"], t["k_start"], t["dk"])


def trajectory_from_dict(context: Context, t: dict):
    return (CartesianTrajectory if t.get("kind", "cartesian") == "cartesian" else SpiralTrajectory).from_dict(context, t)


def _result(ptr, context, shape, what) -> CompasArray:
    _check(ptr, what + "!")
    return CompasArray(context, ptr, np.complex64, shape)


def simulate_magnetization(context: Context, parameters: TissueParameters, sequence) -> CompasArray:
    lib = library()
    if isinstance(sequence, FispSequence):
        ptr = lib.compas_simulate_magnetization_fisp(context.ptr, parameters.ptr, sequence.ptr)
    elif isinstance(sequence, pSSFPSequence):
        ptr = lib.compas_simulate_magnetization_pssfp(context.ptr, parameters.ptr, sequence.ptr)
    else:
        raise CompasError("unknown sequence type")
    return _result(ptr, context, (sequence.nreadouts, parameters.nvoxels), "simulate_magnetization")


def simulate_magnetization_derivative(context: Context, field, echos, parameters: TissueParameters, sequence,
                                      delta: float = 1e-4) -> CompasArray:
    field = FIELDS[field] if isinstance(field, str) else int(field)
    e = _arr(context, echos, np.complex64)
    lib = library()
    fn = (lib.compas_simulate_magnetization_derivative_fisp if isinstance(sequence, FispSequence)
          else lib.compas_simulate_magnetization_derivative_pssfp)
    ptr = fn(context.ptr, field, e.ptr, parameters.ptr, delta, sequence.ptr)
    return _result(ptr, context, e.shape, "simulate_magnetization_derivative")


def simulate_magnetization_derivatives(context, echos, parameters, sequence, delta: float = 1e-4) -> dict:
    return {"T1": simulate_magnetization_derivative(context, 0, echos, parameters, sequence, delta),
            "T2": simulate_magnetization_derivative(context, 1, echos, parameters, sequence, delta)}


def simulate_magnetization_tangents(context: Context, parameters: TissueParameters, sequence) -> dict:
    """Echoes and their exact derivatives ∂/∂T1, ∂/∂T2 in one pass (forward-mode tangents):
    {"echos", "T1", "T2"}, each [nreadouts][nvoxels]. "echos" is simulate_magnetization's
    recurrence (equal to FP32 rounding); "T1"/"T2" are the Δ → 0 limit of
    simulate_magnetization_derivative."""
    if not isinstance(sequence, (FispSequence, pSSFPSequence)):
        raise CompasError("unknown sequence type")
    out = [_P(), _P(), _P()]
    rc = library().compas_b200_simulate_magnetization_tangents(context.ptr, parameters.ptr, sequence.ptr,
                                                               C.byref(out[0]), C.byref(out[1]), C.byref(out[2]))
    if rc != 0:
        _check(None, "simulate_magnetization_tangents!")
    shape = (sequence.nreadouts, parameters.nvoxels)
    return {k: CompasArray(context, p.value, np.complex64, shape) for k, p in zip(("echos", "T1", "T2"), out)}


def magnetization_to_signal(context: Context, echos, parameters: TissueParameters, trajectory, coils,
                            method: Optional[str] = None, low_precision: bool = False) -> CompasArray:
    """method=None uses the reference's C ABI entry point (MatmulFast, or MatmulLow when
    low_precision); a method name from SIGNAL_METHODS selects it explicitly."""
    e = _arr(context, echos, np.complex64)
    c = _arr(context, coils, np.complex64)
    lib = library()
    shape = (c.shape[0], trajectory.nreadouts, trajectory.samples_per_readout)
    if method is not None:
        ptr = lib.compas_b200_magnetization_to_signal(context.ptr, e.ptr, parameters.ptr, trajectory.ptr, c.ptr,
                                                      SIGNAL_METHODS[method])
    elif isinstance(trajectory, CartesianTrajectory):
        ptr = lib.compas_magnetization_to_signal_cartesian(context.ptr, c.shape[0], e.ptr, parameters.ptr, c.ptr,
                                                           trajectory.ptr, int(bool(low_precision)))
    else:
        ptr = lib.compas_magnetization_to_signal_spiral(context.ptr, c.shape[0], e.ptr, parameters.ptr, c.ptr,
                                                        trajectory.ptr)
    return _result(ptr, context, shape, "magnetization_to_signal")


def compute_jacobian(context: Context, echos, dechos: dict, parameters: TissueParameters, trajectory, coils, v,
                     method: Optional[str] = None, low_precision: bool = False) -> CompasArray:
    e, d1, d2 = (_arr(context, a, np.complex64) for a in (echos, dechos["T1"], dechos["T2"]))
    c = _arr(context, coils, np.complex64)
    vv = _arr(context, v, np.complex64)
    lib = library()
    shape = (c.shape[0], trajectory.nreadouts, trajectory.samples_per_readout)
    if method is not None:
        ptr = lib.compas_b200_compute_jacobian(context.ptr, e.ptr, d1.ptr, d2.ptr, parameters.ptr, trajectory.ptr,
                                               c.ptr, vv.ptr, JACOBIAN_METHODS[method])
    else:
        ptr = lib.compas_compute_jacobian(context.ptr, c.shape[0], e.ptr, d1.ptr, d2.ptr, parameters.ptr, c.ptr,
                                          trajectory.ptr, vv.ptr, int(bool(low_precision)))
    return _result(ptr, context, shape, "compute_jacobian")


def compute_jacobian_hermitian(context: Context, echos, dechos: dict, parameters: TissueParameters, trajectory,
                               coils, v, method: Optional[str] = None, low_precision: bool = False) -> CompasArray:
    e, d1, d2 = (_arr(context, a, np.complex64) for a in (echos, dechos["T1"], dechos["T2"]))
    c = _arr(context, coils, np.complex64)
    vv = _arr(context, v, np.complex64)
    lib = library()
    shape = (4, parameters.nvoxels)
    if method is not None:
        ptr = lib.compas_b200_compute_jacobian_hermitian(context.ptr, e.ptr, d1.ptr, d2.ptr, parameters.ptr,
                                                         trajectory.ptr, c.ptr, vv.ptr, JACOBIAN_METHODS[method])
    else:
        ptr = lib.compas_compute_jacobian_hermitian(context.ptr, c.shape[0], e.ptr, d1.ptr, d2.ptr, parameters.ptr,
                                                    trajectory.ptr, c.ptr, vv.ptr, int(bool(low_precision)))
    return _result(ptr, context, shape, "compute_jacobian_hermitian")


def phase_encoding(context: Context, echos, parameters: TissueParameters, trajectory) -> CompasArray:
    e = _arr(context, echos, np.complex64)
    ptr = library().phase_encoding(context.ptr, e.ptr, parameters.ptr, trajectory.ptr)
    return _result(ptr, context, e.shape, "phase_encoding")


def compute_residual(context: Context, lhs, rhs):
    """Returns (Σ|lhs - rhs|², lhs - rhs) like the Julia wrapper."""
    a = _arr(context, lhs, np.complex64)
    b = _arr(context, rhs, np.complex64)
    obj = np.zeros(1, np.float32)
    ptr = library().compas_compute_residual(context.ptr, a.ptr, b.ptr, obj.ctypes.data)
    diff = _result(ptr, context, a.shape, "compute_residual")
    return float(obj[0]), diff


def job_from_dict(context: Context, job: dict) -> tuple:
    """(parameters, sequence, trajectory, coils) of a job dict as made by workloads.batch_jobs."""
    params = TissueParameters.from_soa(context, job["params"])
    seq = (FispSequence if job["kind"] == "fisp" else pSSFPSequence).from_dict(context, job["seq"])
    traj = trajectory_from_dict(context, job["traj"]) if job.get("traj") is not None else None
    coils = job.get("coils") if traj is not None else None
    return params, seq, traj, coils


class SimulationBatch(_Object):
    """compas_b200_make_batch: independent simulate -> signal jobs planned into a few launches
    (persistent work-queue simulation kernels, batched signal kernels).

    jobs: sequence of (parameters, sequence, trajectory or None, coils or None). Each job's
    echoes and signal equal those of simulate_magnetization + magnetization_to_signal(method).
    tangents: per-job flags; a flagged job also gets its exact ∂/∂T1, ∂/∂T2 (derivative())."""

    def __init__(self, context: Context, jobs, method: str = "MatmulFast", tangents=None):
        lib = library()
        n = len(jobs)
        arr_t = C.c_void_p * max(n, 1)
        coil_arrays = [None if j[3] is None else _arr(context, j[3], np.complex64) for j in jobs]
        params = arr_t(*[j[0].ptr for j in jobs])
        seqs = arr_t(*[j[1].ptr for j in jobs])
        trajs = arr_t(*[None if j[2] is None else j[2].ptr for j in jobs])
        coils = arr_t(*[None if c is None else c.ptr for c in coil_arrays])
        flags = None if tangents is None else (C.c_int32 * max(n, 1))(*[int(bool(t)) for t in tangents])
        ptr = lib.compas_b200_make_batch_tangents(context.ptr, n, C.cast(params, _P), C.cast(seqs, _P),
                                                  C.cast(trajs, _P), C.cast(coils, _P), SIGNAL_METHODS[method],
                                                  None if flags is None else C.cast(flags, _P))
        super().__init__(ptr, (list(jobs), coil_arrays))
        self.context = context
        self.jobs = list(jobs)
        self.coil_arrays = coil_arrays

    def __len__(self):
        return len(self.jobs)

    def run(self):
        """Enqueue every job on the context's stream (returns without waiting)."""
        if library().compas_b200_batch_run(self.ptr) != 0:
            _check(None, "compas_b200_batch_run!")

    def derivative(self, job: int, field) -> CompasArray:
        """∂echos/∂T1 ("T1" / 0) or ∂echos/∂T2 ("T2" / 1) of a job made with tangents."""
        f = {"T1": 0, "T2": 1}.get(field, field)
        ptr = library().compas_b200_batch_derivative(self.ptr, int(job), int(f))
        _check(ptr, "compas_b200_batch_derivative!")
        return CompasArray(self.context, ptr, np.complex64, (self.jobs[job][1].nreadouts, self.jobs[job][0].nvoxels))

    def echos(self, job: int) -> CompasArray:
        params, seq = self.jobs[job][0], self.jobs[job][1]
        ptr = library().compas_b200_batch_echos(self.ptr, int(job))
        return _result(ptr, self.context, (seq.nreadouts, params.nvoxels), "compas_b200_batch_echos")

    def signal(self, job: int) -> CompasArray:
        traj, coils = self.jobs[job][2], self.coil_arrays[job]
        if traj is None:
            raise CompasError("job has no trajectory")
        ptr = library().compas_b200_batch_signal(self.ptr, int(job))
        shape = (coils.shape[0], traj.nreadouts, traj.samples_per_readout)
        return _result(ptr, self.context, shape, "compas_b200_batch_signal")


class GaussNewtonStep(_Object):
    """compas_b200_make_gauss_newton: one Gauss-Newton iteration on the device (simulate,
    derivatives — forward differences with step `delta`, or exact tangents for delta=0 — signal,
    residual against `data`, `cg_iterations` CGLS steps of J·v / Jᴴ·v, parameter update),
    captured as a CUDA graph on the first graph run. line_search (default): the update takes the
    first of the steps t = 1, ½ that does not raise the objective, else none."""

    ARRAYS = {"parameters": 0, "echos": 1, "dT1": 2, "dT2": 3, "signal": 4, "gradient": 5, "step": 6,
              "scalars": 7}

    def __init__(self, context: Context, parameters: TissueParameters, sequence, trajectory, coils, data,
                 cg_iterations: int = 4, delta: float = 1e-4, method: str = "GemmFast", line_search: bool = True):
        c = _arr(context, coils, np.complex64)
        d = _arr(context, data, np.complex64)
        ptr = library().compas_b200_make_gauss_newton(context.ptr, parameters.ptr, sequence.ptr, trajectory.ptr,
                                                      c.ptr, d.ptr, int(cg_iterations), float(delta),
                                                      JACOBIAN_METHODS[method])
        super().__init__(ptr, (parameters, sequence, trajectory, c, d))
        self.context = context
        self.nvoxels = parameters.nvoxels
        self.shapes = {"parameters": (9, self.nvoxels), "echos": (sequence.nreadouts, self.nvoxels),
                       "dT1": (sequence.nreadouts, self.nvoxels), "dT2": (sequence.nreadouts, self.nvoxels),
                       "signal": tuple(d.shape), "gradient": (4, self.nvoxels), "step": (4, self.nvoxels),
                       "scalars": (8,)}
        if not line_search:
            self.set_line_search(False)

    def set_line_search(self, on: bool):
        if library().compas_b200_gauss_newton_set_line_search(self.ptr, int(bool(on))) != 0:
            _check(None, "compas_b200_gauss_newton_set_line_search!")

    def step_length(self) -> float:
        """Step length the line search took in the last iteration: 1, 0.5 or 0 (blocks)."""
        return float(self.array("scalars").to_numpy()[7])

    def run(self, graph: bool = True):
        """Enqueue one iteration on the context's stream."""
        if library().compas_b200_gauss_newton_run(self.ptr, int(bool(graph))) != 0:
            _check(None, "compas_b200_gauss_newton_run!")

    def array(self, name: str) -> CompasArray:
        ptr = library().compas_b200_gauss_newton_array(self.ptr, self.ARRAYS[name])
        _check(ptr, "compas_b200_gauss_newton_array!")
        real = name in ("parameters", "step", "scalars")
        return CompasArray(self.context, ptr, np.float32 if real else np.complex64, self.shapes[name])

    def objective(self) -> float:
        """‖y - s(p)‖² of the last iteration, before its update (blocks)."""
        return float(self.array("scalars").to_numpy()[0])

    def graph_kernels(self) -> int:
        return int(library().compas_b200_gauss_newton_graph_kernels(self.ptr))


class ServeEngine(_Object):
    """compas_b200_make_server: continuous-batching request loop on one GPU.

    submit() queues a reconstruction request (simulate -> signal -> residual against `data` and the
    gradient Jᴴ·r with finite-difference derivatives) and returns a ticket; wait() blocks for it.
    Requests are admitted by estimated device footprint against the memory budget, run in
    batches (persistent work-queue simulations, batched signals) on up to
    `max_inflight_batches` streams at once, and give the same bits as the one-request calls."""

    STATS = ("completed", "failed", "batches", "echo_cache_hits", "p50_ms", "p99_ms", "mean_ms", "max_ms",
             "peak_bytes", "max_concurrent_batches")

    def __init__(self, context: Context, memory_budget_gb: float = 150.0, max_inflight_batches: int = 4,
                 max_batch_requests: int = 16, echo_cache_gb: float = 16.0, method: str = "MatmulFast",
                 delta: float = 1e-4):
        ptr = library().compas_b200_make_server(context.ptr, float(memory_budget_gb), int(max_inflight_batches),
                                                int(max_batch_requests), float(echo_cache_gb),
                                                SIGNAL_METHODS[method], float(delta))
        super().__init__(ptr)
        self.context = context
        self._meta = {}

    def submit(self, parameters: TissueParameters, sequence, trajectory, coils, data, echo_key: int = 0,
               inject_wait_timeout: bool = False) -> int:
        """Queue a request. inject_wait_timeout (a test hook of the failure path) makes the batch
        that runs it also run a kernel whose bounded wait gives up, so that batch's requests fail."""
        c = _arr(self.context, coils, np.complex64)
        d = _arr(self.context, data, np.complex64)
        t = library().compas_b200_server_submit_flags(self.ptr, parameters.ptr, sequence.ptr, trajectory.ptr, c.ptr,
                                                      d.ptr, int(echo_key), 1 if inject_wait_timeout else 0)
        if t < 0:
            _check(None, "compas_b200_server_submit!")
        self._meta[t] = (tuple(d.shape), parameters.nvoxels, isinstance(trajectory, CartesianTrajectory))
        return int(t)

    def wait(self, ticket: int) -> dict:
        obj = C.c_float()
        times = (C.c_double * 3)()
        batch = C.c_int()
        if library().compas_b200_server_wait(self.ptr, int(ticket), C.byref(obj), times, C.byref(batch)) != 0:
            _check(None, "compas_b200_server_wait!")
        return {"objective": obj.value, "queued_ms": times[0], "device_ms": times[1], "latency_ms": times[2],
                "batch": batch.value}

    def result(self, ticket: int, which: str = "residual") -> CompasArray:
        shape, nv, _ = self._meta[int(ticket)]
        idx = {"residual": 0, "gradient": 1}[which]
        ptr = library().compas_b200_server_result(self.ptr, int(ticket), idx)
        return _result(ptr, self.context, shape if idx == 0 else (4, nv), "compas_b200_server_result")

    def release(self, ticket: int):
        self._meta.pop(int(ticket), None)
        if library().compas_b200_server_release(self.ptr, int(ticket)) != 0:
            _check(None, "compas_b200_server_release!")

    def drain(self):
        if library().compas_b200_server_drain(self.ptr) != 0:
            _check(None, "compas_b200_server_drain!")

    def stats(self) -> dict:
        out = (C.c_double * len(self.STATS))()
        n = library().compas_b200_server_stats(self.ptr, out, len(self.STATS))
        if n < 0:
            _check(None, "compas_b200_server_stats!")
        return {k: out[i] for i, k in enumerate(self.STATS[:n])}

    def reset_stats(self):
        library().compas_b200_server_reset_stats(self.ptr)


def bfloat16_bits(x) -> np.ndarray:
    """float values -> bfloat16 bit patterns (uint16), rounded to nearest even."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bfloat16_values(bits) -> np.ndarray:
    """bfloat16 bit patterns (uint16) -> float32 values."""
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32)


GEMM_METHODS = {"Pedantic": 0, "Regular": 1, "Fast": 2}


def compute_gemm(context: Context, result: CompasArray, lhs: CompasArray, rhs: CompasArray, alpha: float = 1.0,
                 beta: float = 0.0, method: str = "Regular") -> CompasArray:
    """result = alpha·lhs·rhsᵀ + beta·result in place (compas/utils/gemm.h): float [m][n] result,
    float or bfloat16 [m][k] / [n][k] operands."""
    if library().compas_b200_compute_gemm(context.ptr, result.ptr, lhs.ptr, rhs.ptr, float(alpha), float(beta),
                                          GEMM_METHODS[method]) != 0:
        _check(None, "compas_b200_compute_gemm!")
    return result


def compute_complex_gemm(context: Context, result: CompasArray, lhs: CompasArray, rhs: CompasArray,
                         alpha: float = 1.0, beta: float = 0.0, method: str = "Regular") -> CompasArray:
    """The complex form on planar [2][rows][cols] arrays (plane 0 real, plane 1 imaginary)."""
    if library().compas_b200_compute_complex_gemm(context.ptr, result.ptr, lhs.ptr, rhs.ptr, float(alpha),
                                                  float(beta), GEMM_METHODS[method]) != 0:
        _check(None, "compas_b200_compute_complex_gemm!")
    return result


def convert_complex_to_planar(context: Context, x, bfloat16: bool = False) -> CompasArray:
    """complex [n][m] -> planar [2][n][m] (float32, or bfloat16 when `bfloat16`)."""
    src = _arr(context, x, np.complex64)
    shape = (2,) + src.shape
    out = (CompasArray.from_bfloat16(context, np.zeros(shape, np.float32)) if bfloat16
           else CompasArray.from_numpy(context, np.zeros(shape, np.float32)))
    if library().compas_b200_convert_complex_to_planar(context.ptr, out.ptr, src.ptr) != 0:
        _check(None, "compas_b200_convert_complex_to_planar!")
    return out


def convert_planar_to_complex(context: Context, x) -> CompasArray:
    """planar float [2][n][m] -> complex [n][m]."""
    src = _arr(context, x, np.float32)
    out = CompasArray.from_numpy(context, np.zeros(src.shape[1:], np.complex64))
    if library().compas_b200_convert_planar_to_complex(context.ptr, out.ptr, src.ptr) != 0:
        _check(None, "compas_b200_convert_planar_to_complex!")
    return out


def voxel_shard(nvoxels: int, rank: int, world: int) -> tuple:
    """Voxels [begin, end) of `rank` among `world` ranks (the library's partition: contiguous,
    sizes differ by at most one). Host-only: needs no GPU."""
    b, e = C.c_int64(), C.c_int64()
    if library().compas_b200_voxel_shard(int(nvoxels), int(rank), int(world), C.byref(b), C.byref(e)) != 0:
        _check(None, "compas_b200_voxel_shard")
    return b.value, e.value


def comm_unique_id() -> bytes:
    """A new NCCL unique id (128 bytes): one rank makes it, every rank passes it to Communicator."""
    buf = C.create_string_buffer(128)
    if library().compas_b200_comm_unique_id(buf, 128) != 128:
        _check(None, "compas_b200_comm_unique_id")
    return buf.raw


class Communicator(_Object):
    """compas_b200_make_communicator: the library's NCCL communicator over `world` processes, one
    GPU each (blocks until every rank has joined with the same unique id)."""

    def __init__(self, context: Context, rank: int, world: int, unique_id: bytes):
        if len(unique_id) != 128:
            raise CompasError("an NCCL unique id has 128 bytes")
        ptr = library().compas_b200_make_communicator(context.ptr, int(rank), int(world), bytes(unique_id))
        super().__init__(ptr)
        _check(ptr, "compas_b200_make_communicator!")
        self.context, self.rank, self.world = context, int(rank), int(world)

    def allreduce_sum(self, array: CompasArray) -> CompasArray:
        """In-place sum of a library array over the ranks (ordered on the context's stream)."""
        if library().compas_b200_allreduce_sum(self.context.ptr, self.ptr, array.ptr) != 0:
            _check(None, "compas_b200_allreduce_sum!")
        return array


def magnetization_to_signal_sharded(context: Context, comm: Communicator, echos, parameters: TissueParameters,
                                    trajectory, coils, method: str = "MatmulFast") -> CompasArray:
    """Full signal of a slice whose voxels are sharded over the communicator's ranks: this rank's
    echoes [R][V_rank], parameters and coils; the ranks' partials are summed by NCCL."""
    e = _arr(context, echos, np.complex64)
    c = _arr(context, coils, np.complex64)
    ptr = library().compas_b200_magnetization_to_signal_sharded(context.ptr, comm.ptr, e.ptr, parameters.ptr,
                                                                trajectory.ptr, c.ptr, SIGNAL_METHODS[method])
    return _result(ptr, context, (c.shape[0], trajectory.nreadouts, trajectory.samples_per_readout),
                   "magnetization_to_signal_sharded")


def compute_jacobian_sharded(context: Context, comm: Communicator, echos, dechos: dict, parameters: TissueParameters,
                             trajectory, coils, v, method: str = "GemmFast") -> CompasArray:
    """J·v of a slice whose voxels are sharded over the ranks (this rank's voxels in, full sum out)."""
    e, d1, d2 = (_arr(context, a, np.complex64) for a in (echos, dechos["T1"], dechos["T2"]))
    c = _arr(context, coils, np.complex64)
    vv = _arr(context, v, np.complex64)
    ptr = library().compas_b200_compute_jacobian_sharded(context.ptr, comm.ptr, e.ptr, d1.ptr, d2.ptr, parameters.ptr,
                                                         trajectory.ptr, c.ptr, vv.ptr, JACOBIAN_METHODS[method])
    return _result(ptr, context, (c.shape[0], trajectory.nreadouts, trajectory.samples_per_readout),
                   "compute_jacobian_sharded")


def wait_probe(context: Context, limit_cycles: int = 2_000_000):
    """Enqueue the failure-channel self-test: a kernel whose bounded wait on a barrier nobody
    completes gives up after `limit_cycles` SM cycles; the next synchronize raises CompasError."""
    if library().compas_b200_wait_probe(context.ptr, int(limit_cycles)) != 0:
        _check(None, "compas_b200_wait_probe")


def launch_count() -> int:
    """Kernels launched by libcompas_b200.so so far in this process."""
    return int(library().compas_b200_launch_count())


def set_fisp_launch(config: int = -1, warps: int = -1):
    library().compas_b200_set_fisp_launch(int(config), int(warps))
    _check()


def set_fisp_tangent_launch(config: int = -1):
    library().compas_b200_set_fisp_tangent_launch(int(config))
    _check()


def fisp_tangent_configs() -> list:
    lib = library()
    out = []
    for i in range(lib.compas_b200_fisp_tangent_config_count()):
        k, g = C.c_int(), C.c_int()
        lib.compas_b200_fisp_tangent_config_info(i, C.byref(k), C.byref(g))
        out.append((k.value, g.value))
    return out


def set_pssfp_launch(config: int = -1):
    library().compas_b200_set_pssfp_launch(int(config))
    _check()


def fisp_configs() -> list:
    lib = library()
    out = []
    for i in range(lib.compas_b200_fisp_config_count()):
        k, g = C.c_int(), C.c_int()
        lib.compas_b200_fisp_config_info(i, C.byref(k), C.byref(g))
        out.append((k.value, g.value))
    return out


def fisp_tangent_config_packed(index: int) -> bool:
    """Whether FISP tangent layout `index` is packed (value and tangents as pairs of states)."""
    return bool(library().compas_b200_fisp_tangent_config_packed(int(index)))


def fisp_config_packed(index: int) -> bool:
    """Whether FISP layout `index` is packed (two states per two-wide FP32 instruction)."""
    return bool(library().compas_b200_fisp_config_packed(int(index)))


def pssfp_config_packed(index: int) -> bool:
    """Whether pSSFP layout `index` is packed (two isochromats per two-wide FP32 instruction)."""
    return bool(library().compas_b200_pssfp_config_packed(int(index)))


def fisp_launch_choice(max_state: int, nvoxels: int, npositions: int) -> tuple:
    """(layout index, warps) a FISP simulation of this shape runs with."""
    cfg, w = C.c_int(), C.c_int()
    library().compas_b200_fisp_launch_choice(int(max_state), int(nvoxels), int(npositions), C.byref(cfg), C.byref(w))
    return cfg.value, w.value


def pssfp_launch_choice(nz: int, nvoxels: int) -> int:
    return int(library().compas_b200_pssfp_launch_choice(int(nz), int(nvoxels)))


# tensor-core contraction kinds (COMPAS_B200_TC_* in compas_b200.h)
TC_KINDS = {"cartesian_signal": 0, "cartesian_jacobian": 1, "cartesian_hermitian": 2,
            "spiral_signal": 3, "spiral_jacobian": 4, "spiral_hermitian": 5}


def _tc_kind(kind) -> int:
    return TC_KINDS[kind] if isinstance(kind, str) else int(kind)


def set_tc_launch(kind, tile: int = 0, splits: int = 0):
    """Override the readout tile (Cartesian signal / J·v; a multiple of 16 in [16, 256]) and the
    split count of one tensor-core contraction kind; 0 keeps the tuning table's or built-in choice."""
    library().compas_b200_set_tc_launch(_tc_kind(kind), int(tile), int(splits))
    _check()


def tc_launch_choice(kind, nvoxels: int, nreadouts: int, samples_per_readout: int, ncoils: int,
                     device: int = 0) -> tuple:
    """(tile, splits) a tensor-core contraction of this shape runs with (tile 0 where the kind has none)."""
    tile, splits = C.c_int(), C.c_int()
    rc = library().compas_b200_tc_launch_choice(_tc_kind(kind), int(device), int(nvoxels), int(nreadouts),
                                                int(samples_per_readout), int(ncoils), C.byref(tile),
                                                C.byref(splits))
    if rc != 0:
        _check()
        raise CompasError("compas_b200_tc_launch_choice failed")
    return tile.value, splits.value


def pssfp_configs() -> list:
    lib = library()
    out = []
    for i in range(lib.compas_b200_pssfp_config_count()):
        k, g = C.c_int(), C.c_int()
        lib.compas_b200_pssfp_config_info(i, C.byref(k), C.byref(g))
        out.append((k.value, g.value))
    return out
