"""ctypes binding of libwnfea_cuda.so (the C ABI in include/wnfea_cuda.h).

Mirrors the reference's loader (``_get_hip_lib``, wnfea/solver/fast_kernels.py:96-222):
argtypes/restype are declared once, and a non-zero status raises ``RuntimeError`` with the
library's message (as fast_kernels.py:590-591, 660-661).  Unlike the reference there is no
silent CPU fallback: a missing library raises at first use.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_P = C.c_void_p
_I = C.c_int
_I64 = C.c_int64
_D = C.c_double
_F = C.c_float
_U = C.c_uint64  # uintptr_t stream

class AmgParams(C.Structure):
    """wn_amg_params"""

    _fields_ = [
        ("strength_theta", C.c_double),
        ("max_levels", C.c_int),
        ("coarse_size", C.c_int),
        ("smoother_degree", C.c_int),
        ("cheb_lower", C.c_double),
        ("cheb_safety", C.c_double),
        ("prolong_omega", C.c_double),
        ("smooth_prolongator", C.c_int),
        ("power_iters", C.c_int),
        ("stream_min_mb", C.c_double),
        ("setup_on_device", C.c_int),
        ("coarse_block_smoother", C.c_int),
    ]


class SolveParams(C.Structure):
    """wn_solve_params"""

    _fields_ = [
        ("rtol", C.c_double),
        ("max_iter", C.c_int),
        ("precond", C.c_int),
        ("precision", C.c_int),
        ("inner_rtol", C.c_double),
        ("max_outer", C.c_int),
        ("chunk", C.c_int),
        ("use_graph", C.c_int),
        ("profile", C.c_int),
    ]


class SolveStats(C.Structure):
    """wn_solve_stats"""

    _fields_ = [
        ("iterations", C.c_int),
        ("outer_iterations", C.c_int),
        ("status", C.c_int),
        ("n_levels", C.c_int),
        ("rel_res", C.c_double),
        ("solve_seconds", C.c_double),
        ("setup_seconds", C.c_double),
        ("kernel_launches", C.c_int64),
        ("algorithmic_bytes", C.c_double),
    ]


_PI = C.POINTER(C.c_int)
_PI64 = C.POINTER(C.c_int64)
_PD = C.POINTER(C.c_double)

# name -> (restype, argtypes); must match include/wnfea_cuda.h
SIGNATURES: dict[str, tuple] = {
    "wn_last_error_string": (C.c_char_p, []),
    "wn_version": (_I, []),
    "wn_device_synchronize": (_I, []),
    "wn_solid_create": (_I, [_I64, _I64, _P, _P, C.POINTER(_P)]),
    "wn_solid_destroy": (_I, [_P]),
    "wn_solid_info": (_I, [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I64)]),
    "wn_solid_get_pattern": (_I, [_P, _P, _P]),
    "wn_solid_get_map": (_I, [_P, _P]),
    "wn_bsr3_pattern_host": (_I, [_I64, _I64, _P, C.POINTER(_I64), _P, _P, _P]),
    "wn_solid_set_fixed": (_I, [_P, _P]),
    "wn_assemble_c3d10": (_I, [_P, _P, _I]),
    "wn_assemble_c3d10_device": (_I, [_P, _P, _I, _U]),
    "wn_solid_get_values": (_I, [_P, _P]),
    "wn_solid_device_arrays": (_I, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "wn_spmv_solid_device": (_I, [_P, _I, _P, _P, _U]),
    "wn_solid_set_stream": (_I, [_P, _I]),
    "wn_solid_set_batch_staging": (_I, [_P, _I]),
    "wn_solid_stream_status": (_I, [_P, _I, _PI]),
    "wn_assembly_plan_host": (_I, [_I64, _I64, _P, C.POINTER(_I64), _PI, C.POINTER(_I64), _P, _P, _P, _P, _P]),
    "wn_assembly_chunks_host": (_I, [_I64, _I64, _P, _PI, _PI, C.POINTER(_I64), _P, _P, _P]),
    "wn_solid_stream_test_hook": (_I, [_P, _I64, _I]),
    "wn_stream_tiles_host": (_I, [_I64, _P, _P, _I64, C.POINTER(_I64)]),
    "wn_spmv_bsr_f64_device": (_I, [_I, _I, _I64, _P, _P, _P, _P, _P, _D, _D, _U]),
    "wn_spmv_bsr_f32_device": (_I, [_I, _I, _I64, _P, _P, _P, _P, _P, _F, _F, _U]),
    "wn_spmv_bsr_f64": (_I, [_I, _I, _I64, _I64, _I64, _P, _P, _P, _P, _P, _D, _D]),
    "wn_c3d10_element_stiffness": (_I, [_I64, _P, _P, _P]),
    "wn_c3d10_element_stresses": (_I, [_I64, _P, _P, _P, _P, _P]),
    "wn_c3d10_element_stiffness_noalloc": (_I, [_I64, _I64, _P, _P, _P, _P, _U]),
    "wn_c3d10_internal_forces": (_I, [_P, _P, _P, _P, _P, _I, _I]),
    "wn_fint_c3d10_device": (_I, [_P, _P, _P, _U]),
    "wn_fint_c3d10": (_I, [_P, _P, _P]),
    "wn_stress_c3d10": (_I, [_P, _P, _P, _P, _P]),
    "wn_stress_c3d10_device": (_I, [_P, _P, _P, _P, _P, _U]),
    "wn_adjoint_compliance_device": (_I, [_P, _P, _P, _P, _U]),
    "wn_adjoint_compliance": (_I, [_P, _P, _P, _P]),
    "wn_amg_default_params": (_I, [C.POINTER(AmgParams)]),
    "wn_amg_setup": (_I, [_P, C.POINTER(AmgParams)]),
    "wn_amg_vcycle_device": (_I, [_P, _I, _P, _P, _U]),
    "wn_amg_info": (_I, [_P, _PI, _PI, _PI64, _PI64, _PI64, _PD]),
    "wn_amg_level_matrix": (_I, [_P, _I, _I, _PI, _PI, _PI64, _PI64, _PI64, _P, _P, _P]),
    "wn_amg_level_data": (_I, [_P, _I, _PD, _P]),
    "wn_amg_coarse": (_I, [_P, _PI64, _P, _P]),
    "wn_amg_setup_host": (_I, [_I64, _P, _P, _P, _P, _P, C.POINTER(AmgParams), C.POINTER(_P)]),
    "wn_amg_host_destroy": (_I, [_P]),
    "wn_amg_host_level_matrix": (_I, [_P, _I, _I, _PI, _PI, _PI64, _PI64, _PI64, _P, _P, _P]),
    "wn_amg_host_level_data": (_I, [_P, _I, _PD, _P, _PI64, _PI]),
    "wn_amg_host_coarse": (_I, [_P, _PI64, _P, _P]),
    "wn_solve_device": (_I, [_P, _P, _P, C.POINTER(SolveParams), C.POINTER(SolveStats), _U]),
    "wn_solve": (_I, [_P, _P, _P, C.POINTER(SolveParams), C.POINTER(SolveStats)]),
    "wn_solve_profile": (_I, [_P, _I, _PI, _P, _P, _P, _P]),
    "wn_bsr6_system_create": (_I, [_I64, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    "wn_beam_linear_system": (_I, [_P, C.POINTER(_P)]),
    "wn_solve_multi_device": (_I, [_P, _I, _P, _P, C.POINTER(SolveParams), C.POINTER(SolveStats), _P, _P, _U]),
    "wn_solve_multi": (_I, [_P, _I, _P, _P, C.POINTER(SolveParams), C.POINTER(SolveStats), _P, _P]),
    "wn_beam_internal_forces": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I]),
    "wn_beam_create": (_I, [_I64, _I64, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    "wn_beam_destroy": (_I, [_P]),
    "wn_beam_info": (_I, [_P, _PI64, _PI64, _PI64]),
    "wn_beam_get_pattern": (_I, [_P, _P, _P]),
    "wn_beam_set_fixed": (_I, [_P, _P]),
    "wn_beam_evaluate_device": (_I, [_P, _P, _P, _I, _I, _U]),
    "wn_beam_evaluate": (_I, [_P, _P, _P, _I, _I]),
    "wn_beam_get_tangent": (_I, [_P, _P]),
    "wn_beam_solve_device": (_I, [_P, _P, _P, _I, _D, _I, _PI, _PD, _U]),
    "wn_beam_solve": (_I, [_P, _P, _P, _I, _D, _I, _PI, _PD]),
}

LIB_PATH = Path(__file__).resolve().parent / "libwnfea_cuda.so"
_LIB = None


def lib():
    """Load (once) and return the library; raises if it is missing or incomplete."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = Path(os.environ.get("WNFEA_CUDA_LIB", LIB_PATH))
    if not path.exists():
        raise RuntimeError(
            f"libwnfea_cuda.so not found at {path}; build it with `python -m wnfea_b200.csrc.build` "
            "(this package has no CPU fallback)"
        )
    handle = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = handle
    return handle


def last_error() -> str:
    msg = lib().wn_last_error_string()
    return msg.decode() if msg else ""


class WnError(RuntimeError):
    """A non-zero status from libwnfea_cuda."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


def call(name: str, *args) -> None:
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise WnError(name, rc, last_error())


def ptr(a: np.ndarray | None):
    """Host pointer of a C-contiguous array (None -> NULL)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(C.c_void_p)


def dptr(t) -> int | None:
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else t.data_ptr()
