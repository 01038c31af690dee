"""ctypes binding of ``libsawsim_b200.so`` (the C ABI in include/sawsim_b200.h).

The library is built in-tree by ``sawsim_b200/build.py``.  There is no CPU
fallback: if the library is missing or no CUDA device is present, the calls
below raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / 'libsawsim_b200.so'

SS_OK, SS_EINVAL, SS_ECUDA, SS_ESINGULAR, SS_ENOCONV, SS_ETIMEOUT, SS_ENOMEM, SS_ESTATE = 0, -1, -2, -3, -4, -5, -6, -7
SS_Q9_ME0, SS_Q9_ME1, SS_HEX27, SS_MATRIX = 0, 1, 2, 3
SS_PREC_FP64, SS_PREC_MIXED, SS_PREC_AUTO = 0, 1, 2
SS_MAT_K, SS_MAT_M, SS_MAT_D, SS_MAT_KC, SS_MAT_MC = 0, 1, 2, 3, 4

STATUS_NAMES = {0: 'ok', -1: 'invalid argument', -2: 'CUDA error', -3: 'singular', -4: 'no convergence',
                -5: 'timeout', -6: 'out of device memory', -7: 'call out of order'}

_P = C.c_void_p
_I64P = C.POINTER(C.c_int64)
_I32P = C.POINTER(C.c_int32)
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)

# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ('ss_create', C.c_int, [C.POINTER(_P), C.c_int]),
    ('ss_destroy', None, [_P]),
    ('ss_last_error', C.c_char_p, [_P]),
    ('ss_set_mesh', C.c_int, [_P, C.c_int, C.c_int64, _DP, C.c_int64, _I64P, _I32P]),
    ('ss_set_materials', C.c_int, [_P, C.c_int, C.c_int, _DP, _DP, _DP, _DP]),
    ('ss_set_pml', C.c_int, [_P, C.c_int, _I32P, _DP, _I32P, _DP, _DP, C.c_int, _I32P, C.c_double]),
    ('ss_set_bc', C.c_int, [_P, C.c_int64, C.c_int64, _I64P, C.c_int64, _I64P, C.c_int64, _I64P, C.c_int64,
                            _I64P, _I64P, C.c_int64]),
    ('ss_assemble', C.c_int, [_P]),
    ('ss_set_csr', C.c_int, [_P, C.c_int64, _I64P, _I64P, C.c_int64, C.c_int, _I64P, _DP]),
    ('ss_set_values', C.c_int, [_P, C.c_int, _DP]),
    ('ss_export_csr', C.c_int, [_P, C.c_int, _I64P, _I64P, _I64P, _I64P, _DP]),
    ('ss_analyze', C.c_int, [_P]),
    ('ss_set_damping', C.c_int, [_P, C.c_double]),
    ('ss_sweep', C.c_int, [_P, C.c_int, _DP, C.c_double, C.c_int, _DP, _IP, _IP]),
    ('ss_solve_fields', C.c_int, [_P, C.c_double, C.c_double, _DP, _DP]),
    ('ss_solve_adjoint', C.c_int, [_P, C.c_double, C.c_int, _DP]),
    ('ss_adjoint_gradient', C.c_int, [_P, C.c_int, _DP, C.c_double, C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP,
                                      _DP, _DP, _DP, _IP]),
    ('ss_stats', C.c_int, [_P, _DP, C.c_int]),
    ('ss_set_option', C.c_int, [_P, C.c_char_p, C.c_double]),
    ('ss_measure_gemm_ceiling', C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _DP]),
    ('ss_analyze_host', C.c_int, [C.c_int, C.c_int64, _DP, C.c_int64, _I64P, C.c_int64, C.c_int64, _I64P, C.c_int64,
                                  _I64P, C.c_int64, _I64P, C.c_int64, _I64P, _I64P, C.c_int64, _I64P, _DP, _I64P,
                                  _I64P, _I32P, _I32P, _I32P, _I32P, _I64P, _I64P]),
    ('ss_analyze_host_csr', C.c_int, [C.c_int64, _I64P, _I64P, C.c_int64, C.c_int, _I64P, _DP, C.c_int64, _I64P,
                                      C.c_int64, _I64P, C.c_int64, _I64P, C.c_int64, _I64P, _I64P, C.c_int64, _I64P,
                                      _DP, _I64P, _I64P, _I32P, _I32P, _I32P, _I32P, _I64P, _I64P]),
    ('ss_assemble_q9_noalloc', C.c_int, [C.c_int, C.c_int64, _P, C.c_int64, _P, _P, _P, _P, _P, _P, C.c_int, _P, _P,
                                         _P, _P, _P, _P, C.c_double, _P, _P, _P, C.c_int64, _P, _P, _P]),
]

_lib = None


def load() -> C.CDLL:
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f'{LIB_PATH.name} is not built; run `python -m sawsim_b200.build` '
                               '(the sweep has no CPU fallback)')
        lib = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


class SawsimError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f'{STATUS_NAMES.get(code, code)}: {msg}')
        self.code = code


def ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def cplx(a) -> np.ndarray:
    """complex array -> interleaved float64 view."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.view(np.float64)
