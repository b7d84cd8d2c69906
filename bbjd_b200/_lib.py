"""ctypes binding of libbbjd_gpu.so (the C-ABI declared in include/bbjd.h
and include/bbjd_gpu.h).

The structs below mirror the C layouts field by field; ``complex`` values
are a pair of doubles, which the x86-64 calling convention passes and lays
out exactly like C's ``double complex``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libbbjd_gpu.so")


class zcomplex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]

    @classmethod
    def of(cls, z) -> "zcomplex":
        z = complex(z)
        return cls(z.real, z.imag)

    def value(self) -> complex:
        return complex(self.re, self.im)


bbjd_int = C.c_int64
zptr = C.POINTER(zcomplex)
MATVEC_FN = C.CFUNCTYPE(C.c_int, bbjd_int, C.c_void_p, C.c_void_p, C.c_void_p)


class Params(C.Structure):
    _fields_ = [
        ("n", bbjd_int), ("nev", bbjd_int), ("sigma", zcomplex), ("target", C.c_int),
        ("maxsub", bbjd_int), ("minsub", bbjd_int), ("tol", C.c_double), ("maxiter", bbjd_int),
        ("inner_maxiter", bbjd_int), ("inner_tol", C.c_double), ("v0", C.c_void_p),
        ("matvec_A", MATVEC_FN), ("matvec_B", MATVEC_FN), ("precond", MATVEC_FN),
        ("op_data", C.c_void_p), ("verbose", C.c_int),
    ]


class Result(C.Structure):
    _fields_ = [
        ("nconv", bbjd_int), ("eigenvalues", C.c_void_p), ("eigenvectors", C.c_void_p),
        ("residuals", C.POINTER(C.c_double)), ("iters", bbjd_int), ("status", C.c_int),
    ]


class Workspace(C.Structure):
    _fields_ = [
        ("n", bbjd_int), ("maxsub", bbjd_int), ("nev", bbjd_int),
        ("V", C.c_void_p), ("W", C.c_void_p), ("AV", C.c_void_p), ("BV", C.c_void_p),
        ("MA", C.c_void_p), ("MB", C.c_void_p), ("SA", C.c_void_p), ("SB", C.c_void_p),
        ("ZA", C.c_void_p), ("ZB", C.c_void_p), ("nlock", bbjd_int), ("kdim", bbjd_int),
        ("gmres_V", C.c_void_p), ("gmres_H", C.c_void_p), ("gmres_cs", C.c_void_p),
        ("gmres_sn", C.c_void_p), ("gmres_g", C.c_void_p), ("inner_maxiter", bbjd_int),
        ("tmp1", C.c_void_p), ("tmp2", C.c_void_p), ("tmp3", C.c_void_p), ("tmp4", C.c_void_p),
        ("swap_nm", C.c_void_p), ("Q_right", C.c_void_p), ("Q_left", C.c_void_p),
        ("h_work", C.c_void_p),
    ]


class DeviceExt(C.Structure):
    _fields_ = [
        ("precision", C.c_int), ("record_timing", C.c_int), ("projected", C.c_int),
        ("lock_rule", C.c_int), ("lock_rel", C.c_double), ("stream", C.c_void_p),
        ("evec_layout", C.c_int), ("ritz_estimate", C.c_int), ("host_overlap", C.c_int),
        ("conv_iters", C.c_void_p), ("seconds_total", C.c_double),
        ("seconds_qz", C.c_double), ("seconds_device", C.c_double),
        ("seconds_restart", C.c_double), ("bytes_device", C.c_double),
        ("kernel_launches", C.c_int64), ("dgks_passes", C.c_int64), ("restarts", C.c_int64),
        ("duplicates", C.c_int64), ("ritz_refinements", C.c_int64),
        ("ritz_fallbacks", C.c_int64), ("seconds_qz_exposed", C.c_double),
        ("guess_hits", C.c_int64), ("guess_misses", C.c_int64),
        ("kernel_ms", C.c_double * 8), ("kernel_bytes", C.c_double * 8),
        ("kernel_calls", C.c_int64 * 8),
    ]


KERNEL_CLASSES = ("spmv", "orth", "pencil", "ritz", "precond", "restart", "small", "gmres")

# every symbol include/*.h declares, with (restype, argtypes)
SIGNATURES = {
    "bbjd_params_init": (None, [C.POINTER(Params)]),
    "bbjd_workspace_alloc": (C.POINTER(Workspace), [C.POINTER(Params)]),
    "bbjd_workspace_free": (None, [C.POINTER(Workspace)]),
    "bbjd_solve": (C.c_int, [C.POINTER(Params), C.POINTER(Workspace), C.POINTER(Result)]),
    "bbjd_result_free": (None, [C.POINTER(Result)]),
    "bbjd_mgs_orthogonalize": (C.c_double, [bbjd_int, bbjd_int, C.c_void_p, C.c_void_p]),
    "bbjd_correction_gmres": (C.c_int, [bbjd_int, C.c_void_p, C.c_void_p, zcomplex, zcomplex,
                                        C.c_void_p, C.c_void_p, MATVEC_FN, MATVEC_FN, MATVEC_FN,
                                        C.c_void_p, bbjd_int, C.c_double, C.POINTER(Workspace)]),
    "bbjd_bbt_create": (C.c_int, [bbjd_int, bbjd_int, bbjd_int] + [C.c_void_p] * 6 +
                        [C.c_int, C.POINTER(C.c_void_p)]),
    "bbjd_bbt_free": (None, [C.c_void_p]),
    "bbjd_bbt_n": (bbjd_int, [C.c_void_p]),
    "bbjd_bbt_matvec_bytes": (C.c_double, [C.c_void_p]),
    "bbjd_bbt_matvec": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bbjd_precond_create": (C.c_int, [C.c_void_p, zcomplex, C.c_int, C.c_int,
                                      C.POINTER(C.c_void_p)]),
    "bbjd_precond_free": (None, [C.c_void_p]),
    "bbjd_precond_solve_bytes": (C.c_double, [C.c_void_p, C.c_int]),
    "bbjd_precond_factor_seconds": (C.c_double, [C.c_void_p]),
    "bbjd_precond_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bbjd_device_ext_init": (None, [C.POINTER(DeviceExt)]),
    "bbjd_solve_device": (C.c_int, [C.POINTER(Params), C.POINTER(DeviceExt), C.c_void_p,
                                    C.c_void_p, C.POINTER(Workspace), C.POINTER(Result)]),
    "bbjd_solve_batch": (C.c_int, [C.c_int, C.POINTER(Params), C.POINTER(DeviceExt),
                                   C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                   C.POINTER(C.POINTER(Workspace)), C.POINTER(Result), C.c_int]),
    "bbjd_dev_orthogonalize": (C.c_int, [bbjd_int, bbjd_int, C.c_void_p, bbjd_int, C.c_void_p,
                                         C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p]),
    "bbjd_dev_orthogonalize_static": (C.c_int, [bbjd_int, bbjd_int, C.c_void_p, bbjd_int,
                                                C.c_void_p, C.POINTER(C.c_double),
                                                C.POINTER(C.c_int), C.c_void_p]),
    "bbjd_dev_restart_gemm": (C.c_int, [bbjd_int, bbjd_int, bbjd_int, C.c_void_p, bbjd_int,
                                        C.c_void_p, bbjd_int, C.c_void_p, C.c_void_p]),
    "bbjd_dev_restart_gemm_stalled": (C.c_int, [bbjd_int, bbjd_int, bbjd_int, C.c_void_p, bbjd_int,
                                        C.c_void_p, bbjd_int, C.c_void_p, C.c_void_p]),
    "bbjd_dev_gram": (C.c_int, [bbjd_int, bbjd_int, C.c_void_p, C.c_void_p, bbjd_int,
                                C.c_void_p, bbjd_int, C.c_void_p]),
    "bbjd_gpu_version": (C.c_char_p, []),
}

_lib = None


def load(build_if_missing: bool = True):
    """Load libbbjd_gpu.so, building it first when it is absent.

    There is no CPU fallback: without the library every solver entry point
    raises.
    """
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) and build_if_missing:
        from . import build as _build
        _build.build()
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"bbjd_b200: CUDA library not built ({LIB_PATH}); "
                          "run `python -m bbjd_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data


STATUS_MSG = {
    -1: "memory allocation failed",
    -2: "invalid parameters",
    -3: "callback error (matvec or preconditioner failed)",
    -4: "LAPACK error in projected eigenproblem",
    -5: "subspace breakdown",
    -6: "CUDA error",
    -7: "device wait timed out",
}
