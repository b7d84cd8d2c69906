"""ctypes wrapper of the C restatement oracle/c/bbt_oracle.c (test
infrastructure): exact block-bordered LU of A - sigma B on the host, with
the ``.solve(b)`` interface the reference's preconditioner argument expects
(reference bbjd.py:125-127, 208-219)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle_bbt.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            subprocess.run(["make", "-s", "-C", _HERE, "c"], check=True)
        lib = C.CDLL(_SO)
        lib.bbt_lu_factor.restype = C.c_void_p
        lib.bbt_lu_factor.argtypes = [C.c_int64] * 3 + [C.c_void_p] * 6 + [C.c_double, C.c_double]
        lib.bbt_lu_solve.restype = C.c_int
        lib.bbt_lu_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.bbt_lu_free.argtypes = [C.c_void_p]
        _lib = lib
    return _lib


class BBTLUHost:
    """Exact LU of A - sigma B for a BBTPencil, factored on the CPU."""

    def __init__(self, pencil, sigma: complex):
        if pencil.b > 128 or pencil.t > 256:
            raise ValueError("block size <= 128 and t <= 256")
        lib = _load()
        s = complex(sigma)
        arr = [np.ascontiguousarray(a, dtype=np.complex128)
               for a in (pencil.Ad, pencil.Al, pencil.Au, pencil.Bd)]
        E = np.ascontiguousarray(pencil.E, dtype=np.complex128)
        F = np.ascontiguousarray(pencil.F, dtype=np.complex128)
        self._keep = arr + [E, F]
        h = lib.bbt_lu_factor(pencil.b, pencil.nblk, pencil.t, *[a.ctypes.data for a in arr[:3]],
                              arr[3].ctypes.data, E.ctypes.data if pencil.t else None,
                              F.ctypes.data if pencil.t else None, s.real, s.imag)
        if not h:
            raise np.linalg.LinAlgError("singular pivot in the block-bordered LU")
        self._h = h
        self.n = pencil.n
        self._lib = lib

    def solve(self, b):
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = np.empty_like(b)
        if self._lib.bbt_lu_solve(self._h, b.ctypes.data, x.ctypes.data) != 0:
            raise MemoryError("bbt_lu_solve")
        return x

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.bbt_lu_free(self._h)
            self._h = None


class BlockJacobiHost:
    """Block-Jacobi preconditioner of A - sigma B for a BBTPencil on the host
    (test infrastructure): the inverses of the interior diagonal blocks
    Ad_j - sigma Bd_j and of the t x t tau corner of A (B's tau rows are
    zero), with the ``.solve(b)`` interface of the reference's
    preconditioner argument (reference bbjd.py:125-127).  The same operator
    as the device's block Jacobi."""

    def __init__(self, pencil, sigma: complex):
        s = complex(sigma)
        self.b, self.nblk, self.nb, self.n = pencil.b, pencil.nblk, pencil.nb, pencil.n
        self.Dinv = np.linalg.inv(pencil.Ad - s * pencil.Bd)
        self.Ginv = np.linalg.inv(pencil.F[:, pencil.nb:]) if pencil.t else None

    def solve(self, r):
        r = np.asarray(r, dtype=np.complex128)
        x = np.empty_like(r)
        x[:self.nb] = np.einsum("jic,jc->ji", self.Dinv,
                                r[:self.nb].reshape(self.nblk, self.b)).reshape(-1)
        if self.Ginv is not None:
            x[self.nb:] = self.Ginv @ r[self.nb:]
        return x
