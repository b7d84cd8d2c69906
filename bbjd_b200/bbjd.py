"""jdqz(): the reference's Python entry point (reference bbjd.py:59-277) over
the B200 engine.

Same signature, defaults, validation, return values and error mapping as the
reference.  Two operator paths:

* **device path** -- ``A`` is a block-bordered pencil (:class:`BBTPencil` on
  the host or :class:`DevicePencil` already in HBM; ``B`` must then be
  ``None``, the pencil carries its own ``B``).  ``preconditioner`` is
  ``'exact'`` (device block-bordered LU of A - sigma B), ``'block_jacobi'``,
  a prebuilt :class:`DevicePreconditioner`, or ``None``.  The whole solve
  runs on the GPU except the k x k projected QZ.
* **callback path** -- anything the reference accepts (scipy sparse, dense
  arrays, LinearOperator) with a host ``.solve`` preconditioner.  The
  products run on the host through callbacks exactly as in the reference;
  the subspace work (orthogonalisation, projected pencil, restarts, Ritz
  vectors) runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np
import scipy.sparse as sp

from . import _lib
from .pencils import BBTPencil

# Target enum values (include/bbjd.h bbjd_target; reference bbjd.py:48-56)
_TARGET_MAP = {
    'nearest': 0,
    'LM': 1,
    'SM': 2,
    'LR': 3,
    'SR': 4,
    'LI': 5,
    'SI': 6,
}


class DevicePencil:
    """A block-bordered pencil resident on the current GPU (bbjd_bbt_create)."""

    def __init__(self, pencil: BBTPencil | None = None, *, arrays: dict | None = None,
                 b: int = 0, nblk: int = 0, t: int = 0):
        """Upload ``pencil`` (host layout), or ``arrays`` already in the
        C-ABI's column-major layout (``BBTPencil.device_arrays()``, e.g. in
        pinned memory) with their ``b``, ``nblk``, ``t``."""
        lib = _lib.load()
        if pencil is not None:
            pencil.validate()
            arrays = pencil.device_arrays()
            b, nblk, t = pencil.b, pencil.nblk, pencil.t
        elif arrays is None:
            raise ValueError("pass a BBTPencil or its device-layout arrays")
        else:
            nb, n = b * nblk, b * nblk + t
            want = {"Ad": nblk * b * b, "Al": nblk * b * b, "Au": nblk * b * b,
                    "Bd": nblk * b * b, "E": nb * t, "FT": n * t}
            for name, count in want.items():
                if name not in arrays:
                    if count:
                        raise ValueError(f"arrays lacks {name!r}")
                    continue
                a = arrays[name]
                if hasattr(a, "data_ptr"):
                    nbytes, contiguous = a.numel() * a.element_size(), a.is_contiguous()
                else:
                    nbytes, contiguous = a.nbytes, a.flags.c_contiguous or a.flags.f_contiguous
                if nbytes != 16 * count or not contiguous:
                    raise ValueError(f"{name!r} must be {count} contiguous complex128 values "
                                     f"({16 * count} bytes); got {nbytes} bytes"
                                     + ("" if contiguous else ", not contiguous"))
        addr = lambda a: a.data_ptr() if hasattr(a, "data_ptr") else _lib.ptr(a)  # noqa: E731
        h = C.c_void_p()
        st = lib.bbjd_bbt_create(b, nblk, t, addr(arrays["Ad"]), addr(arrays["Al"]),
                                 addr(arrays["Au"]), addr(arrays["E"]) if t else None,
                                 addr(arrays["FT"]) if t else None, addr(arrays["Bd"]), 1,
                                 C.byref(h))
        if st != 0:
            raise RuntimeError(f"bbjd_bbt_create failed: {_lib.STATUS_MSG.get(st, st)}")
        self.handle = h
        self.b, self.nblk, self.t = b, nblk, t
        self.n = nblk * b + t
        self.shape = (self.n, self.n)
        self._lib = lib

    def matvec_bytes(self) -> float:
        return self._lib.bbjd_bbt_matvec_bytes(self.handle)

    def close(self):
        if getattr(self, "handle", None):
            self._lib.bbjd_bbt_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DevicePreconditioner:
    """M^-1 for A - sigma B on the device: kind 'exact' (block-bordered LU)
    or 'block_jacobi'.  Factored once; reusable across solves."""

    KINDS = {"exact": 1, "lu": 1, "block_jacobi": 2}

    def __init__(self, pencil: DevicePencil, sigma: complex, kind: str = "exact",
                 precision: str = "fp64"):
        if kind not in self.KINDS:
            raise ValueError(f"preconditioner kind must be one of {list(self.KINDS)}")
        lib = _lib.load()
        h = C.c_void_p()
        st = lib.bbjd_precond_create(pencil.handle, _lib.zcomplex.of(sigma), self.KINDS[kind],
                                     0 if precision == "fp64" else 1, C.byref(h))
        if st != 0:
            raise RuntimeError(f"bbjd_precond_create failed: {_lib.STATUS_MSG.get(st, st)}")
        self.handle = h
        self.sigma = complex(sigma)
        self.kind = kind
        self.n = pencil.n
        self._lib = lib
        self._pencil = pencil  # the factors borrow the pencil's tau rows

    @property
    def factor_seconds(self) -> float:
        return self._lib.bbjd_precond_factor_seconds(self.handle)

    def solve_bytes(self, nrhs: int = 1) -> float:
        return self._lib.bbjd_precond_solve_bytes(self.handle, nrhs)

    def close(self):
        if getattr(self, "handle", None):
            self._lib.bbjd_precond_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SparseLU:
    """Device LU of a block-bordered sparse matrix, in the place of the
    sparse LU the reference's users build for ``A - sigma B`` (reference
    README.md:40-44: ``SparseLU(M, colamd=True, pin_dense_rows=True)``).

    ``M`` (scipy sparse or dense) must have the block-bordered form
    (:func:`bbjd_b200.structure.detect`); it is packed, uploaded and
    factored once by the device block-bordered LU, which needs no fill-
    reducing ordering and keeps the dense tau rows in a t x t Schur
    complement, so ``colamd`` and ``pin_dense_rows`` are accepted for
    compatibility and have no effect.  ``solve(b)`` takes and returns host
    arrays; passed as ``jdqz``'s preconditioner with a block-bordered
    ``A, B`` the factors are applied on the device directly.
    """

    def __init__(self, M, colamd: bool = True, pin_dense_rows: bool = True,
                 precision: str = "fp64"):
        from .structure import matrix_from_sparse
        P = matrix_from_sparse(M)
        if P is None:
            raise ValueError("SparseLU: M does not have the block-bordered form (block-"
                             "tridiagonal interior with b in (8, 16, 32), at most 128 tau rows)")
        self.b, self.t, self.n = P.b, P.t, P.n
        self.shape = (P.n, P.n)
        self._dev = DevicePencil(P)
        self.device = DevicePreconditioner(self._dev, 0.0, "exact", precision=precision)

    def solve(self, rhs) -> np.ndarray:
        import torch
        x = np.asarray(rhs, dtype=np.complex128)
        if x.shape[0] != self.n or x.ndim not in (1, 2):
            raise ValueError(f"rhs must have shape ({self.n},) or ({self.n}, m); got {x.shape}")
        cols = x.reshape(self.n, -1)
        xd = torch.from_numpy(np.ascontiguousarray(cols.T)).to("cuda")
        yd = torch.empty_like(xd)
        lib = self.device._lib
        for j in range(xd.shape[0]):
            st = lib.bbjd_precond_solve(self.device.handle, 1, xd[j].data_ptr(), yd[j].data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
            if st != 0:
                raise RuntimeError(f"bbjd_precond_solve failed: {_lib.STATUS_MSG.get(st, st)}")
        y = yd.cpu().numpy().T
        return y.reshape(x.shape).copy()

    def close(self):
        self.device.close()
        self._dev.close()


def _raise_status(status: int, nconv: int, k: int, iters: int, verbose: int):
    """Status mapping of reference bbjd.py:248-266."""
    if status < 0:
        msg = _lib.STATUS_MSG.get(status, f"unknown error (status={status})")
        raise RuntimeError(f"JDQZ solver failed: {msg}")
    if status == 1 and verbose >= 1:
        warnings.warn(f"JDQZ: only {nconv}/{k} eigenvalues converged in {iters} iterations.",
                      RuntimeWarning, stacklevel=3)


def _marshal(res: _lib.Result, n: int, row_major: bool = False):
    """Copy a bbjd_result out before bbjd_result_free.  ``row_major``: the
    device already wrote the (n, nconv) row-major array (BBJD_EVEC_ROW_MAJOR),
    so the copy is contiguous; otherwise the n x nconv column-major vectors
    are transposed on the host as in the reference (_bbjd_c.c:240-246)."""
    nconv = int(res.nconv)
    if nconv > 0:
        ev = np.ctypeslib.as_array(C.cast(res.eigenvalues, C.POINTER(C.c_double)),
                                   shape=(2 * nconv,)).view(np.complex128).copy()
        vecs = np.ctypeslib.as_array(C.cast(res.eigenvectors, C.POINTER(C.c_double)),
                                     shape=(2 * n * nconv,)).view(np.complex128)
        if row_major:
            evecs = vecs.reshape(n, nconv).copy()
        else:
            evecs = np.array(vecs.reshape(nconv, n).T)      # (n, nconv), C order
        resid = np.ctypeslib.as_array(res.residuals, shape=(nconv,)).copy()
    else:
        ev = np.zeros(0, np.complex128)
        evecs = np.zeros((n, 0), np.complex128)
        resid = np.zeros(0)
    return ev, evecs, resid


class _Callbacks:
    """Host trampolines (the role of reference _bbjd_c.c:43-123): wrap the
    library's host pointers as numpy views, call the Python callable, copy
    the result back.  The first exception is kept and re-raised after the
    solve, and later callbacks fail immediately (reference _bbjd_c.c:47)."""

    def __init__(self, n, fA, fB, fP):
        self.n = n
        self.error = None
        self.fns = [self._wrap(fA), self._wrap(fB), self._wrap(fP) if fP is not None else None]

    def _wrap(self, f):
        n = self.n

        def tramp(nn, x, y, data):
            if self.error is not None:
                return -1
            try:
                xa = np.ctypeslib.as_array(C.cast(x, C.POINTER(C.c_double)),
                                           shape=(2 * n,)).view(np.complex128)
                xa.flags.writeable = False
                ya = np.asarray(f(xa), dtype=np.complex128).reshape(-1)
                if ya.shape != (n,):
                    raise ValueError(f"operator returned shape {ya.shape}, expected ({n},)")
                C.memmove(y, ya.ctypes.data, 16 * n)
                return 0
            except BaseException as e:  # noqa: BLE001 - propagated after the solve
                self.error = e
                return -1
        return _lib.MATVEC_FN(tramp)


def jdqz_c(n, nev, sigma, target, matvec_A, matvec_B, precond_solve, tol=1e-10, maxiter=200,
           maxsub=0, minsub=0, inner_maxiter=0, inner_tol=1e-2, verbose=0, v0=None):
    """Drop-in for the reference's extension function ``_bbjd_c.jdqz_c``
    (reference _bbjd_c.c:128-259): same arguments, returns
    ``(eigenvalues, eigenvectors, residuals, nconv, iters, status)``."""
    lib = _lib.load()
    n = int(n)
    nev = int(nev)
    v0_arr = None
    if v0 is not None:
        v0_arr = np.ascontiguousarray(v0, dtype=np.complex128)
        if v0_arr.ndim != 1 or v0_arr.shape[0] != n:
            raise ValueError(f"v0 must have shape ({n},)")
    cb = _Callbacks(n, matvec_A, matvec_B, precond_solve)
    p = _lib.Params()
    lib.bbjd_params_init(C.byref(p))
    p.n, p.nev = n, nev
    p.sigma = _lib.zcomplex.of(sigma)
    p.target = int(target)
    p.tol = float(tol)
    p.maxiter, p.maxsub, p.minsub = int(maxiter), int(maxsub), int(minsub)
    p.inner_maxiter, p.inner_tol = int(inner_maxiter), float(inner_tol)
    p.matvec_A, p.matvec_B = cb.fns[0], cb.fns[1]
    if cb.fns[2] is not None:
        p.precond = cb.fns[2]
    p.verbose = int(verbose)
    p.v0 = v0_arr.ctypes.data if v0_arr is not None else None
    ws = lib.bbjd_workspace_alloc(C.byref(p))
    if not ws:
        raise MemoryError("bbjd_workspace_alloc failed")
    res = _lib.Result()
    try:
        status = lib.bbjd_solve(C.byref(p), ws, C.byref(res))
    finally:
        lib.bbjd_workspace_free(ws)
    try:
        if cb.error is not None:
            raise cb.error
        ev, evecs, resid = _marshal(res, n)
    finally:
        lib.bbjd_result_free(C.byref(res))
    return ev, evecs, resid, int(res.nconv), int(res.iters), int(status)


_PROJECTED = {"auto": 0, "qz": 1, "schur": 2}
_LOCK = {"robust": 0, "reference": 1}
_RITZ = {"auto": 0, "fp64": 1, "fp32": 2}
_OVERLAP = {"auto": 0, "off": 1}


def _solve_device(dev: DevicePencil, pc, k, sigma, target, tol, maxiter, maxsub, minsub,
                  inner_maxiter, inner_tol, v0, verbose, timing, projected="auto",
                  lock="robust", precision="fp64", ritz_estimate="auto", host_overlap="auto"):
    lib = _lib.load()
    n = dev.n
    p = _lib.Params()
    lib.bbjd_params_init(C.byref(p))
    p.n, p.nev = n, int(k)
    p.sigma = _lib.zcomplex.of(sigma)
    p.target = int(target)
    p.tol = float(tol)
    p.maxiter, p.maxsub, p.minsub = int(maxiter), int(maxsub), int(minsub)
    p.inner_maxiter, p.inner_tol = int(inner_maxiter), float(inner_tol)
    p.verbose = int(verbose)
    p.v0 = v0.ctypes.data if v0 is not None else None
    ext = _lib.DeviceExt()
    lib.bbjd_device_ext_init(C.byref(ext))
    ext.record_timing = 1 if timing else 0
    if precision not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'")
    ext.precision = 1 if precision == "mixed" else 0
    if projected not in _PROJECTED:
        raise ValueError(f"projected must be one of {list(_PROJECTED)}")
    ext.projected = _PROJECTED[projected]
    if lock not in _LOCK:
        raise ValueError(f"lock must be one of {list(_LOCK)}")
    ext.lock_rule = _LOCK[lock]
    if ritz_estimate not in _RITZ:
        raise ValueError(f"ritz_estimate must be one of {list(_RITZ)}")
    ext.ritz_estimate = _RITZ[ritz_estimate]
    if host_overlap not in _OVERLAP:
        raise ValueError(f"host_overlap must be one of {list(_OVERLAP)}")
    ext.host_overlap = _OVERLAP[host_overlap]
    conv_iters = np.zeros(int(k), dtype=np.int64)
    ext.conv_iters = conv_iters.ctypes.data
    ext.evec_layout = 1        # BBJD_EVEC_ROW_MAJOR: the (n, nconv) array comes back ready
    ws = lib.bbjd_workspace_alloc(C.byref(p))
    if not ws:
        raise MemoryError("bbjd_workspace_alloc failed (device memory)")
    res = _lib.Result()
    try:
        status = lib.bbjd_solve_device(C.byref(p), C.byref(ext), dev.handle,
                                       pc.handle if pc is not None else None, ws, C.byref(res))
    finally:
        lib.bbjd_workspace_free(ws)
    try:
        ev, evecs, resid = _marshal(res, n, row_major=True)
    finally:
        lib.bbjd_result_free(C.byref(res))
    stats = {
        "seconds_total": ext.seconds_total, "seconds_qz": ext.seconds_qz,
        "seconds_device": ext.seconds_device, "seconds_restart": ext.seconds_restart,
        "bytes_device": ext.bytes_device, "kernel_launches": int(ext.kernel_launches),
        "dgks_passes": int(ext.dgks_passes), "restarts": int(ext.restarts),
        "duplicates": int(ext.duplicates), "ritz_refinements": int(ext.ritz_refinements),
        "ritz_fallbacks": int(ext.ritz_fallbacks),
        "seconds_qz_exposed": ext.seconds_qz_exposed, "guess_hits": int(ext.guess_hits),
        "guess_misses": int(ext.guess_misses),
        "conv_iters": conv_iters[:int(res.nconv)].copy(),
        "kernels": {name: {"ms": ext.kernel_ms[i], "bytes": ext.kernel_bytes[i],
                           "calls": int(ext.kernel_calls[i])}
                    for i, name in enumerate(_lib.KERNEL_CLASSES)},
    }
    return ev, evecs, resid, int(res.nconv), int(res.iters), int(status), stats


def jdqz(
    A,
    B=None,
    k: int = 6,
    sigma: complex = 0.0,
    which: str = 'nearest',
    tol: float = 1e-10,
    maxiter: int = 200,
    maxsub: int = 0,
    minsub: int = 0,
    inner_maxiter: int = 0,
    inner_tol: float = 1e-2,
    preconditioner=None,
    v0=None,
    verbose: int = 0,
    return_info: bool = False,
    timing: bool = False,
    projected: str = "auto",
    lock: str = "robust",
    precision: str = "fp64",
    oracle=None,
    ritz_estimate: str = "auto",
    host_overlap: str = "auto",
):
    """Jacobi-Davidson QZ for ``A x = lambda B x``, the eigenvalues nearest
    ``sigma`` first.  Parameters, defaults, returns and errors are those of
    the reference (reference bbjd.py:59-158): returns ``(eigenvalues,
    eigenvectors)`` or, with ``return_info``, also an info dict with
    ``nconv``, ``iters``, ``status`` and ``residuals`` (plus ``device`` with
    timing and traffic statistics on the device path).

    maxsub 0 means max(3k + 10, 40) capped at n; minsub 0 means
    max(2k + 5, 20) (the values the reference's C core uses,
    jd_core.c:95-98 and 750-752).

    Device path only: ``timing`` records per-kernel-class CUDA-event times
    in ``info['device']``; ``projected`` picks the projected eigensolver
    ('qz': ZGGES + ZTGSEN as the reference; 'schur': the harmonic standard
    form, same deflating subspaces, ~4x cheaper; 'auto': 'schur' for the
    'nearest' and 'SM' targets).  The callback path always uses 'qz'.
    ``lock`` picks how converged values are recognised: 'robust' (a relative
    window and an eigenvector-angle test, so an ill-conditioned eigenvalue is
    not returned twice) or 'reference' (the reference's absolute 100 tol
    window, jd_core.c:369, 439).  ``precision='mixed'`` stores the device
    LU factors in complex64 and runs the first CGS pass against V over a
    complex64 copy of V (the second pass, DGKS, residuals, projected pencil
    and QZ stay FP64).  ``oracle``: reference eigenvalues (e.g. from an FP64
    run or ARPACK); with ``return_info`` the info dict then holds
    ``error_vs_oracle``, the largest distance from a returned eigenvalue to
    its nearest oracle value.  ``ritz_estimate`` (Schur form only): 'fp32'
    ('auto') ranks the candidates between restarts by complex64 estimates
    of the projected eigenvalues and refines the chosen one to an FP64
    eigenpair by Rayleigh-quotient iteration (the FP64 path takes over when
    that does not converge); 'fp64' computes all of them in FP64.  The
    returned values and the convergence test are FP64 either way.
    ``host_overlap`` (FP32 estimates only): 'auto' computes the estimates
    on a second host thread while the device iterates on the target guessed
    from the previous one (a rejected guess repeats that device work); 'off'
    computes them first.  Both return the same bits.  ``info['device']``
    reports ``conv_iters`` (the outer iteration at which each returned pair
    converged), ``guess_hits`` / ``guess_misses`` and
    ``seconds_qz_exposed`` (the projected-solve seconds not hidden behind
    the device).
    """
    if which not in _TARGET_MAP:
        raise ValueError(f"which must be one of {list(_TARGET_MAP.keys())}; got {which!r}")
    sigma = complex(sigma)
    target = _TARGET_MAP[which]

    if isinstance(A, (BBTPencil, DevicePencil)):
        if B is not None:
            raise ValueError("a block-bordered pencil carries its own B; pass B=None")
        dev = A if isinstance(A, DevicePencil) else DevicePencil(A)
        n = dev.n
        if v0 is not None:
            v0 = np.ascontiguousarray(v0, dtype=np.complex128)
            if v0.shape != (n,):
                raise ValueError(f"v0 must have shape ({n},); got {v0.shape}")
        own_pc = False
        if preconditioner is None:
            pc = None
        elif isinstance(preconditioner, DevicePreconditioner):
            pc = preconditioner
        elif isinstance(preconditioner, str):
            pc = DevicePreconditioner(dev, sigma, preconditioner, precision=precision)
            own_pc = True
        else:
            raise ValueError("with a block-bordered pencil the preconditioner must be 'exact', "
                             "'block_jacobi', a DevicePreconditioner or None")
        try:
            ev, evecs, resid, nconv, iters, status, stats = _solve_device(
                dev, pc, k, sigma, target, tol, maxiter, maxsub, minsub, inner_maxiter,
                inner_tol, v0, verbose, timing, projected, lock, precision, ritz_estimate,
                host_overlap)
        finally:
            if own_pc:
                pc.close()
        _raise_status(status, nconv, k, iters, verbose)
        if return_info:
            return ev, evecs, _with_oracle({"nconv": nconv, "iters": iters, "status": status,
                                            "residuals": resid, "device": stats}, ev, oracle)
        return ev, evecs

    # ---- sparse block-bordered pencil: packed and solved on the device ----
    device_pc = (preconditioner is None or isinstance(preconditioner, (str, SparseLU,
                                                                         DevicePreconditioner)))
    if device_pc and (sp.issparse(A) or isinstance(A, np.ndarray)) and \
            (B is None or sp.issparse(B) or isinstance(B, np.ndarray)):
        from .structure import pencil_from_sparse
        P = pencil_from_sparse(A, B, b_is_identity=B is None)
        if P is not None:
            pc = preconditioner.device if isinstance(preconditioner, SparseLU) else preconditioner
            if pc is not None and not isinstance(pc, str) and pc.n != P.n:
                raise ValueError(f"preconditioner has size {pc.n}; the pencil has {P.n}")
            return jdqz(P, None, k=k, sigma=sigma, which=which, tol=tol, maxiter=maxiter,
                        maxsub=maxsub, minsub=minsub, inner_maxiter=inner_maxiter,
                        inner_tol=inner_tol, preconditioner=pc, v0=v0, verbose=verbose,
                        return_info=return_info, timing=timing, projected=projected,
                        lock=lock, precision=precision, oracle=oracle,
                        ritz_estimate=ritz_estimate, host_overlap=host_overlap)
        if isinstance(preconditioner, (str, SparseLU, DevicePreconditioner)):
            raise ValueError("a device preconditioner needs a block-bordered A, B pencil")

    # ---- callback path: validation as reference bbjd.py:160-224 ----
    if isinstance(A, np.ndarray):
        A = sp.csr_matrix(A)
    if callable(A) and not hasattr(A, "shape"):
        raise ValueError("a bare callable A needs its size; wrap it in a LinearOperator")
    n = A.shape[0]
    if A.shape != (n, n):
        raise ValueError(f"A must be square; got shape {A.shape}")
    if B is None:
        B_op = sp.eye(n, dtype=np.complex128, format='csr')
    elif isinstance(B, np.ndarray):
        B_op = sp.csr_matrix(B)
    else:
        B_op = B

    if sp.issparse(A):
        A_csc = A.astype(np.complex128).tocsc()
        matvec_A = lambda x: A_csc @ x  # noqa: E731
    elif hasattr(A, 'matvec'):
        matvec_A = lambda x: np.asarray(A.matvec(x), dtype=np.complex128)  # noqa: E731
    elif callable(A):
        matvec_A = A
    else:
        raise ValueError("A must be a sparse matrix, LinearOperator, or callable")
    if sp.issparse(B_op):
        B_csc = B_op.astype(np.complex128).tocsc()
        matvec_B = lambda x: B_csc @ x  # noqa: E731
    elif hasattr(B_op, 'matvec'):
        matvec_B = lambda x: np.asarray(B_op.matvec(x), dtype=np.complex128)  # noqa: E731
    elif callable(B_op):
        matvec_B = B_op
    else:
        raise ValueError("B must be a sparse matrix, LinearOperator, or callable")

    if preconditioner is not None:
        if hasattr(preconditioner, 'solve'):
            pcobj = preconditioner
            precond_solve = lambda x: np.asarray(pcobj.solve(x), dtype=np.complex128)  # noqa: E731
        elif callable(preconditioner):
            precond_solve = preconditioner
        else:
            raise ValueError("preconditioner must have a .solve(b) method or be callable")
    else:
        precond_solve = None

    if v0 is not None:
        v0 = np.ascontiguousarray(v0, dtype=np.complex128)
        if v0.shape != (n,):
            raise ValueError(f"v0 must have shape ({n},); got {v0.shape}")

    evals, evecs, resid, nconv, iters, status = jdqz_c(
        n=n, nev=k, sigma=sigma, target=target, matvec_A=matvec_A, matvec_B=matvec_B,
        precond_solve=precond_solve, tol=tol, maxiter=maxiter, maxsub=maxsub, minsub=minsub,
        inner_maxiter=inner_maxiter, inner_tol=inner_tol, verbose=verbose, v0=v0)
    _raise_status(status, nconv, k, iters, verbose)
    if return_info:
        return evals, evecs, _with_oracle({'nconv': nconv, 'iters': iters, 'status': status,
                                           'residuals': resid}, evals, oracle)
    return evals, evecs


def _with_oracle(info: dict, ev, oracle) -> dict:
    if oracle is not None:
        ref = np.asarray(oracle, dtype=np.complex128).reshape(-1)
        info["error_vs_oracle"] = (float(max(np.min(np.abs(ref - e)) for e in ev))
                                   if len(ev) and len(ref) else float("nan"))
    return info


def jdqz_device(pencil, **kwargs):
    """``jdqz`` on a block-bordered pencil already on the device or on the
    host (:class:`DevicePencil` / :class:`BBTPencil`): the device path with
    ``jdqz``'s keyword arguments, without the sparse-structure detection."""
    if not isinstance(pencil, (BBTPencil, DevicePencil)):
        raise TypeError("jdqz_device takes a BBTPencil or a DevicePencil")
    return jdqz(pencil, None, **kwargs)


def jdqz_batch(pencils, sigmas, k: int = 6, tol: float = 1e-10, maxiter: int = 200,
               maxsub: int = 0, minsub: int = 0, preconditioner: str = "exact",
               precision: str = "fp64", v0s=None, threads: int = 8, projected: str = "auto",
               lock: str = "robust", ritz_estimate: str = "auto"):
    """Independent 'nearest sigma' solves of a sigma-sweep on one GPU
    (bbjd_solve_batch): solve i is ``jdqz(pencils[i], k=k, sigma=sigmas[i],
    ...)``; up to `threads` run at once, each on its own host thread and
    CUDA stream, largest pencils first.  Solves may share a pencil (it is
    uploaded once).  Returns a list of ``(eigenvalues, eigenvectors, info)``
    and the batch's wall time in seconds.  The results do not depend on
    `threads` (the batch's projected eigenvalues always come from OpenBLAS,
    so they can differ from a single ``jdqz`` call, which may use MKL, by
    rounding)."""
    import time as _time
    lib = _lib.load()
    count = len(pencils)
    if len(sigmas) != count:
        raise ValueError("one sigma per pencil")
    if ritz_estimate not in _RITZ:
        raise ValueError(f"ritz_estimate must be one of {list(_RITZ)}")
    # one device copy per distinct pencil: the solves of a sweep over sigma
    # of the same pencil share it (read-only during the solves)
    uploaded: dict = {}
    devs = []
    for p in pencils:
        if isinstance(p, DevicePencil):
            devs.append(p)
        else:
            if id(p) not in uploaded:
                uploaded[id(p)] = DevicePencil(p)
            devs.append(uploaded[id(p)])
    pcs = [DevicePreconditioner(d, s, preconditioner, precision=precision) if preconditioner
           else None for d, s in zip(devs, sigmas)]
    if v0s is None:
        from .pencils import start_vector
        v0s = [start_vector(d.n, 1 + i) for i, d in enumerate(devs)]
    v0s = [np.ascontiguousarray(v, dtype=np.complex128) for v in v0s]
    params = (_lib.Params * count)()
    exts = (_lib.DeviceExt * count)()
    mats = (C.c_void_p * count)(*[d.handle.value for d in devs])
    pch = (C.c_void_p * count)(*[p.handle.value if p is not None else None for p in pcs])
    wss = (C.POINTER(_lib.Workspace) * count)()
    results = (_lib.Result * count)()
    for i, (d, s) in enumerate(zip(devs, sigmas)):
        p = params[i]
        lib.bbjd_params_init(C.byref(p))
        p.n, p.nev = d.n, int(k)
        p.sigma = _lib.zcomplex.of(s)
        p.tol, p.maxiter, p.maxsub, p.minsub = float(tol), int(maxiter), int(maxsub), int(minsub)
        if v0s[i].shape != (d.n,):
            raise ValueError(f"v0s[{i}] must have shape ({d.n},)")
        p.v0 = v0s[i].ctypes.data
        lib.bbjd_device_ext_init(C.byref(exts[i]))
        exts[i].precision = 1 if precision == "mixed" else 0
        exts[i].projected = _PROJECTED[projected]
        exts[i].lock_rule = _LOCK[lock]
        exts[i].ritz_estimate = _RITZ[ritz_estimate]
        exts[i].evec_layout = 1
        wss[i] = lib.bbjd_workspace_alloc(C.byref(p))
        if not wss[i]:
            for j in range(i):
                lib.bbjd_workspace_free(wss[j])
            raise MemoryError("bbjd_workspace_alloc failed (device memory)")
    t0 = _time.perf_counter()
    try:
        status = lib.bbjd_solve_batch(count, params, exts, mats, pch, wss, results, int(threads))
    finally:
        wall = _time.perf_counter() - t0
        for i in range(count):
            lib.bbjd_workspace_free(wss[i])
    if status < 0:
        for i in range(count):
            lib.bbjd_result_free(C.byref(results[i]))
        raise RuntimeError(f"JDQZ batch failed: {_lib.STATUS_MSG.get(status, status)}")
    out = []
    for i, d in enumerate(devs):
        try:
            ev, evecs, resid = _marshal(results[i], d.n, row_major=True)
        finally:
            lib.bbjd_result_free(C.byref(results[i]))
        out.append((ev, evecs, {"nconv": int(results[i].nconv), "iters": int(results[i].iters),
                                "status": int(results[i].status), "residuals": resid,
                                "seconds": exts[i].seconds_total,
                                "seconds_qz": exts[i].seconds_qz}))
    for p in pcs:
        if p is not None:
            p.close()
    return out, wall
