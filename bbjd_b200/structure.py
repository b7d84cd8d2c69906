"""Recognise the block-bordered structure in scipy sparse matrices.

The reference's users hand ``jdqz`` scipy sparse ``A`` and ``B`` (CSR
preferred, reference README.md:36-58) and a sparse LU of ``A - sigma B``.
When those matrices have the block-bordered form -- ``A`` block-tridiagonal
over ``nblk`` blocks of size ``b`` in its first ``nb = n - t`` rows and
columns, any entries in the ``t`` border columns and the ``t`` trailing tau
rows, ``B`` block-diagonal over the same blocks and zero outside them -- the
pencil is packed into :class:`~bbjd_b200.pencils.BBTPencil` and the whole
solve runs on the device.  Anything else keeps the callback path.

Detection is exact, never approximate: a candidate ``(b, t)`` is accepted
only if every stored entry of ``A`` (and ``B``) lands in a block the format
holds, so the packed pencil reproduces the sparse matrices entry for entry.
``b`` is tried in the sizes the kernels support (8, 16, 32), smallest
first, so the packed pencil stores the fewest explicit zeros.  ``t`` is
taken from ``B``'s trailing zero rows and from the trailing run of rows that
reach further left of the diagonal than any block-tridiagonal row can
(2 x 32 columns); ``t`` is at most 128.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .pencils import BBTPencil

BLOCK_SIZES = (8, 16, 32)
MAX_TAU = 128
_REACH = 2 * max(BLOCK_SIZES)
_CHUNK = 1 << 22           # stored entries handled per vectorised step


def _csr(M) -> sp.csr_matrix:
    M = sp.csr_matrix(M, dtype=np.complex128)
    M.sum_duplicates()
    M.sort_indices()
    return M


def _row_chunks(M: sp.csr_matrix, r0: int, r1: int):
    """(rows, cols, vals) of the stored entries of rows [r0, r1), in pieces
    of about _CHUNK entries."""
    ip = M.indptr
    r = r0
    while r < r1:
        hi = int(np.searchsorted(ip, ip[r] + _CHUNK, side="right")) - 1
        hi = min(max(hi, r + 1), r1)
        s, e = ip[r], ip[hi]
        rows = np.repeat(np.arange(r, hi, dtype=np.int64), np.diff(ip[r:hi + 1]))
        yield rows, M.indices[s:e].astype(np.int64), M.data[s:e]
        r = hi


def _tau_candidates(A: sp.csr_matrix, B: sp.csr_matrix | None) -> list[int]:
    n = A.shape[0]
    cands = []
    if B is not None:
        nz_rows = np.nonzero(np.diff(B.indptr))[0]
        cands.append(n - (int(nz_rows[-1]) + 1) if len(nz_rows) else n)
    cnt = np.diff(A.indptr)
    lo = np.full(n, n, dtype=np.int64)
    has = cnt > 0
    lo[has] = A.indices[A.indptr[:-1][has]]
    far = lo < np.arange(n, dtype=np.int64) - _REACH
    near = np.nonzero(~far)[0]
    cands.append(n - (int(near[-1]) + 1) if len(near) else n)
    cands.append(0)
    out = []
    for t in cands:
        if 0 <= t <= MAX_TAU and t < n and t not in out:
            out.append(t)
    return out


def _fits(A: sp.csr_matrix, B: sp.csr_matrix | None, b: int, t: int, identity_b: bool) -> bool:
    n = A.shape[0]
    nb = n - t
    if nb <= 0 or nb % b:
        return False
    for rows, cols, _ in _row_chunks(A, 0, nb):
        m = cols < nb
        if np.any(np.abs(rows[m] // b - cols[m] // b) > 1):
            return False
    if identity_b:
        return t == 0
    if B is None:
        return True
    if B.indptr[-1] != B.indptr[nb]:            # B's tau rows must be zero
        return False
    for rows, cols, _ in _row_chunks(B, 0, nb):
        if np.any(cols >= nb) or np.any(rows // b != cols // b):
            return False
    return True


def detect(A, B=None, *, b_is_identity: bool = False):
    """``(b, t)`` of the block-bordered form of ``A`` (and ``B``), or None.

    ``B=None`` with ``b_is_identity`` means B = I (the reference's default),
    which the form holds only without tau rows (t = 0).  ``B=None`` without
    it checks ``A`` alone (a matrix to factor, not a pencil)."""
    A = _csr(A)
    n = A.shape[0]
    if A.shape != (n, n) or n < 2:
        return None
    Bc = _csr(B) if B is not None else None
    if Bc is not None and Bc.shape != A.shape:
        return None
    for t in _tau_candidates(A, Bc):
        for b in BLOCK_SIZES:
            if _fits(A, Bc, b, t, b_is_identity and Bc is None):
                return b, t
    return None


def _blocks(M: sp.csr_matrix, b: int, nblk: int, t: int, diag_only: bool):
    nb = nblk * b
    D = np.zeros((nblk, 1 if diag_only else 3, b, b), dtype=np.complex128)
    E = np.zeros((nb, t), dtype=np.complex128)
    for rows, cols, vals in _row_chunks(M, 0, nb):
        m = cols < nb
        r, c, v = rows[m], cols[m], vals[m]
        blk = r // b
        slot = np.zeros_like(blk) if diag_only else c // b - blk + 1
        D[blk, slot, r % b, c % b] = v
        if t and not diag_only:
            mb = ~m
            E[rows[mb], cols[mb] - nb] = vals[mb]
    return D, E


def pencil_from_sparse(A, B=None, b: int | None = None, t: int | None = None,
                       *, b_is_identity: bool = True) -> BBTPencil | None:
    """Pack sparse ``A``, ``B`` (None: the identity) into a BBTPencil, or
    return None when they do not have the block-bordered form."""
    if b is None or t is None:
        bt = detect(A, B, b_is_identity=b_is_identity)
        if bt is None:
            return None
        b, t = bt
    A = _csr(A)
    n = A.shape[0]
    nblk = (n - t) // b
    nb = nblk * b
    D, E = _blocks(A, b, nblk, t, diag_only=False)
    F = A[nb:, :].toarray() if t else np.zeros((0, n), dtype=np.complex128)
    if B is None:
        Bd = np.broadcast_to(np.eye(b, dtype=np.complex128), (nblk, b, b)).copy()
    else:
        Bd = _blocks(_csr(B), b, nblk, 0, diag_only=True)[0][:, 0]
    P = BBTPencil(b, nblk, t, np.ascontiguousarray(D[:, 1]), np.ascontiguousarray(D[:, 0]),
                  np.ascontiguousarray(D[:, 2]), E, np.ascontiguousarray(F), Bd)
    P.validate()
    return P


def matrix_from_sparse(M, b: int | None = None, t: int | None = None) -> BBTPencil | None:
    """Pack a single block-bordered matrix (``M = A - sigma B`` for a
    factorisation) as the ``A`` of a pencil with ``B = 0``."""
    if b is None or t is None:
        bt = detect(M, None, b_is_identity=False)
        if bt is None:
            return None
        b, t = bt
    P = pencil_from_sparse(M, None, b, t)
    P.Bd = np.zeros_like(P.Bd)
    return P
