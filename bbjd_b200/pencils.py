"""Block-bordered (BBT) pencils: the host-side format and a seeded generator.

A BBT pencil is the structure spectral PDE discretisations produce and the
reference's deployment targets (reference ``include/bbjd.h:7-9``,
``README.md:38-44``):

* ``A`` is block-tridiagonal over ``nblk`` diagonal blocks of size ``b``
  (``nb = nblk*b`` interior rows), plus ``t`` dense border columns in the
  interior rows and ``t`` dense tau rows, so ``n = nb + t``;
* ``B`` is block-diagonal over the same blocks, and its tau rows are zero
  (``B`` is singular whenever ``t > 0``).

Host layout (numpy, row-major blocks as a user writes them):

=============  ==================  ==========================================
field          shape               meaning
=============  ==================  ==========================================
``Ad``         (nblk, b, b)        ``A[jb:jb+b, jb:jb+b]``
``Al``         (nblk, b, b)        ``A[jb:jb+b, jb-b:jb]`` (``Al[0]`` = 0)
``Au``         (nblk, b, b)        ``A[jb:jb+b, jb+b:jb+2b]`` (``Au[-1]`` = 0)
``E``          (nb, t)             ``A[:nb, nb:]`` border columns
``F``          (t, n)              ``A[nb:, :]`` tau rows (corner included)
``Bd``         (nblk, b, b)        ``B[jb:jb+b, jb:jb+b]``
=============  ==================  ==========================================

The device layout (column-major blocks, ``F`` stored transposed) is produced
by :meth:`BBTPencil.device_arrays`; the CUDA SpMV and LU kernels read it.

The generator restates the synthetic pencil the benchmark configurations
describe (block noise ``cn(b,b)/sqrt(b)``, per-block diagonal shift
``i*linspace(-50,50,nblk)[j] + linspace(0,10,nblk)[j]``, border and tau
entries ``cn/sqrt(n)``, ``B = blockdiag(I + 0.1 cn(b,b)/sqrt(b))`` with zero
tau rows), with ``cn = (N(0,1) + i N(0,1))/sqrt(2)`` drawn from
``numpy.random.default_rng(seed)`` in the fixed order below.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp


@dataclass
class BBTPencil:
    b: int
    nblk: int
    t: int
    Ad: np.ndarray
    Al: np.ndarray
    Au: np.ndarray
    E: np.ndarray
    F: np.ndarray
    Bd: np.ndarray

    @property
    def nb(self) -> int:
        return self.nblk * self.b

    @property
    def n(self) -> int:
        return self.nb + self.t

    # ------------------------------------------------------------------
    def validate(self) -> None:
        b, nblk, t, nb, n = self.b, self.nblk, self.t, self.nb, self.n
        for name in ("Ad", "Al", "Au", "Bd"):
            a = getattr(self, name)
            if a.shape != (nblk, b, b):
                raise ValueError(f"{name} must have shape {(nblk, b, b)}; got {a.shape}")
        if self.E.shape != (nb, t):
            raise ValueError(f"E must have shape {(nb, t)}; got {self.E.shape}")
        if self.F.shape != (t, n):
            raise ValueError(f"F must have shape {(t, n)}; got {self.F.shape}")

    # ------------------------------------------------------------------
    def matvec_A(self, x: np.ndarray) -> np.ndarray:
        """Host A @ x straight from the block arrays (checker use)."""
        b, nblk, nb = self.b, self.nblk, self.nb
        xb = x[:nb].reshape(nblk, b)
        y = np.empty(self.n, dtype=np.complex128)
        yb = np.einsum("jic,jc->ji", self.Ad, xb)
        yb[1:] += np.einsum("jic,jc->ji", self.Al[1:], xb[:-1])
        yb[:-1] += np.einsum("jic,jc->ji", self.Au[:-1], xb[1:])
        if self.t:
            yb += (self.E @ x[nb:]).reshape(nblk, b)
            y[nb:] = self.F @ x
        y[:nb] = yb.reshape(-1)
        return y

    def matvec_B(self, x: np.ndarray) -> np.ndarray:
        b, nblk, nb = self.b, self.nblk, self.nb
        y = np.zeros(self.n, dtype=np.complex128)
        y[:nb] = np.einsum("jic,jc->ji", self.Bd, x[:nb].reshape(nblk, b)).reshape(-1)
        return y

    # ------------------------------------------------------------------
    def to_csc(self, which: str = "A") -> sp.csc_matrix:
        """Assemble A or B as scipy CSC (the form the reference's wrapper
        turns into matvec closures, reference ``bbjd.py:183-205``)."""
        b, nblk, t, nb, n = self.b, self.nblk, self.t, self.nb, self.n
        if which == "B":
            K = sp.bsr_matrix((self.Bd, np.arange(nblk), np.arange(nblk + 1)),
                              shape=(nb, nb))
            if t == 0:
                return K.tocsc()
            return sp.bmat([[K, None], [None, sp.csc_matrix((t, t), dtype=np.complex128)]],
                           format="csc")
        # block-tridiagonal interior as BSR: block row j holds columns j-1, j, j+1
        cols, data, indptr = [], [], [0]
        for j in range(nblk):
            if j > 0:
                cols.append(j - 1)
                data.append(j * 3 + 0)
            cols.append(j)
            data.append(j * 3 + 1)
            if j < nblk - 1:
                cols.append(j + 1)
                data.append(j * 3 + 2)
            indptr.append(len(cols))
        blocks = np.stack([self.Al, self.Ad, self.Au], axis=1).reshape(nblk * 3, b, b)
        K = sp.bsr_matrix((blocks[np.asarray(data)], np.asarray(cols), np.asarray(indptr)),
                          shape=(nb, nb))
        if t == 0:
            return K.tocsc()
        top = sp.hstack([K.tocsc(), sp.csc_matrix(self.E)], format="csc")
        return sp.vstack([top, sp.csc_matrix(self.F)], format="csc")

    def shifted(self, sigma: complex) -> "BBTPencil":
        """The pencil with A replaced by A - sigma B (interior blocks only:
        B's tau rows and border are zero)."""
        return BBTPencil(self.b, self.nblk, self.t, self.Ad - sigma * self.Bd,
                         self.Al, self.Au, self.E, self.F, self.Bd)

    def device_arrays(self) -> dict:
        """Column-major-in-block copies the CUDA kernels read.

        Blocks are stored ``[j][c][i]`` (element (i, c) of block j at
        ``j*b*b + c*b + i``) so that the lane owning row i reads column c
        of 32 rows with one coalesced 512-byte transaction; ``E`` is
        column-major (ld = nb); ``F`` is stored transposed, ``FT[col][tau]``,
        so that a warp reads the t tau entries of one column contiguously.
        Every array is returned flat (1-D, contiguous) in that order, so a
        caller that copies or reinterprets it (pinned buffers, ``.view``)
        cannot reorder it by accident.
        """
        tr = lambda a: np.ascontiguousarray(np.transpose(a, (0, 2, 1))).reshape(-1)  # noqa: E731
        none = np.zeros((0,), np.complex128)
        return {
            "Ad": tr(self.Ad), "Al": tr(self.Al), "Au": tr(self.Au), "Bd": tr(self.Bd),
            "E": np.ascontiguousarray(self.E.T).reshape(-1) if self.t else none,
            "FT": np.ascontiguousarray(self.F.T).reshape(-1) if self.t else none,
        }


def _cn(rng: np.random.Generator, shape) -> np.ndarray:
    re = rng.standard_normal(shape)
    im = rng.standard_normal(shape)
    out = np.empty(shape, dtype=np.complex128)
    out.real = re
    out.imag = im
    out *= 1.0 / np.sqrt(2.0)
    return out


def make_pencil(b: int, nblk: int, t: int, seed: int = 0) -> BBTPencil:
    """Seeded synthetic BBT pencil (see the module docstring for the law)."""
    rng = np.random.default_rng(seed)
    nb = b * nblk
    n = nb + t
    sb = 1.0 / np.sqrt(b)
    Ad = _cn(rng, (nblk, b, b))
    Ad *= sb
    shifts = 1j * np.linspace(-50.0, 50.0, nblk) + np.linspace(0.0, 10.0, nblk)
    idx = np.arange(b)
    Ad[:, idx, idx] += shifts[:, None]
    Al = _cn(rng, (nblk, b, b))
    Al *= sb
    Al[0] = 0.0
    Au = _cn(rng, (nblk, b, b))
    Au *= sb
    Au[-1] = 0.0
    sn = 1.0 / np.sqrt(n)
    E = _cn(rng, (nb, t))
    E *= sn
    F = _cn(rng, (t, n))
    F *= sn
    Bd = _cn(rng, (nblk, b, b))
    Bd *= 0.1 * sb
    Bd[:, idx, idx] += 1.0
    return BBTPencil(b, nblk, t, Ad, Al, Au, E, F, Bd)


def start_vector(n: int, seed: int = 1) -> np.ndarray:
    """Seeded start vector: real normal draws cast to complex128."""
    return np.random.default_rng(seed).standard_normal(n).astype(np.complex128)


# The workloads the benchmark configurations name (sizes only; solver
# parameters live with the callers).
CONFIGS = {
    "n4104": dict(b=16, nblk=256, t=8, sigma=3.0 + 0j, k=8, maxsub=40, minsub=20, tol=1e-10),
    "n1e6": dict(b=32, nblk=31250, t=64, sigma=3.0 + 0j, k=64, maxsub=200, minsub=80,
                 tol=1e-10, maxiter=2000),
    "n1e6_gmres": dict(b=32, nblk=31250, t=64, sigma=3.0 + 0j, k=32, maxsub=120, minsub=48,
                       tol=1e-10, inner_maxiter=50, inner_tol=1e-3),
}
