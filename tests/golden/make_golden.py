"""Generate the golden fixtures of the parity tests by running the reference.

Runs the reference's own ``jdqz`` (its ``bbjd.py`` imported from the
reference checkout, with its C core built from the reference's sources by
``oracle/Makefile`` into ``oracle/_ref``) on seeded inputs and stores what it
returns -- eigenvalues, residuals, iteration counts -- plus ARPACK
shift-invert eigenvalues of the same pencils, as small ``.npz`` files here.

Only this script reads the reference checkout; the fixtures it writes are
what the tests read (the GPU box has no reference checkout).

    python tests/golden/make_golden.py [--ref REFERENCE_CHECKOUT] [--only case,...]
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np
import scipy.sparse as sp
from scipy.sparse.linalg import eigs, splu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bbjd_b200.pencils import make_pencil, start_vector  # noqa: E402


class _LU:
    def __init__(self, M):
        self._lu = splu(sp.csc_matrix(M))

    def solve(self, b):
        return self._lu.solve(b)


def _arpack(A, B, sigma, k):
    vals = eigs(A, k=k, M=B, sigma=sigma, which="LM", return_eigenvectors=False, tol=1e-13)
    return vals[np.argsort(np.abs(vals - sigma))]


def bbt_case(name, b, nblk, t, sigma, k, maxsub, minsub, seed=0, inner_maxiter=0,
             inner_tol=1e-2, pc_shift=0.0, maxiter=2000, n_arpack=None, pc="exact", v0_seed=None):
    from bbjd import jdqz  # the reference wrapper
    P = make_pencil(b, nblk, t, seed=seed)
    A, B = P.to_csc("A"), P.to_csc("B")
    if pc == "block_jacobi":
        from oracle.bbt_lu import BlockJacobiHost
        lu = BlockJacobiHost(P, sigma + pc_shift)
    else:
        lu = _LU((A - (sigma + pc_shift) * B).tocsc())
    v0 = start_vector(P.n, seed + 1 if v0_seed is None else v0_seed)
    t0 = time.time()
    ev, evec, info = jdqz(A, B, k=k, sigma=sigma, tol=1e-10, maxiter=maxiter, maxsub=maxsub,
                          minsub=minsub, inner_maxiter=inner_maxiter, inner_tol=inner_tol,
                          preconditioner=lu, v0=v0, return_info=True)
    dt = time.time() - t0
    # B is singular (zero tau rows): ARPACK in shift-invert mode with M = B
    # needs the generalized form OPinv = (A - sigma B)^-1, fed through the LU
    from scipy.sparse.linalg import LinearOperator
    luA = splu((A - sigma * B).tocsc())
    op = LinearOperator(A.shape, matvec=lambda x: luA.solve(B @ x), dtype=np.complex128)
    mu = eigs(op, k=n_arpack or (k + 16), which="LM", return_eigenvectors=False, tol=1e-13)
    arp = sigma + 1.0 / mu
    arp = arp[np.argsort(np.abs(arp - sigma))]
    res = np.array([np.linalg.norm(A @ evec[:, j] - ev[j] * (B @ evec[:, j])) / np.linalg.norm(evec[:, j])
                    for j in range(info["nconv"])])
    out = dict(kind="bbt", b=b, nblk=nblk, t=t, seed=seed, sigma=sigma, k=k, maxsub=maxsub,
               minsub=minsub, inner_maxiter=inner_maxiter, inner_tol=inner_tol, pc_shift=pc_shift,
               preconditioner=pc, v0_seed=seed + 1 if v0_seed is None else v0_seed,
               maxiter=maxiter, eigenvalues=ev, residuals=info["residuals"], unscaled_residuals=res,
               iters=info["iters"], nconv=info["nconv"], status=info["status"], arpack=arp,
               seconds=dt)
    np.savez(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: nconv={info['nconv']} iters={info['iters']} {dt:.2f}s")


def diag_case():
    from bbjd import jdqz
    d = 0.1 * np.arange(1, 51, dtype=np.complex128)
    A = sp.diags(d, format="csr")
    B = sp.eye(50, format="csr", dtype=np.complex128)
    ev, _, info = jdqz(A, B, k=5, sigma=0.0, tol=1e-10, preconditioner=_LU(A), return_info=True,
                       maxiter=200)
    np.savez(os.path.join(HERE, "diag50.npz"), kind="diag", eigenvalues=ev, iters=info["iters"],
             nconv=info["nconv"], residuals=info["residuals"])
    print(f"diag50: nconv={info['nconv']} iters={info['iters']}")


def random_case():
    """The reference test suite's random sparse pencil (n=200, seed 42)."""
    from bbjd import jdqz
    n = 200
    np.random.seed(42)
    A = sp.random(n, n, density=0.05, format="csr", dtype=np.complex128)
    A = A + 5.0 * sp.eye(n, dtype=np.complex128)
    A.data += 0.1j * np.random.randn(A.nnz)
    B = sp.eye(n, format="csr", dtype=np.complex128)
    sigma = 5.0
    ev, _, info = jdqz(A, B, k=6, sigma=sigma, tol=1e-10, preconditioner=_LU(A - sigma * B),
                       return_info=True, maxiter=500, maxsub=150, minsub=60)
    ref = eigs(A, k=12, sigma=sigma, which="LM", return_eigenvectors=False)
    np.savez(os.path.join(HERE, "random200.npz"), kind="random", A_data=A.tocsr().data,
             A_indices=A.tocsr().indices, A_indptr=A.tocsr().indptr, n=n, sigma=sigma,
             eigenvalues=ev, iters=info["iters"], nconv=info["nconv"], arpack=ref,
             residuals=info["residuals"])
    print(f"random200: nconv={info['nconv']} iters={info['iters']}")


# The sigma-sweep configuration scaled to CPU size: pencils of the same
# generator (b = t = 16) with uneven n, each with its own sigma on Re = 3
# (seeded draws), k = 4, maxsub 80, minsub 32.
SWEEP = dict(b=16, t=16, k=4, maxsub=80, minsub=32, nblks=(120, 173, 236, 301),
             im=(-31.7, -8.2, 12.9, 36.4))


def sweep_cases():
    for i, (nblk, im) in enumerate(zip(SWEEP["nblks"], SWEEP["im"])):
        bbt_case(f"sweep_{i}", b=SWEEP["b"], nblk=nblk, t=SWEEP["t"], sigma=complex(3.0, im),
                 k=SWEEP["k"], maxsub=SWEEP["maxsub"], minsub=SWEEP["minsub"], seed=100 + i,
                 v0_seed=1 + i)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("BBJD_REFERENCE", "/root/reference"),
                    help="reference checkout (default: $BBJD_REFERENCE)")
    ap.add_argument("--only", default=None, help="comma-separated case names")
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))   # _bbjd_c built from the reference
    sys.path.insert(0, args.ref)                               # the reference's bbjd.py
    os.environ.setdefault("OMP_NUM_THREADS", "4")
    cases = {
        "bbt_n4104": lambda: bbt_case("bbt_n4104", b=16, nblk=256, t=8, sigma=3.0, k=8, maxsub=40,
                                      minsub=20),
        "bbt_n516": lambda: bbt_case("bbt_n516", b=8, nblk=64, t=4, sigma=3.0, k=6, maxsub=30,
                                     minsub=12),
        "bbt_n516_gmres": lambda: bbt_case("bbt_n516_gmres", b=8, nblk=64, t=4, sigma=3.0, k=3,
                                           maxsub=30, minsub=12, inner_maxiter=20, inner_tol=1e-2,
                                           pc_shift=0.5, maxiter=600),
        "bbt_n1056_b32": lambda: bbt_case("bbt_n1056_b32", b=32, nblk=32, t=32, sigma=3.0, k=6,
                                          maxsub=40, minsub=16, seed=3),
        # the inner-GMRES configuration (block Jacobi, inner 50 / 1e-3, maxsub
        # 120 / minsub 48) at a CPU-runnable size
        "bbt_n8256_gmres_bj": lambda: bbt_case("bbt_n8256_gmres_bj", b=32, nblk=256, t=64,
                                               sigma=3.0, k=4, maxsub=120, minsub=48,
                                               inner_maxiter=50, inner_tol=1e-3,
                                               pc="block_jacobi", maxiter=1500),
        "sweep": sweep_cases,
        "diag50": diag_case,
        "random200": random_case,
    }
    for name in (args.only.split(",") if args.only else cases):
        cases[name]()


if __name__ == "__main__":
    main()
