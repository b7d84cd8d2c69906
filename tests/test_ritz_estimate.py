"""The property the default projected solve relies on: between restarts,
complex64 estimates of the harmonic projected eigenvalues rank the
candidates like FP64 ones, so the target that is then refined in FP64 is the
one the FP64 ranking picks.  Checked on the projected pencils of the numpy
oracle's own JDQZ run on a pencil with the bench's block structure
(b = 32, t = 64; smaller n).  CPU only: numpy's complex64 eigensolver
stands in for the library's CGEEV / CHSEQR."""
import numpy as np
from scipy.sparse.linalg import splu

from bbjd_b200.pencils import make_pencil, start_vector
from oracle import jdqz_np


def test_complex64_ranking_picks_the_fp64_target(monkeypatch):
    P = make_pencil(32, 64, 64, seed=0)
    A, B = P.to_csc("A"), P.to_csc("B")
    sigma = 3.0
    lu = splu((A - sigma * B).tocsc())
    sc = 1 / np.sqrt(1 + abs(sigma) ** 2)
    nu0, mu0 = sc, -sigma * sc                        # harmonic pair of the engine
    seen = []
    orig = jdqz_np.solve_projected

    def pick(w, conv, tol):
        lam = (1 / w - mu0) / nu0
        free = [l for l in lam
                if not any(abs(l - c) < max(tol * 100, 1e-6 * max(1, abs(l))) for c in conv)]
        return min(free, key=lambda l: abs(l - sigma)) if free else None

    def record(MA, MB, k, sig, target, nkeep, conv, tol):
        H = np.linalg.solve(nu0 * MA[:k, :k] + mu0 * MB[:k, :k], MB[:k, :k])
        l64 = pick(np.linalg.eigvals(H), conv, tol)
        l32 = pick(np.linalg.eigvals(H.astype(np.complex64)).astype(np.complex128), conv, tol)
        if l64 is not None:
            seen.append((l64, l32))
        return orig(MA, MB, k, sig, target, nkeep, conv, tol)

    monkeypatch.setattr(jdqz_np, "solve_projected", record)
    out = jdqz_np.jdqz(P.n, 6, lambda x: A @ x, lambda x: B @ x, lu.solve, sigma=sigma, tol=1e-10,
                       maxiter=200, maxsub=60, minsub=24, v0=start_vector(P.n, 1))
    assert out["nconv"] >= 2 and len(seen) == out["iters"]
    for l64, l32 in seen:
        # the same candidate, its complex64 value within ~1e-6 relative
        assert l32 is not None and abs(l64 - l32) <= 1e-5 * max(1.0, abs(l64))
