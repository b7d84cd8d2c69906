"""The CPU oracle (oracle/jdqz_np.py) pinned against the reference's own
outputs (tests/golden, produced by running the reference) and against the
known answers of the reference's test suite.  CPU only."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import splu

from bbjd_b200.pencils import make_pencil, start_vector
from oracle import jdqz_np
from tests.parity import (SUITE_ATOL, adjoint_pencil, assert_eigs_match, assert_no_duplicates,
                           eig_bound, eig_condition, match_set, nearest)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


def _run_bbt(g):
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    A, B = P.to_csc("A"), P.to_csc("B")
    sigma = complex(g["sigma"])
    lu = splu((A - (sigma + complex(g["pc_shift"])) * B).tocsc())
    out = jdqz_np.jdqz(P.n, int(g["k"]), lambda x: A @ x, lambda x: B @ x, lu.solve,
                       sigma=sigma, tol=1e-10, maxiter=int(g["maxiter"]), maxsub=int(g["maxsub"]),
                       minsub=int(g["minsub"]), inner_maxiter=int(g["inner_maxiter"]),
                       inner_tol=float(g["inner_tol"]), v0=start_vector(P.n, int(g["seed"]) + 1))
    return P, A, B, out


@pytest.mark.parametrize("name", ["bbt_n516", "bbt_n516_gmres", "bbt_n1056_b32"])
def test_oracle_matches_reference_bbt(name):
    g = _load(name)
    P, A, B, out = _run_bbt(g)
    assert out["nconv"] == int(g["nconv"])
    ev, X = out["eigenvalues"], out["eigenvectors"]
    # each value within its conditioning-aware bound of ARPACK's and of the
    # reference run's value, one to one with the reference's set
    assert_eigs_match(P, ev, X, g["arpack"])
    assert_eigs_match(P, ev, X, g["eigenvalues"], ref_resid=g["unscaled_residuals"])
    assert sorted(nearest(ev, g["eigenvalues"])) == list(range(int(g["nconv"])))
    # the iteration path follows the reference's closely (rounding only)
    assert abs(out["iters"] - int(g["iters"])) <= max(10, 0.25 * int(g["iters"]))
    for lam, x in zip(out["eigenvalues"], out["eigenvectors"].T):
        assert np.linalg.norm(A @ x - lam * (B @ x)) / np.linalg.norm(x) < 1e-8
    assert_no_duplicates(out["eigenvalues"])


def test_oracle_diagonal_known_answer():
    """Reference test_diagonal_5_nearest_sigma0 (tests/test_bbjd.py:162-174)."""
    d = 0.1 * np.arange(1, 51, dtype=np.complex128)
    A = sp.diags(d, format="csc")
    lu = splu(A)
    out = jdqz_np.jdqz(50, 5, lambda x: A @ x, lambda x: x.copy(), lu.solve, sigma=0.0,
                       tol=1e-10, maxiter=200)
    assert out["nconv"] == 5
    assert np.allclose(np.sort(out["eigenvalues"].real), [0.1, 0.2, 0.3, 0.4, 0.5], atol=1e-10)
    g = _load("diag50")
    assert np.allclose(np.sort(out["eigenvalues"].real), np.sort(g["eigenvalues"].real), atol=1e-10)


def test_oracle_small_n_and_start_vector():
    """Reference test_small_n and test_start_vector (tests/test_bbjd.py:335-347, 444-457)."""
    A = sp.diags([1.0, 2.0, 3.0, 4.0, 5.0], dtype=np.complex128, format="csc")
    lu = splu(A)
    out = jdqz_np.jdqz(5, 2, lambda x: A @ x, lambda x: x.copy(), lu.solve, sigma=0.0)
    assert out["nconv"] == 2
    assert np.allclose(np.sort(out["eigenvalues"].real), [1.0, 2.0], atol=1e-10)
    d = 0.1 * np.arange(1, 21, dtype=np.complex128)
    A = sp.diags(d, format="csc")
    lu = splu(A)
    v0 = np.zeros(20, np.complex128)
    v0[0] = 1.0
    out = jdqz_np.jdqz(20, 1, lambda x: A @ x, lambda x: x.copy(), lu.solve, sigma=0.0, v0=v0)
    assert out["nconv"] == 1 and out["iters"] == 1
    assert abs(out["eigenvalues"][0] - 0.1) < 1e-12


def test_oracle_random_sparse_matches_reference():
    g = _load("random200")
    n = int(g["n"])
    A = sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=(n, n)).tocsc()
    sigma = complex(g["sigma"])
    lu = splu((A - sigma * sp.eye(n, format="csc")).tocsc())
    out = jdqz_np.jdqz(n, 6, lambda x: A @ x, lambda x: x.copy(), lu.solve, sigma=sigma,
                       tol=1e-10, maxiter=500, maxsub=150, minsub=60)
    assert out["nconv"] == 6
    assert match_set(out["eigenvalues"], g["arpack"]).max() < SUITE_ATOL
    assert match_set(out["eigenvalues"], g["eigenvalues"]).max() < SUITE_ATOL


@pytest.mark.parametrize("name", ["bbt_n4104", "bbt_n516", "bbt_n1056_b32", "bbt_n516_gmres"])
def test_golden_reference_agrees_with_arpack(name):
    """The pinned reference outputs themselves lie on ARPACK's spectrum,
    each within the conditioning-aware bound its own residual gives (the
    bound the device results are held to; it is not loose: the reference's
    worst value uses 0.35 of it)."""
    g = _load(name)
    assert int(g["nconv"]) == int(g["k"])
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    ref = g["arpack"]
    for lam, r in zip(g["eigenvalues"], g["unscaled_residuals"]):
        i = int(np.argmin(np.abs(ref - lam)))
        kap = eig_condition(P, ref[i])
        assert abs(lam - ref[i]) <= eig_bound(lam, kap, r)


def test_bound_detects_a_wrong_value():
    """A reference value moved by ten times its first-order error estimate
    fails the bound (the check can fail)."""
    g = _load("bbt_n4104")
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    lam, r = g["eigenvalues"][0], g["unscaled_residuals"][0]
    ref = g["arpack"][int(np.argmin(np.abs(g["arpack"] - lam)))]
    kap = eig_condition(P, ref)
    moved = ref + 10 * eig_bound(lam, kap, r)
    assert abs(moved - ref) > eig_bound(moved, kap, r)


def test_adjoint_pencil_is_the_conjugate_transpose():
    P = make_pencil(8, 6, 3, seed=2)
    lam = 3.0 + 0.4j
    M = (P.to_csc("A") - lam * P.to_csc("B")).toarray()
    H = adjoint_pencil(P, lam).to_csc("A").toarray()
    np.testing.assert_allclose(H, M.conj().T, rtol=0, atol=1e-14)


@pytest.mark.parametrize("b,nblk,t", [(8, 64, 4), (16, 33, 8), (32, 5, 32), (8, 1, 2), (4, 10, 0)])
def test_c_restatement_lu_matches_superlu(b, nblk, t):
    """The C block-bordered LU (oracle/c/bbt_oracle.c) against SuperLU."""
    from oracle.bbt_lu import BBTLUHost
    P = make_pencil(b, nblk, t, seed=4)
    sigma = 3.0 + 0.5j
    M = (P.to_csc("A") - sigma * P.to_csc("B")).tocsc()
    lu = BBTLUHost(P, sigma)
    rng = np.random.default_rng(0)
    r = rng.standard_normal(P.n) + 1j * rng.standard_normal(P.n)
    x = lu.solve(r)
    assert np.linalg.norm(M @ x - r) / np.linalg.norm(r) < 1e-11
    xs = splu(M).solve(r)
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-9
