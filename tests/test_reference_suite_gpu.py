"""The reference's own test cases (tests/test_bbjd.py there), run against
bbjd_b200.jdqz through the host-callback path: scipy matrices as operators,
SuperLU as the preconditioner, the subspace work on the GPU.  The known
answers are the reference's."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import LinearOperator, splu

from bbjd_b200 import jdqz, jdqz_c
from tests.parity import match_set

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
# Size multiplier of the scalable cases, as the reference suite's BBJD_PMULT
# (1 = the quick sizes; 10 catches more numerical issues in minutes).
PMULT = int(os.environ.get("BBJD_PMULT", "1"))


class LU:
    def __init__(self, M):
        self._lu = splu(sp.csc_matrix(M))

    def solve(self, b):
        return self._lu.solve(b)


def diagonal(n, spacing=0.1):
    d = np.arange(1, n + 1, dtype=np.complex128) * spacing
    return sp.diags(d, format="csr"), sp.eye(n, format="csr", dtype=np.complex128)


def residual(A, B, lam, x):
    return np.linalg.norm(A @ x - lam * (B @ x)) / np.linalg.norm(x)


def test_diagonal_5_nearest_sigma0():            # reference :162-174
    A, B = diagonal(50 * PMULT)
    ev, _, info = jdqz(A, B, k=5, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=True,
                       maxiter=200)
    assert info["nconv"] == 5
    assert np.allclose(np.sort(ev.real), [0.1, 0.2, 0.3, 0.4, 0.5], atol=1e-10)


def test_diagonal_nearest_to_interior_sigma():   # reference :176-209
    n = 50
    A, B = diagonal(n)
    sigma = 5.05
    ev, _, info = jdqz(A, B, k=3, sigma=sigma, tol=1e-10, preconditioner=LU(A - sigma * B),
                       return_info=True)
    assert info["nconv"] >= 3
    allv = 0.1 * np.arange(1, n + 1)
    d = np.abs(allv - sigma)
    ok = set(np.round(allv[d <= np.sort(d)[2] + 1e-12], 10))
    for e in ev[:3]:
        assert round(float(e.real), 10) in ok


def test_residuals_below_tol():                  # reference :211-220
    A, B = diagonal(50 * PMULT)
    ev, evecs, info = jdqz(A, B, k=5, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=True)
    for j in range(info["nconv"]):
        assert residual(A, B, ev[j], evecs[:, j]) < 100 * 1e-10


def test_random_sparse_vs_reference_and_arpack():  # reference :235-261
    g = dict(np.load(os.path.join(GOLDEN, "random200.npz")))
    n = int(g["n"])
    A = sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=(n, n))
    B = sp.eye(n, format="csr", dtype=np.complex128)
    sigma = complex(g["sigma"])
    ev, evecs, info = jdqz(A, B, k=6, sigma=sigma, tol=1e-10, preconditioner=LU(A - sigma * B),
                           return_info=True, maxiter=500, maxsub=150, minsub=60)
    assert info["nconv"] == 6
    assert match_set(ev, g["arpack"]).max() < 1e-8
    assert match_set(ev, g["eigenvalues"]).max() < 1e-8
    for j in range(6):
        assert residual(A, B, ev[j], evecs[:, j]) < 1e-8


def test_no_preconditioner():                    # reference :321-333
    A, B = diagonal(20)
    _, _, info = jdqz(A, B, k=2, sigma=0.0, tol=1e-8, return_info=True, maxiter=500)
    assert info["nconv"] >= 1


def test_small_n():                              # reference :335-347
    A = sp.diags([1.0, 2.0, 3.0, 4.0, 5.0], dtype=np.complex128, format="csr")
    B = sp.eye(5, format="csr", dtype=np.complex128)
    ev, _, info = jdqz(A, B, k=2, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=True)
    assert info["nconv"] == 2
    assert np.allclose(np.sort(ev.real), [1.0, 2.0], atol=1e-10)


def test_request_subset_of_eigenvalues():        # reference :349-360
    A, B = diagonal(20)
    _, _, info = jdqz(A, B, k=5, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=True,
                      maxiter=200)
    assert info["nconv"] == 5


def test_complex_sigma():                        # reference :362-385
    n = 30
    np.random.seed(7)
    d = np.arange(1, n + 1, dtype=np.complex128) + 0.1j * np.random.randn(n)
    A = sp.diags(d, format="csr")
    B = sp.eye(n, format="csr", dtype=np.complex128)
    sigma = 15.0 + 0.1j
    ev, _, info = jdqz(A, B, k=3, sigma=sigma, tol=1e-10, preconditioner=LU(A - sigma * B),
                       return_info=True)
    assert info["nconv"] == 3
    assert max(abs(e - sigma) for e in ev) < 3.0


def test_return_arity_and_shapes():              # reference :393-416
    A, B = diagonal(20)
    out = jdqz(A, B, k=2, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=False)
    assert len(out) == 2 and out[0].shape == (2,) and out[1].shape == (20, 2)
    out = jdqz(A, B, k=2, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=True)
    assert len(out) == 3 and {"nconv", "iters", "status", "residuals"} <= set(out[2])


def test_dense_and_linear_operator_inputs():     # reference :418-442
    A, B = diagonal(10)
    _, _, info = jdqz(A.toarray(), B.toarray(), k=2, sigma=0.0, tol=1e-10,
                      preconditioner=LU(sp.csr_matrix(A)), return_info=True)
    assert info["nconv"] == 2
    Aop = LinearOperator((10, 10), matvec=lambda x: A @ x, dtype=np.complex128)
    Bop = LinearOperator((10, 10), matvec=lambda x: B @ x, dtype=np.complex128)
    _, _, info = jdqz(Aop, Bop, k=2, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=True)
    assert info["nconv"] == 2


def test_start_vector():                         # reference :444-457
    A, B = diagonal(20)
    v0 = np.zeros(20, np.complex128)
    v0[0] = 1.0
    ev, _, info = jdqz(A, B, k=1, sigma=0.0, tol=1e-10, preconditioner=LU(A), v0=v0,
                       return_info=True)
    assert info["nconv"] == 1 and info["iters"] == 1
    assert abs(ev[0] - 0.1) < 1e-12
    with pytest.raises(ValueError):
        jdqz(A, B, k=1, sigma=0.0, preconditioner=LU(A), v0=v0[:-1])


def test_inner_gmres_with_approximate_preconditioner():   # reference :459-479
    g = dict(np.load(os.path.join(GOLDEN, "random200.npz")))
    n = int(g["n"])
    A = sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=(n, n))
    B = sp.eye(n, format="csr", dtype=np.complex128)
    sigma = 5.0
    approx = LU(A - (sigma + 0.5) * B)
    iters = {}
    for inner in (0, 20):
        ev, evecs, info = jdqz(A, B, k=2, sigma=sigma, tol=1e-10, maxiter=300,
                               preconditioner=approx, inner_maxiter=inner, inner_tol=1e-2,
                               return_info=True)
        assert info["nconv"] == 2
        assert match_set(ev, g["arpack"]).max() < 1e-8
        for j in range(2):
            assert residual(A, B, ev[j], evecs[:, j]) < 1e-8
        iters[inner] = info["iters"]
    assert iters[20] <= iters[0]


def test_verbose_does_not_crash():               # reference :481-496
    A, B = diagonal(20)
    ev, _, info = jdqz(A, B, k=2, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=True,
                       verbose=2)
    assert info["nconv"] == 2
    assert np.allclose(np.sort(ev.real), [0.1, 0.2], atol=1e-10)


def test_clustered_eigenvalues():                # reference :509-525
    d = np.array([1.0, 1.001, 1.002, 2.0, 3.0, 4.0, 5.0], dtype=np.complex128)
    A = sp.diags(d, format="csr")
    B = sp.eye(7, format="csr", dtype=np.complex128)
    sigma = 0.9995
    ev, _, info = jdqz(A, B, k=3, sigma=sigma, tol=1e-10, preconditioner=LU(A - sigma * B),
                       return_info=True, maxiter=500, maxsub=30, minsub=10)
    assert info["nconv"] == 3
    assert np.allclose(np.sort(ev.real), [1.0, 1.001, 1.002], atol=1e-8)


def test_repeated_eigenvalue():                  # reference :527-543
    d = np.array([1.0, 2.0, 2.0, 3.0, 4.0], dtype=np.complex128)
    A = sp.diags(d, format="csr")
    B = sp.eye(5, format="csr", dtype=np.complex128)
    ev, _, info = jdqz(A, B, k=3, sigma=2.0, tol=1e-10, preconditioner=LU(A), return_info=True,
                       maxiter=300)
    assert info["nconv"] >= 2
    for e in ev[:info["nconv"]]:
        assert min(abs(e - x) for x in (1.0, 2.0, 3.0, 4.0)) < 1e-8


def test_schur_locking_no_reconverge():          # reference :580-598
    A, B = diagonal(20)
    ev, _, info = jdqz(A, B, k=5, sigma=0.0, tol=1e-10, preconditioner=LU(A), return_info=True,
                       maxiter=300)
    assert info["nconv"] == 5
    got = np.sort(ev.real)
    assert np.all(np.diff(got) > 0.05)


def test_thick_restart_preserves_locked():       # reference :601-618
    g = dict(np.load(os.path.join(GOLDEN, "random200.npz")))
    n = int(g["n"])
    A = sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=(n, n))
    B = sp.eye(n, format="csr", dtype=np.complex128)
    _, _, info = jdqz(A, B, k=4, sigma=5.0, tol=1e-10, preconditioner=LU(A - 5.0 * B),
                      return_info=True, maxiter=2000, maxsub=30, minsub=15)
    assert info["nconv"] >= 2


def test_callback_exception_propagates():
    """A Python exception in an operator reaches the caller (reference
    _bbjd_c.c:47, 212-216)."""
    A, B = diagonal(10)

    def bad(x):
        raise KeyError("boom")
    with pytest.raises(KeyError):
        jdqz_c(10, 2, 0.0, 0, bad, lambda x: B @ x, None)


def test_jdqz_c_tuple_contract():
    A, B = diagonal(12)
    lu = LU(A)
    ev, evecs, res, nconv, iters, status = jdqz_c(12, 2, 0.0, 0, lambda x: A @ x, lambda x: B @ x,
                                                  lu.solve, tol=1e-10)
    assert nconv == 2 and status == 0 and evecs.shape == (12, 2) and res.shape == (2,)
    assert np.all(res < 1e-10) and iters >= 1


def _golden_random():
    g = dict(np.load(os.path.join(GOLDEN, "random200.npz")))
    n = int(g["n"])
    A = sp.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=(n, n))
    return g, A, sp.eye(n, format="csr", dtype=np.complex128)


def test_random_fewer_eigenvalues():               # reference :263-279
    from scipy.sparse.linalg import eigs
    g, A, B = _golden_random()
    sigma = complex(g["sigma"])
    ref, _ = eigs(A, k=3, sigma=sigma, which="LM")
    ev, _, info = jdqz(A, B, k=3, sigma=sigma, tol=1e-10, preconditioner=LU(A - sigma * B),
                       return_info=True, maxiter=500)
    assert info["nconv"] == 3
    assert match_set(ev, ref).max() < 1e-8


def test_target_found_after_locking():             # reference :556-578
    # after the first lock the target is scanned for over all positions,
    # not read from position `locked`: all three pairs converge
    g, A, B = _golden_random()
    sigma = complex(g["sigma"])
    _, _, info = jdqz(A, B, k=3, sigma=sigma, tol=1e-10, preconditioner=LU(A - sigma * B),
                      return_info=True, maxiter=500, maxsub=150, minsub=60)
    assert info["nconv"] == 3


def _banded_with_tau(n, bandwidth=7, n_tau=4, shift=3.0, seed=123):
    """Banded random matrix with dense leading rows (spectral-PDE shape, the
    reference suite's block-banded + tau case), B = I."""
    rng = np.random.default_rng(seed)
    offsets = list(range(-bandwidth, bandwidth + 1))
    diags = [rng.standard_normal(n - abs(o)) + 0.1j * rng.standard_normal(n - abs(o)) for o in offsets]
    A = sp.diags(diags, offsets, shape=(n, n), format="lil", dtype=np.complex128)
    for i in range(n_tau):
        A[i, :] = rng.standard_normal(n) + 0.1j * rng.standard_normal(n)
    A = A.tocsr() + shift * sp.eye(n, dtype=np.complex128)
    return A, sp.eye(n, format="csr", dtype=np.complex128)


def test_block_banded_tau():                       # reference :290-318
    import scipy.linalg as sl
    A, B = _banded_with_tau(300 * PMULT)
    sigma = 3.0 + 0j
    lam = sl.eigvals(A.toarray())
    ref = lam[np.argsort(np.abs(lam - sigma))[:6]]
    ev, evecs, info = jdqz(A, B, k=6, sigma=sigma, tol=1e-10, preconditioner=LU(A - sigma * B),
                           return_info=True, maxiter=500, maxsub=150, minsub=60)
    assert info["nconv"] == 6
    assert match_set(ev, ref).max() < 1e-8
    for j in range(6):
        assert residual(A, B, ev[j], evecs[:, j]) < 1e-8


def test_larger_random():                          # reference :631-647
    n = 500 * PMULT
    rng = np.random.default_rng(42)
    density = 0.02 if n <= 1000 else min(0.02, 50.0 / n)   # nnz ~ n at large sizes
    A = sp.random(n, n, density=density, format="csr", dtype=np.complex128, random_state=7)
    A = A + 5 * sp.eye(n, dtype=np.complex128)
    A.data += 0.1j * rng.standard_normal(A.nnz)
    B = sp.eye(n, format="csr", dtype=np.complex128)
    sigma = 5.0 + 0j
    _, _, info = jdqz(A, B, k=5, sigma=sigma, tol=1e-10, preconditioner=LU(A - sigma * B),
                      return_info=True, maxiter=500, maxsub=100, minsub=40)
    assert info["nconv"] >= 3
