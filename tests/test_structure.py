"""Block-bordered structure detection and packing from scipy sparse (CPU)."""
import numpy as np
import pytest
import scipy.sparse as sp

from bbjd_b200 import structure
from bbjd_b200.pencils import make_pencil


def _same(P, Q):
    assert (P.b, P.nblk, P.t) == (Q.b, Q.nblk, Q.t)
    for name in ("Ad", "Al", "Au", "E", "F", "Bd"):
        np.testing.assert_array_equal(getattr(P, name), getattr(Q, name), err_msg=name)


@pytest.mark.parametrize("b,nblk,t", [(8, 20, 5), (16, 12, 3), (32, 6, 2), (16, 10, 0), (8, 9, 128)])
def test_round_trip_csc_csr_dense(b, nblk, t):
    P = make_pencil(b, nblk, t, seed=3)
    A, B = P.to_csc("A"), P.to_csc("B")
    assert structure.detect(A, B) == (b, t)
    _same(structure.pencil_from_sparse(A, B), P)
    _same(structure.pencil_from_sparse(A.tocsr(), B.tocsr()), P)
    _same(structure.pencil_from_sparse(A.toarray(), B.toarray()), P)


def test_small_chunks(monkeypatch):
    monkeypatch.setattr(structure, "_CHUNK", 37)
    P = make_pencil(16, 11, 4, seed=5)
    _same(structure.pencil_from_sparse(P.to_csc("A"), P.to_csc("B")), P)


def test_matvec_of_packed_pencil():
    P = make_pencil(8, 15, 6, seed=7)
    A, B = P.to_csc("A"), P.to_csc("B")
    Q = structure.pencil_from_sparse(A, B)
    x = np.random.default_rng(0).standard_normal(P.n) + 1j
    np.testing.assert_allclose(Q.matvec_A(x), A @ x, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(Q.matvec_B(x), B @ x, rtol=1e-13, atol=1e-13)


def test_identity_b_only_without_tau_rows():
    P = make_pencil(16, 8, 0, seed=1)
    A = P.to_csc("A")
    assert structure.detect(A, None, b_is_identity=True) == (16, 0)
    Q = structure.pencil_from_sparse(A, None)
    np.testing.assert_array_equal(Q.Bd, np.broadcast_to(np.eye(16), Q.Bd.shape))
    P3 = make_pencil(16, 8, 3, seed=1)
    assert structure.detect(P3.to_csc("A"), None, b_is_identity=True) is None


def test_shifted_matrix_for_factorisation():
    P = make_pencil(16, 10, 4, seed=2)
    sigma = 3.0 - 1.5j
    M = (P.to_csc("A") - sigma * P.to_csc("B")).tocsr()
    Q = structure.matrix_from_sparse(M)
    assert (Q.b, Q.t) == (16, 4)
    S = P.shifted(sigma)
    np.testing.assert_allclose(Q.Ad, S.Ad, rtol=1e-15, atol=1e-15)
    np.testing.assert_array_equal(Q.Al, S.Al)
    np.testing.assert_array_equal(Q.E, S.E)
    np.testing.assert_array_equal(Q.F, S.F)
    assert not Q.Bd.any()


def test_rejects_other_structures():
    rng = np.random.default_rng(0)
    R = sp.random(200, 200, density=0.05, random_state=1, format="csr") + sp.eye(200)
    assert structure.detect(R, sp.eye(200)) is None
    assert structure.pencil_from_sparse(R, sp.eye(200)) is None
    # B with an entry in a tau row cannot be held by the format
    P = make_pencil(8, 10, 3, seed=4)
    B = P.to_csc("B").tolil()
    B[P.nb + 1, 2] = 1.0
    assert structure.detect(P.to_csc("A"), B) is None
    # an entry three 8-blocks off the diagonal: the 16-blocks still hold it
    A = P.to_csc("A").tolil()
    A[0, 3 * 8 + 1] = rng.standard_normal()
    assert structure.detect(A.tocsr(), P.to_csc("B")) == (16, 3)
    # a block-tridiagonal matrix with 24 x 24 blocks fits none of 8, 16, 32
    blocks = sp.kron(sp.diags([1.0, 1.0, 1.0], [-1, 0, 1], shape=(8, 8), dtype=np.float64),
                     np.ones((24, 24)))
    assert structure.detect(blocks.tocsr(), None, b_is_identity=True) is None


def test_detected_b_is_smallest_that_fits():
    # a b = 8 pencil is also block-tridiagonal at b = 16 and 32 when nb allows;
    # the smallest block size wins
    P = make_pencil(8, 16, 2, seed=8)
    assert structure.detect(P.to_csc("A"), P.to_csc("B")) == (8, 2)
