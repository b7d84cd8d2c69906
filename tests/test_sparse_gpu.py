"""The reference's usage pattern on the device path: scipy sparse A, B and a
SparseLU of A - sigma B (reference README.md:36-58) packed into the
block-bordered format and solved on the GPU, checked against the reference's
own golden run and against the same pencil given directly."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import splu

from bbjd_b200 import SparseLU, jdqz, make_pencil, start_vector
from tests.parity import assert_eigs_match, assert_no_duplicates, nearest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    return g, P


def _kw(g, P):
    return dict(k=int(g["k"]), sigma=complex(g["sigma"]), tol=1e-10, maxiter=int(g["maxiter"]),
                maxsub=int(g["maxsub"]), minsub=int(g["minsub"]),
                v0=start_vector(P.n, int(g["seed"]) + 1), return_info=True)


def test_sparse_pencil_runs_the_device_path_bit_identically():
    g, P = _golden("bbt_n516")
    A, B = P.to_csc("A").tocsr(), P.to_csc("B").tocsr()
    ev1, x1, i1 = jdqz(P, preconditioner="exact", timing=True, **_kw(g, P))
    ev2, x2, i2 = jdqz(A, B, preconditioner="exact", timing=True, **_kw(g, P))
    assert i2["device"]["kernel_launches"] > 0       # the device engine ran
    assert i1["iters"] == i2["iters"]
    np.testing.assert_array_equal(ev1, ev2)
    np.testing.assert_array_equal(x1, x2)


@pytest.mark.parametrize("name", ["bbt_n516", "bbt_n4104"])
def test_readme_pattern_with_sparse_lu(name):
    g, P = _golden(name)
    A, B = P.to_csc("A").tocsr(), P.to_csc("B").tocsr()
    sigma = complex(g["sigma"])
    M = (A - sigma * B).tocsr()
    lu = SparseLU(M, colamd=True, pin_dense_rows=True)
    ev, evecs, info = jdqz(A, B, preconditioner=lu, **_kw(g, P))
    assert info["nconv"] == int(g["k"]) and info["status"] == 0
    assert "device" in info
    nA, nB = sp.linalg.norm(A), sp.linalg.norm(B)
    for lam, x in zip(ev, evecs.T):
        r = A @ x - lam * (B @ x)
        assert np.linalg.norm(r) / ((nA + abs(lam) * nB) * np.linalg.norm(x)) < 1e-10
    assert_eigs_match(P, ev, evecs, g["arpack"])
    assert_eigs_match(P, ev, evecs, g["eigenvalues"], ref_resid=g["unscaled_residuals"])
    assert sorted(nearest(ev, g["eigenvalues"])) == list(range(int(g["k"])))
    assert_no_duplicates(ev)
    lu.close()


def test_sparse_lu_solve_matches_superlu():
    P = make_pencil(16, 40, 6, seed=11)
    sigma = 2.0 + 1.0j
    M = (P.to_csc("A") - sigma * P.to_csc("B")).tocsc()
    lu = SparseLU(M)
    ref = splu(M)
    rng = np.random.default_rng(0)
    rhs = rng.standard_normal((P.n, 3)) + 1j * rng.standard_normal((P.n, 3))
    y = lu.solve(rhs)
    y_ref = ref.solve(rhs)
    assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < 1e-10
    y1 = lu.solve(rhs[:, 0])
    assert y1.shape == (P.n,)
    np.testing.assert_allclose(y1, y[:, 0], rtol=0, atol=1e-12 * np.abs(y[:, 0]).max())
    assert np.linalg.norm(M @ y1 - rhs[:, 0]) / np.linalg.norm(rhs[:, 0]) < 1e-10
    lu.close()


def test_non_block_bordered_input_keeps_the_callback_path():
    n = 120
    rng = np.random.default_rng(2)
    A = sp.random(n, n, density=0.1, random_state=3, format="csr") + sp.diags(np.arange(1.0, n + 1))
    B = sp.eye(n, format="csr")
    ev, _, info = jdqz(A.astype(np.complex128), B, k=2, sigma=0.0, tol=1e-10,
                       preconditioner=splu(A.tocsc().astype(np.complex128)), return_info=True,
                       v0=rng.standard_normal(n) + 0j)
    assert info["nconv"] == 2 and "device" not in info
    with pytest.raises(ValueError):
        SparseLU(A)
