"""Device path for every target of the reference (`which`, reference
bbjd.py:48-56, jd_core.c:387-396) and for pencils without tau rows (B
invertible), checked against the numpy restatement of the reference's
algorithm (oracle/jdqz_np.py) on the same inputs."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import splu

from bbjd_b200 import jdqz, make_pencil, start_vector
from oracle import jdqz_np
from tests.parity import assert_eigs_match, assert_no_duplicates, match_set, nearest

pytestmark = pytest.mark.gpu

TARGETS = {"nearest": 0, "LM": 1, "SM": 2, "LR": 3, "SR": 4, "LI": 5, "SI": 6}


def _residuals_ok(A, B, ev, evecs, tol=1e-8):
    for lam, x in zip(ev, evecs.T):
        assert np.linalg.norm(A @ x - lam * (B @ x)) / np.linalg.norm(x) < tol


KEY = {"nearest": lambda z: abs(z - (3.0 + 2.0j)), "LM": lambda z: -abs(z), "SM": abs,
       "LR": lambda z: -z.real, "SR": lambda z: z.real, "LI": lambda z: -z.imag,
       "SI": lambda z: z.imag}
# direction in which each target's shift sits beyond the end of the spectrum
AWAY = {"LR": 1.0, "SR": -1.0, "LI": 1.0j, "SI": -1.0j}


@pytest.mark.parametrize("which", list(TARGETS))
def test_device_targets_match_oracle(which):
    # t = 0: B = blockdiag(I + 0.1 noise) is invertible, so every target is
    # a finite, well-defined end of the spectrum
    P = make_pencil(8, 24, 0, seed=4)
    A, B = P.to_csc("A"), P.to_csc("B")
    lam = np.linalg.eigvals(np.linalg.solve(B.toarray(), A.toarray()))
    best = sorted(lam, key=KEY[which])
    # the shift a user picks for the preconditioner: near the wanted end
    if which == "nearest":
        sigma = 3.0 + 2.0j
    elif which == "SM":
        sigma = 0.0
    elif which == "LM":
        sigma = best[0] * (1 + 0.5 / abs(best[0]))
    else:
        sigma = best[0] + 0.5 * AWAY[which]
    kw = dict(sigma=sigma, tol=1e-10, maxiter=1500, maxsub=60, minsub=24)
    v0 = start_vector(P.n, 2)
    lu = splu((A - sigma * B).tocsc())
    ev, evecs, info = jdqz(P, k=2, which=which, preconditioner="exact", v0=v0, return_info=True,
                           **kw)
    ref = jdqz_np.jdqz(P.n, 2, lambda x: A @ x, lambda x: B @ x, lu.solve, target=TARGETS[which],
                       v0=v0, **kw)
    assert info["nconv"] == ref["nconv"] == 2
    _residuals_ok(A, B, ev, evecs)
    # each value within its conditioning-aware bound of the exact (dense)
    # eigenvalue, and the same two the oracle returns
    lam_arr = np.asarray(lam)
    assert_eigs_match(P, ev, evecs, lam_arr)
    assert sorted(nearest(ev, lam_arr)) == sorted(nearest(ref["eigenvalues"], lam_arr))
    assert_no_duplicates(ev)
    # the 2 found lie among the 6 best of the dense spectrum
    assert match_set(ev, best[:6]).max() < 1e-6


def test_tau_free_pencil_with_identity_b_runs_on_device():
    # A block-tridiagonal without tau rows and B = None (the identity): the
    # sparse input is recognised (t = 0) and solved on the device; the
    # reference's callback path (host splu preconditioner) gives the same set
    P = make_pencil(16, 40, 0, seed=6)
    A = P.to_csc("A").tocsr()
    sigma = 2.0 - 1.0j
    v0 = start_vector(P.n, 3)
    kw = dict(k=4, sigma=sigma, tol=1e-10, maxiter=800, maxsub=40, minsub=16, v0=v0,
              return_info=True)
    ev, evecs, info = jdqz(A, None, preconditioner="exact", **kw)
    assert "device" in info and info["nconv"] == 4
    I = sp.eye(P.n, format="csr", dtype=np.complex128)
    ev_cb, x_cb, info_cb = jdqz(A, None, preconditioner=splu((A - sigma * I).tocsc()), **kw)
    assert "device" not in info_cb and info_cb["nconv"] == 4
    _residuals_ok(A, I, ev, evecs)
    Pi = make_pencil(16, 40, 0, seed=6)
    Pi.Bd[:] = np.eye(16)
    r_cb = [np.linalg.norm(A @ x - l * x) / np.linalg.norm(x) for l, x in zip(ev_cb, x_cb.T)]
    assert_eigs_match(Pi, ev, evecs, ev_cb, ref_resid=r_cb)
    assert sorted(nearest(ev, ev_cb)) == [0, 1, 2, 3]
