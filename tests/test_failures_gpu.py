"""Failure detection with injected faults on the host (none faults a GPU).

NaN or Inf reaching the solve -- from a host callback, the start vector or
the pencil itself -- ends it with BBJD_ERR_BREAKDOWN ("subspace breakdown",
a RuntimeError in Python), the status the reference maps a breakdown to
(reference include/bbjd.h:70-78, bbjd.py:248-257), instead of iterating on
non-finite numbers until maxiter.  A callback that fails returns
BBJD_ERR_CALLBACK, and a Python exception inside a callback propagates
unchanged (reference _bbjd_c.c:212-216)."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import LinearOperator, splu

from bbjd_b200 import jdqz, make_pencil, start_vector

pytestmark = pytest.mark.gpu


def _callback_pencil():
    P = make_pencil(8, 32, 4, seed=3)
    A, B = P.to_csc("A").tocsr(), P.to_csc("B").tocsr()
    lu = splu((A - 3.0 * B).tocsc())
    return P, A, B, lu


class _NaNAfter:
    """A matvec that returns NaN from its `after`-th call on."""

    def __init__(self, M, after, value=np.nan):
        self.M, self.after, self.calls, self.value = M, after, 0, value

    def __call__(self, x):
        self.calls += 1
        y = self.M @ x
        if self.calls >= self.after:
            y[len(y) // 2] = self.value
        return y


@pytest.mark.parametrize("value", [np.nan, np.inf])
def test_nonfinite_callback_result_is_a_breakdown(value):
    P, A, B, lu = _callback_pencil()
    mv = _NaNAfter(A, after=7, value=value)
    with pytest.raises(RuntimeError, match="breakdown"):
        jdqz(LinearOperator(A.shape, matvec=mv, dtype=np.complex128), B, k=2, sigma=3.0,
             tol=1e-10, maxiter=200, maxsub=20, minsub=8, preconditioner=lu,
             v0=start_vector(P.n, 1))
    assert mv.calls < 20          # stopped at once, not after maxiter


def test_nonfinite_preconditioner_result_is_a_breakdown():
    P, A, B, lu = _callback_pencil()

    class BadLU:
        calls = 0

        def solve(self, b):
            self.calls += 1
            x = lu.solve(b)
            if self.calls >= 3:
                x[0] = np.nan
            return x

    with pytest.raises(RuntimeError, match="breakdown"):
        jdqz(A, B, k=2, sigma=3.0, tol=1e-10, maxiter=200, maxsub=20, minsub=8,
             preconditioner=BadLU(), v0=start_vector(P.n, 1))


def test_nonfinite_start_vector_is_a_breakdown():
    P = make_pencil(8, 32, 4, seed=3)
    v0 = start_vector(P.n, 1)
    v0[5] = np.nan
    with pytest.raises(RuntimeError, match="breakdown"):
        jdqz(P, k=2, sigma=3.0, preconditioner="exact", v0=v0)


def test_nonfinite_device_pencil_is_a_breakdown():
    """An Inf in a block of the device pencil (no preconditioner, so no
    factorisation meets it first)."""
    P = make_pencil(8, 32, 4, seed=3)
    P.Au[4, 2, 3] = np.inf
    with pytest.raises(RuntimeError, match="breakdown"):
        jdqz(P, k=2, sigma=3.0, maxiter=50, maxsub=20, minsub=8, v0=start_vector(P.n, 1))


def test_failing_callback_status_and_python_exception():
    P, A, B, lu = _callback_pencil()

    def boom(x):
        raise KeyError("matvec failed")

    with pytest.raises(KeyError):
        jdqz(LinearOperator(A.shape, matvec=boom, dtype=np.complex128), B, k=2, sigma=3.0,
             preconditioner=lu, v0=start_vector(P.n, 1))
    # the solve after a failed one runs normally (no state left behind)
    ev, _ = jdqz(A, B, k=2, sigma=3.0, tol=1e-10, maxiter=300, maxsub=20, minsub=8,
                 preconditioner=lu, v0=start_vector(P.n, 1))
    assert len(ev) == 2
    assert sp.issparse(A)
