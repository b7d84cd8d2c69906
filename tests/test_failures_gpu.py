"""Failure detection with injected faults on the host (none faults a GPU).

NaN or Inf reaching the solve -- from a host callback, the start vector or
the pencil itself -- ends it with BBJD_ERR_BREAKDOWN ("subspace breakdown",
a RuntimeError in Python), the status the reference maps a breakdown to
(reference include/bbjd.h:70-78, bbjd.py:248-257), instead of iterating on
non-finite numbers until maxiter.  A callback that fails returns
BBJD_ERR_CALLBACK, and a Python exception inside a callback propagates
unchanged (reference _bbjd_c.c:212-216).  A device-side wait that runs out
(the TMA-staged restart GEMM's mbarrier waits, made to wait for bytes that
never come) returns BBJD_ERR_DEVICE_TIMEOUT and leaves the context usable."""
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


def test_restart_gemm_wait_that_runs_out_is_a_device_timeout():
    """Every stage of the stalled variant expects 16 bytes more than its TMA
    loads bring, so no wait completes: each gives up after ~1 ms, the kernel
    writes nothing and reports a timeout.  The same GEMM right after runs
    normally on the same context."""
    import torch

    from bbjd_b200 import _lib
    lib = _lib.load()
    n, k, keep = 1000, 40, 20
    rng = np.random.default_rng(2)
    X = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    Z = np.asfortranarray(rng.standard_normal((k, keep)) + 1j * rng.standard_normal((k, keep)))
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to("cuda")     # column-major n x k
    before = Xd.clone()
    st = lib.bbjd_dev_restart_gemm_stalled(n, k, keep, Xd.data_ptr(), n, Z.ctypes.data, k,
                                           Xd.data_ptr(), None)
    assert st == -7                                     # BBJD_ERR_DEVICE_TIMEOUT
    assert torch.equal(Xd, before)                      # nothing written
    assert lib.bbjd_dev_restart_gemm(n, k, keep, Xd.data_ptr(), n, Z.ctypes.data, k,
                                     Xd.data_ptr(), None) == 0
    out = Xd.cpu().numpy().reshape(-1, n).T[:, :keep]
    ref = X @ Z
    assert np.abs(out - ref).max() < 1e-12 * np.abs(ref).max()
