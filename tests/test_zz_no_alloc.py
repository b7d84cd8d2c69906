"""bbjd_dev_orthogonalize_static: the orthogonalisation entry point that
allocates nothing, for callers that cannot call cudaMalloc where they
orthogonalise (a framework that owns all device memory, or a pipeline that
must not stall the device).  Its output must equal the allocating entry
point's, call after call, since every call reuses the same static scratch.
Collected last on purpose (file name), so a run that stops at the first
failure has run every other test already."""
import ctypes as C

import numpy as np
import pytest

from bbjd_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_N, MAX_K = 8388608, 256


def _case(n, k, seed):
    rng = np.random.default_rng(seed)
    Q = np.linalg.qr(rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k)))[0]
    v = rng.standard_normal(n) + 1j * rng.standard_normal(n) + Q @ (rng.standard_normal(k) * 100)
    return Q, v


def _orth(fn, Qd, n, k, v):
    import torch
    vd = torch.from_numpy(v.copy()).to("cuda")
    nrm, second = C.c_double(), C.c_int()
    st = fn(n, k, Qd.data_ptr() if k else 0, n, vd.data_ptr(), C.byref(nrm), C.byref(second), None)
    assert st == 0
    return vd.cpu().numpy(), nrm.value, second.value


@pytest.mark.parametrize("n,k", [(100003, 200), (4104, 37), (1000, 0)])
def test_static_matches_allocating_twice(n, k):
    import torch
    lib = _lib.load()
    Q, v = _case(n, max(k, 1), 5)
    Q = Q[:, :k]
    Qd = torch.from_numpy(np.ascontiguousarray(Q.T)).to("cuda")   # column-major n x k
    ref_v, ref_n, ref_s = _orth(lib.bbjd_dev_orthogonalize, Qd, n, k, v)
    # two calls in a row: the shared scratch keeps the first call's contents
    for _ in range(2):
        got_v, got_n, got_s = _orth(lib.bbjd_dev_orthogonalize_static, Qd, n, k, v)
        # FP64: 1e-12 relative (the kernel tests' bound)
        assert np.linalg.norm(got_v - ref_v) <= 1e-12 * np.linalg.norm(v)
        assert abs(got_n - ref_n) <= 1e-12 * max(1.0, ref_n)
        assert got_s == ref_s


def test_static_allocates_nothing_after_warm_up():
    """After one warm-up call (which, under lazy module loading, loads the
    module holding the static scratch), a call leaves the device's free
    memory unchanged, also at the largest size it accepts."""
    import torch
    lib = _lib.load()
    for n, k in [(4104, 8), (MAX_N, 4)]:
        Qd = torch.randn(k, n, dtype=torch.complex128, device="cuda")   # column-major n x k
        Qd = torch.linalg.qr(Qd.T)[0].T.contiguous()
        vd = torch.randn(n, dtype=torch.complex128, device="cuda")
        ref = vd.clone()
        nrm, second = C.c_double(), C.c_int()
        call = lambda x: lib.bbjd_dev_orthogonalize_static(  # noqa: E731
            n, k, Qd.data_ptr(), n, x.data_ptr(), C.byref(nrm), C.byref(second), None)
        assert call(vd) == 0                      # warm-up
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        vd.copy_(ref)
        assert call(vd) == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        # and the result is orthogonal to Q to FP64 accuracy
        h = torch.mv(Qd.conj(), vd)
        assert float(h.abs().max()) <= 1e-12 * float(ref.norm())
        del Qd, vd, ref
        torch.cuda.empty_cache()


def test_static_rejects_sizes_beyond_its_scratch():
    lib = _lib.load()
    nrm, second = C.c_double(), C.c_int()
    # rejected on the host before anything is launched
    assert lib.bbjd_dev_orthogonalize_static(1000, MAX_K + 1, 1, 1000, 1, C.byref(nrm),
                                             C.byref(second), None) == -2
    assert lib.bbjd_dev_orthogonalize_static(MAX_N + 1, 4, 1, MAX_N + 1, 1, C.byref(nrm),
                                             C.byref(second), None) == -2
