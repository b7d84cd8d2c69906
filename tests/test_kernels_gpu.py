"""Kernel-level parity of the device kernels against host references, through
the C-ABI.  Integer-free floating-point work: tolerances are stated per test
(FP64 throughout; reductions differ from numpy only in summation order)."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import splu

from bbjd_b200 import DevicePencil, DevicePreconditioner, _lib, make_pencil
from oracle import jdqz_np

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def _host(t):
    return t.cpu().numpy()


def _rand(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


SPMV_CASES = [(8, 64, 4), (16, 256, 8), (16, 33, 8), (32, 100, 64), (32, 7, 32), (16, 40, 0),
              (8, 1, 3), (32, 31, 96), (16, 50, 16), (8, 21, 1), (32, 9, 2), (8, 3, 16)]


@pytest.mark.parametrize("b,nblk,t", SPMV_CASES)
def test_bbt_matvec_matches_host(b, nblk, t):
    import torch
    P = make_pencil(b, nblk, t, seed=11)
    dev = DevicePencil(P)
    x = _rand(P.n, 3)
    xd = _dev(x)
    yA = torch.empty_like(xd)
    yB = torch.empty_like(xd)
    lib = _lib.load()
    assert lib.bbjd_bbt_matvec(dev.handle, xd.data_ptr(), yA.data_ptr(), yB.data_ptr(), None) == 0
    torch.cuda.synchronize()
    refA, refB = P.matvec_A(x), P.matvec_B(x)
    # FP64, different summation order: 1e-13 relative to the row scale
    scale = np.abs(x).max() * (np.abs(P.Ad).max() * 3 * b + 1)
    assert np.abs(_host(yA) - refA).max() < 1e-13 * scale
    assert np.abs(_host(yB) - refB).max() < 1e-13 * scale
    assert np.all(_host(yB)[P.nb:] == 0)


LU_CASES = [(8, 64, 4), (16, 33, 8), (16, 256, 8), (32, 100, 64), (8, 1, 2), (8, 2, 0), (32, 3, 32)]


@pytest.mark.parametrize("b,nblk,t", LU_CASES)
@pytest.mark.parametrize("nrhs", [1, 2])
def test_bbt_lu_solve_matches_scipy(b, nblk, t, nrhs):
    import torch
    P = make_pencil(b, nblk, t, seed=5)
    sigma = 3.0 + 0.25j
    dev = DevicePencil(P)
    pc = DevicePreconditioner(dev, sigma, "exact")
    M = (P.to_csc("A") - sigma * P.to_csc("B")).tocsc()
    r = np.stack([_rand(P.n, 10 + q) for q in range(nrhs)])
    rd = _dev(r)
    xd = torch.empty_like(rd)
    lib = _lib.load()
    assert lib.bbjd_precond_solve(pc.handle, nrhs, rd.data_ptr(), xd.data_ptr(), None) == 0
    torch.cuda.synchronize()
    x = _host(xd)
    ref = splu(M)
    for q in range(nrhs):
        # backward error of the device solve, and agreement with SuperLU
        res = np.linalg.norm(M @ x[q] - r[q]) / (sp.linalg.norm(M) * np.linalg.norm(x[q]))
        assert res < 1e-13
        xs = ref.solve(r[q])
        assert np.linalg.norm(x[q] - xs) / np.linalg.norm(xs) < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bbt_lu_graph_replay_matches_direct_launches(precision):
    """On a stream of its own the BCR solve is captured into a CUDA graph at
    the second call with the same buffers and replayed from the third on:
    every call gives the bits the direct launches on the default stream
    give, with fresh right-hand sides in the same buffer between calls."""
    import torch
    P = make_pencil(32, 300, 16, seed=6)
    dev = DevicePencil(P)
    pc = DevicePreconditioner(dev, 3.0 + 0.1j, "exact", precision=precision)
    lib = _lib.load()
    rd = torch.empty((2, P.n), dtype=torch.complex128, device="cuda")
    xd = torch.empty_like(rd)
    ref = torch.empty_like(rd)
    stream = torch.cuda.Stream()
    for call in range(4):
        r = np.stack([_rand(P.n, 40 + 2 * call + q) for q in range(2)])
        rd.copy_(torch.from_numpy(r))
        assert lib.bbjd_precond_solve(pc.handle, 2, rd.data_ptr(), ref.data_ptr(), None) == 0
        torch.cuda.synchronize()
        assert lib.bbjd_precond_solve(pc.handle, 2, rd.data_ptr(), xd.data_ptr(),
                                      stream.cuda_stream) == 0
        stream.synchronize()
        assert torch.equal(xd, ref), call
    pc.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bbt_lu_full_size_backward_error(precision):
    """The benchmark's n = 1,000,064 pencil, whose BCR solve replaces its
    levels below 64 blocks and the top block by the reduced system's dense
    inverse: the 2-RHS solve's backward error, computed on the host with
    the numpy block product, is at the FP64 level (complex64 level for the
    mixed factors)."""
    import torch
    P = make_pencil(32, 31250, 64, seed=0)
    sigma = 3.0
    dev = DevicePencil(P)
    pc = DevicePreconditioner(dev, sigma, "exact", precision=precision)
    r = np.stack([_rand(P.n, 21), _rand(P.n, 22)])
    rd = _dev(r)
    xd = torch.empty_like(rd)
    lib = _lib.load()
    assert lib.bbjd_precond_solve(pc.handle, 2, rd.data_ptr(), xd.data_ptr(), None) == 0
    torch.cuda.synchronize()
    x = _host(xd)
    nA = np.sqrt(sum(np.vdot(a, a).real for a in (P.Ad, P.Al, P.Au, P.E, P.F)))
    nB = np.sqrt(np.vdot(P.Bd, P.Bd).real)
    bound = 1e-13 if precision == "fp64" else 1e-5
    for q in range(2):
        res = P.matvec_A(x[q]) - sigma * P.matvec_B(x[q]) - r[q]
        assert np.linalg.norm(res) / ((nA + abs(sigma) * nB) * np.linalg.norm(x[q])) < bound
    pc.close()
    dev.close()


def test_bbt_lu_in_place():
    import torch
    P = make_pencil(16, 50, 8, seed=1)
    dev = DevicePencil(P)
    pc = DevicePreconditioner(dev, 2.0, "exact")
    r = _rand(P.n, 4)
    rd = _dev(r)
    lib = _lib.load()
    assert lib.bbjd_precond_solve(pc.handle, 1, rd.data_ptr(), rd.data_ptr(), None) == 0
    torch.cuda.synchronize()
    M = (P.to_csc("A") - 2.0 * P.to_csc("B")).tocsc()
    assert np.linalg.norm(M @ _host(rd) - r) / np.linalg.norm(r) < 1e-11


@pytest.mark.parametrize("b,nblk,t", [(8, 20, 4), (32, 10, 64)])
def test_block_jacobi_matches_host(b, nblk, t):
    import torch
    P = make_pencil(b, nblk, t, seed=2)
    sigma = 3.0
    dev = DevicePencil(P)
    pc = DevicePreconditioner(dev, sigma, "block_jacobi")
    r = _rand(P.n, 1)
    rd = _dev(r)
    xd = torch.empty_like(rd)
    lib = _lib.load()
    assert lib.bbjd_precond_solve(pc.handle, 1, rd.data_ptr(), xd.data_ptr(), None) == 0
    torch.cuda.synchronize()
    D = P.Ad - sigma * P.Bd
    ref = np.concatenate([np.linalg.solve(D[j], r[j * b:(j + 1) * b]) for j in range(nblk)] +
                         ([np.linalg.solve(P.F[:, P.nb:], r[P.nb:])] if t else []))
    assert np.linalg.norm(_host(xd) - ref) / np.linalg.norm(ref) < 1e-12


# 64 <= k <= 216: the update and the re-pass dots share one read of Q
# (cgs_tail's fused kernel: three tile buffers up to k = 143, two above);
# other k take the separate dot pass.
# repass=False: v has no large component along Q, so the DGKS flag stays
# down and the re-pass is skipped.
@pytest.mark.parametrize("n,k,repass", [(1000, 0, True), (1000, 1, True), (4104, 37, True),
                                        (100003, 200, True), (50, 50, True), (70, 64, True),
                                        (7001, 105, True), (7001, 143, True), (7001, 144, True),
                                        (7001, 216, True), (7001, 217, True), (70001, 120, False),
                                        (2000, 100, False), (33, 5, False), (100003, 64, True)])
def test_orthogonalize_matches_oracle(n, k, repass):
    import torch
    rng = np.random.default_rng(n + k)
    Q = np.linalg.qr(rng.standard_normal((n, max(k, 1))) + 1j * rng.standard_normal((n, max(k, 1))))[0][:, :k]
    v = _rand(n, 9) + (Q @ _rand(k, 8) * 1000 if k and repass else 0)
    Qd = _dev(np.asfortranarray(Q).T.copy()) if k else _dev(np.zeros(1, np.complex128))
    vd = _dev(v)
    nrm = C.c_double()
    second = C.c_int()
    lib = _lib.load()
    assert lib.bbjd_dev_orthogonalize(n, k, Qd.data_ptr(), n, vd.data_ptr(), C.byref(nrm),
                                      C.byref(second), None) == 0
    vv = v.copy()
    ref_nrm = jdqz_np.block_orthogonalize(Q, vv)
    assert abs(nrm.value - ref_nrm) < 1e-12 * max(1.0, ref_nrm)
    assert np.linalg.norm(_host(vd) - vv) < 1e-12 * np.linalg.norm(v)
    if k:
        # the DGKS decision (reference jd_core.c:232) made on the device
        # matches the host's: a large component along Q forces the re-pass
        after1 = np.linalg.norm(v - Q @ (Q.conj().T @ v))
        assert second.value == int(after1 < 0.7071 * np.linalg.norm(v)) == int(repass)
        assert np.abs(Q.conj().T @ _host(vd)).max() < 1e-12 * np.linalg.norm(v)


# keep <= 128: the TMA-staged kernel (in place); 64-row tiles and 16-column
# K-slices with ragged ends, one- and three-column-tile widths
@pytest.mark.parametrize("n,k,keep", [(1000, 40, 20), (100000, 200, 80), (777, 30, 29), (5000, 150, 128),
                                      (64, 17, 16), (130, 1, 1), (4159, 200, 128), (20000, 97, 33)])
def test_restart_gemm_matches_numpy(n, k, keep):
    import torch
    rng = np.random.default_rng(1)
    X = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    Z = np.asfortranarray(rng.standard_normal((k, keep)) + 1j * rng.standard_normal((k, keep)))
    Xd = _dev(X.T.copy())        # column-major n x k
    lib = _lib.load()
    outd = torch.empty_like(Xd) if keep > 128 else Xd   # in place when one column tile
    zh = np.asfortranarray(Z)
    assert lib.bbjd_dev_restart_gemm(n, k, keep, Xd.data_ptr(), n, zh.ctypes.data, k,
                                     outd.data_ptr(), None) == 0
    out = _host(outd).reshape(-1, n).T[:, :keep]
    ref = X @ Z
    assert np.abs(out - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("n,keep", [(1000, 20), (100000, 80), (3000, 100)])
def test_gram_matches_numpy(n, keep):
    rng = np.random.default_rng(2)
    X = rng.standard_normal((n, keep)) + 1j * rng.standard_normal((n, keep))
    Y = rng.standard_normal((n, keep)) + 1j * rng.standard_normal((n, keep))
    Xd, Yd = _dev(X.T.copy()), _dev(Y.T.copy())
    Cm = np.zeros((keep, keep), np.complex128, order="F")
    lib = _lib.load()
    assert lib.bbjd_dev_gram(n, keep, Xd.data_ptr(), Yd.data_ptr(), n, Cm.ctypes.data, keep, None) == 0
    ref = X.conj().T @ Y
    assert np.abs(Cm - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("b,nblk,t", [(16, 256, 8), (32, 100, 64), (8, 33, 4)])
@pytest.mark.parametrize("kind", ["exact", "block_jacobi"])
def test_mixed_precision_preconditioner(b, nblk, t, kind):
    """complex64 factors, FP64 vectors and arithmetic: the solve agrees with
    the FP64 factors to complex64 accuracy (1e-5 relative here; the outer JD
    iteration supplies the rest)."""
    import torch
    P = make_pencil(b, nblk, t, seed=8)
    dev = DevicePencil(P)
    sigma = 3.0 + 0.1j
    p64 = DevicePreconditioner(dev, sigma, kind, precision="fp64")
    p32 = DevicePreconditioner(dev, sigma, kind, precision="mixed")
    assert p32.solve_bytes(2) < 0.85 * p64.solve_bytes(2)
    r = np.stack([_rand(P.n, 1), _rand(P.n, 2)])
    rd = _dev(r)
    x64, x32 = torch.empty_like(rd), torch.empty_like(rd)
    lib = _lib.load()
    assert lib.bbjd_precond_solve(p64.handle, 2, rd.data_ptr(), x64.data_ptr(), None) == 0
    assert lib.bbjd_precond_solve(p32.handle, 2, rd.data_ptr(), x32.data_ptr(), None) == 0
    torch.cuda.synchronize()
    a, c = _host(x64), _host(x32)
    for q in range(2):
        assert np.linalg.norm(c[q] - a[q]) / np.linalg.norm(a[q]) < 1e-5
