"""End-to-end parity of the device JDQZ against the reference's own results
(tests/golden, produced by running the reference) and against ARPACK, on
the block-bordered pencils the reference targets.  See tests/parity.py for
the criteria and their tolerances."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from bbjd_b200 import (DevicePencil, DevicePreconditioner, jdqz, jdqz_device, make_pencil,
                       start_vector)
from tests.parity import (assert_eigs_match, assert_no_duplicates, eig_bound, match_set, nearest,
                          unscaled_residual)

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


def _check_pairs(P, ev, evecs, g, tol=1e-10):
    A, B = P.to_csc("A"), P.to_csc("B")
    nA, nB = sp.linalg.norm(A), sp.linalg.norm(B)
    for lam, x in zip(ev, evecs.T):
        r = A @ x - lam * (B @ x)
        # normalised residual: the acceptance test of the benchmark metric
        assert np.linalg.norm(r) / ((nA + abs(lam) * nB) * np.linalg.norm(x)) < tol
        # the reference test suite's unscaled measure (tests/test_bbjd.py:96-98)
        assert np.linalg.norm(r) / np.linalg.norm(x) < 1e-8
    # each value within its conditioning-aware bound of ARPACK's value
    assert_eigs_match(P, ev, evecs, g["arpack"])
    assert_no_duplicates(ev)


def _same_as_reference(P, ev, evecs, g):
    """The reference's own set, one to one, each value within the bound its
    residual and the reference's give."""
    assert_eigs_match(P, ev, evecs, g["eigenvalues"], ref_resid=g["unscaled_residuals"])
    assert sorted(nearest(ev, g["eigenvalues"])) == list(range(len(g["eigenvalues"])))


@pytest.mark.parametrize("projected,ritz", [("qz", "auto"), ("schur", "fp32"), ("schur", "fp64")])
@pytest.mark.parametrize("name", ["bbt_n516", "bbt_n1056_b32", "bbt_n4104"])
def test_device_jdqz_matches_reference(name, projected, ritz):
    g = _load(name)
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    sigma = complex(g["sigma"])
    ev, evecs, info = jdqz(P, k=int(g["k"]), sigma=sigma, tol=1e-10, maxiter=int(g["maxiter"]),
                           maxsub=int(g["maxsub"]), minsub=int(g["minsub"]),
                           preconditioner="exact", v0=start_vector(P.n, int(g["seed"]) + 1),
                           return_info=True, projected=projected, ritz_estimate=ritz,
                           timing=True)
    assert info["nconv"] == int(g["k"]) and info["status"] == 0
    d = info["device"]
    if projected == "schur" and ritz == "fp32":
        # FP32 estimates ranked the candidates and were refined in FP64
        assert d["ritz_refinements"] > 0
    else:
        assert d["ritz_refinements"] == 0 and d["ritz_fallbacks"] == 0
    _check_pairs(P, ev, evecs, g)
    _same_as_reference(P, ev, evecs, g)
    # same algorithm: the iteration count differs from the reference's only
    # through rounding (the reference itself varies by ~5% with BLAS threads)
    assert abs(info["iters"] - int(g["iters"])) <= max(10, 0.25 * int(g["iters"]))
    # solver-measure residuals below tol, reported per pair
    assert np.all(info["residuals"] < 1e-10)


def test_device_jdqz_gmres_matches_reference():
    g = _load("bbt_n516_gmres")
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    sigma = complex(g["sigma"])
    dev = DevicePencil(P)
    approx = DevicePreconditioner(dev, sigma + complex(g["pc_shift"]), "exact")
    ev, evecs, info = jdqz(dev, k=int(g["k"]), sigma=sigma, tol=1e-10, maxiter=int(g["maxiter"]),
                           maxsub=int(g["maxsub"]), minsub=int(g["minsub"]),
                           inner_maxiter=int(g["inner_maxiter"]), inner_tol=float(g["inner_tol"]),
                           preconditioner=approx, v0=start_vector(P.n, 1), return_info=True)
    assert info["nconv"] == int(g["k"])
    _check_pairs(P, ev, evecs, g)
    _same_as_reference(P, ev, evecs, g)
    assert abs(info["iters"] - int(g["iters"])) <= max(10, 0.25 * int(g["iters"]))


def test_device_jdqz_block_jacobi_gmres():
    """The inner-GMRES configuration's preconditioner on a small pencil."""
    g = _load("bbt_n1056_b32")
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    ev, evecs, info = jdqz(P, k=3, sigma=3.0, tol=1e-10, maxiter=1500, maxsub=40, minsub=16,
                           inner_maxiter=50, inner_tol=1e-3, preconditioner="block_jacobi",
                           v0=start_vector(P.n, 4), return_info=True)
    assert info["nconv"] == 3
    _check_pairs(P, ev, evecs, g)
    # three of the four nearest to sigma in the ARPACK set
    assert set(nearest(ev, g["arpack"])) <= {0, 1, 2, 3}


def test_device_without_preconditioner_and_random_start():
    """No preconditioner (t = r projected, reference jd_core.c:956-965) and
    the seeded random start (v0 = None): on a 66-row pencil the search space
    can grow to hold the wanted eigenvector, so the pair converges."""
    P = make_pencil(8, 8, 2, seed=9)
    ev, evecs, info = jdqz(P, k=1, sigma=3.0, tol=1e-9, maxiter=300, maxsub=60, minsub=30,
                           return_info=True)
    assert info["nconv"] == 1
    A, B = P.to_csc("A"), P.to_csc("B")
    for lam, x in zip(ev, evecs.T):
        assert np.linalg.norm(A @ x - lam * (B @ x)) / np.linalg.norm(x) < 1e-7


def test_device_v0_length_checked():
    P = make_pencil(8, 4, 2)
    with pytest.raises(ValueError):
        jdqz(P, k=1, sigma=3.0, preconditioner="exact", v0=np.ones(P.n - 1))


def test_pinned_arrays_are_the_same_pencil():
    """A pencil uploaded from pinned torch copies of its device arrays (the
    end-to-end input path) is the pencil uploaded from the BBTPencil: the
    same solve gives bitwise the same eigenvalues."""
    import torch
    P = make_pencil(16, 40, 8, seed=2)
    pinned = {k: torch.from_numpy(v.view(np.float64)).pin_memory()
              for k, v in P.device_arrays().items()}
    kw = dict(k=3, sigma=3.0, preconditioner="exact", maxsub=24, minsub=10, maxiter=300,
              v0=start_vector(P.n, 1))
    ev_a = jdqz(P, **kw)[0]
    ev_b = jdqz(DevicePencil(arrays=pinned, b=16, nblk=40, t=8), **kw)[0]
    assert len(ev_a) == 3
    np.testing.assert_array_equal(ev_a, ev_b)


def test_device_stats_reported():
    P = make_pencil(16, 64, 8, seed=0)
    ev, evecs, info = jdqz(P, k=2, sigma=3.0, preconditioner="exact", maxsub=20, minsub=8,
                           maxiter=500, v0=start_vector(P.n, 1), return_info=True, timing=True)
    d = info["device"]
    assert info["nconv"] == 2
    assert d["kernel_launches"] > 0 and d["bytes_device"] > 0
    assert d["kernels"]["spmv"]["calls"] > 0 and d["kernels"]["spmv"]["ms"] > 0
    assert d["restarts"] >= 1


def test_mixed_precision_form_n4104():
    """The mixed-precision form of the n = 4104 configuration: complex64 LU
    factors and a complex64 first CGS pass; every pair still meets the FP64
    residual tolerance and matches the reference's FP64 eigenvalues; the
    iteration count changes by the (reported) amount below."""
    g = _load("bbt_n4104")
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    kw = dict(k=int(g["k"]), sigma=complex(g["sigma"]), tol=1e-10, maxiter=int(g["maxiter"]),
              maxsub=int(g["maxsub"]), minsub=int(g["minsub"]), preconditioner="exact",
              v0=start_vector(P.n, int(g["seed"]) + 1), return_info=True)
    ev64, evecs64, i64 = jdqz(P, precision="fp64", **kw)
    ev32, evecs32, i32 = jdqz(P, precision="mixed", **kw)
    assert i32["nconv"] == int(g["k"])
    _check_pairs(P, ev32, evecs32, g)
    _same_as_reference(P, ev32, evecs32, g)
    # per-eigenvalue error against the FP64 form: within the bound both
    # pairs' residuals give (the outer iteration refines the complex64 work
    # to FP64 accuracy)
    r64 = [unscaled_residual(P, l, x) for l, x in zip(ev64, evecs64.T)]
    err, bnd = assert_eigs_match(P, ev32, evecs32, ev64, ref_resid=r64)
    assert sorted(nearest(ev32, ev64)) == list(range(int(g["k"])))
    # the outer iteration absorbs the complex64 preconditioner: iteration
    # count within 50 % of the FP64 form's
    assert i32["iters"] <= 1.5 * i64["iters"] + 10
    print(f"mixed vs fp64 iterations {i32['iters']} vs {i64['iters']}, "
          f"max |dlambda| vs FP64 {err.max():.2e} (bound {bnd.min():.2e}..{bnd.max():.2e})")


def test_batched_sweep_equals_one_at_a_time():
    """The batched sigma-sweep form (several independent pencils, each with
    its own sigma on Re = 3, solved concurrently on one GPU) returns exactly
    what the same batch returns solved one at a time (concurrency changes
    nothing), the same eigenvalues as single jdqz calls (which may take the
    other LAPACK for the projected eigenvalues), and every pair converges."""
    from bbjd_b200 import jdqz_batch
    rng = np.random.default_rng(4)
    nblks = [int(x) for x in rng.integers(120, 360, size=6)]
    sigmas = [complex(3.0, float(s)) for s in rng.uniform(-40, 40, size=6)]
    pencils = [make_pencil(16, nb, 16, seed=100 + i) for i, nb in enumerate(nblks)]
    kw = dict(k=4, tol=1e-10, maxiter=800, maxsub=40, minsub=16)
    batch, wall = jdqz_batch(pencils, sigmas, threads=4, **kw)
    serial, _ = jdqz_batch(pencils, sigmas, threads=1, **kw)
    for i, (P, s) in enumerate(zip(pencils, sigmas)):
        bev, bvec, binfo = batch[i]
        sev, svec, sinfo = serial[i]
        assert binfo["nconv"] == sinfo["nconv"] == 4
        assert binfo["iters"] == sinfo["iters"]
        assert np.array_equal(bev, sev) and np.array_equal(bvec, svec)
        ev, evecs, info = jdqz(P, sigma=s, preconditioner="exact", v0=start_vector(P.n, 1 + i),
                               return_info=True, **kw)
        assert info["nconv"] == 4
        r1 = [unscaled_residual(P, l, x) for l, x in zip(ev, evecs.T)]
        assert_eigs_match(P, bev, bvec, ev, ref_resid=r1)
        assert sorted(nearest(bev, ev)) == [0, 1, 2, 3]
        A, B = P.to_csc("A"), P.to_csc("B")
        for lam, x in zip(bev, bvec.T):
            assert np.linalg.norm(A @ x - lam * (B @ x)) / np.linalg.norm(x) < 1e-8


def test_jdqz_device_reports_error_vs_oracle():
    g = _load("bbt_n516")
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    ev, evecs, info = jdqz_device(P, k=int(g["k"]), sigma=complex(g["sigma"]), tol=1e-10,
                              maxiter=int(g["maxiter"]), maxsub=int(g["maxsub"]),
                              minsub=int(g["minsub"]), preconditioner="exact",
                              v0=start_vector(P.n, int(g["seed"]) + 1), return_info=True,
                              oracle=g["eigenvalues"])
    assert info["nconv"] == int(g["k"])
    assert info["error_vs_oracle"] == pytest.approx(match_set(ev, g["eigenvalues"]).max())
    err, bnd = assert_eigs_match(P, ev, evecs, g["eigenvalues"], ref_resid=g["unscaled_residuals"])
    assert info["error_vs_oracle"] <= bnd.max()


def test_device_maxiter_returns_partial_result():
    """Stopping at maxiter is not an error (status 1, reference bbjd.py:262-266):
    the pairs found so far come back, with a RuntimeWarning at verbose >= 1."""
    P = make_pencil(16, 64, 8, seed=0)
    with pytest.warns(RuntimeWarning):
        ev, evecs, info = jdqz(P, k=6, sigma=3.0, maxiter=12, maxsub=20, minsub=8,
                               preconditioner="exact", v0=start_vector(P.n, 1),
                               return_info=True, verbose=1)
    assert info["status"] == 1 and info["nconv"] < 6
    assert ev.shape == (info["nconv"],) and evecs.shape == (P.n, info["nconv"])
    assert len(info["residuals"]) == info["nconv"]


@pytest.mark.parametrize("bad", [dict(k=0), dict(tol=-1.0), dict(k=10_000)])
def test_device_invalid_parameters_raise(bad):
    P = make_pencil(8, 16, 2, seed=0)
    kw = dict(k=2, sigma=3.0, tol=1e-10, preconditioner="exact", v0=start_vector(P.n, 1))
    kw.update(bad)
    # as the reference: a parameter the C core rejects is a RuntimeError, a
    # workspace it cannot allocate a MemoryError (reference _bbjd_c.c:199-200)
    with pytest.raises((RuntimeError, ValueError, MemoryError)):
        jdqz(P, **kw)


def test_host_overlap_changes_no_result():
    """The target guessed from the previous one and checked against the FP32
    estimates computed on a second host thread while the device iterates
    (host_overlap='auto') gives bit for bit what the same rule gives with the
    estimates computed first ('off'): same pairs, iterations, guess counts
    and convergence iterations.  The pencil has restarts and locks."""
    g = _load("bbt_n4104")
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    kw = dict(k=int(g["k"]), sigma=complex(g["sigma"]), tol=1e-10, maxiter=int(g["maxiter"]),
              maxsub=int(g["maxsub"]), minsub=int(g["minsub"]), preconditioner="exact",
              v0=start_vector(P.n, int(g["seed"]) + 1), return_info=True)
    ev_a, x_a, ia = jdqz(P, host_overlap="auto", **kw)
    ev_b, x_b, ib = jdqz(P, host_overlap="off", **kw)
    assert ia["nconv"] == int(g["k"]) and ia["iters"] == ib["iters"]
    np.testing.assert_array_equal(ev_a, ev_b)
    np.testing.assert_array_equal(x_a, x_b)
    da, db = ia["device"], ib["device"]
    assert da["guess_hits"] == db["guess_hits"] > 0
    assert da["guess_misses"] == db["guess_misses"]
    assert da["restarts"] >= 1
    np.testing.assert_array_equal(da["conv_iters"], db["conv_iters"])
    ci = da["conv_iters"]
    assert len(ci) == ia["nconv"] and np.all(np.diff(ci) >= 0) and ci[-1] < ia["iters"]
    # both runs hold the parity bounds
    _check_pairs(P, ev_a, x_a, g)
    _same_as_reference(P, ev_a, x_a, g)


def test_full_size_first_pairs_match_reference_run():
    """The benchmark's n = 1,000,064 pencil (b = 32, 31,250 blocks, t = 64,
    sigma = 3, maxsub 200, minsub 80), 200 outer iterations from the same
    start vector as the reference's own C core run cached in
    tests/golden/bbt_n1000064.npz: the same pairs converge at the same
    iterations (within two), each eigenvalue within its conditioning-aware
    bound of ARPACK's and of the reference's value, and each pair passes the
    normalised residual test computed on the host with the numpy block
    product, independently of the device kernels."""
    g = _load("bbt_n1000064")
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    its = 200
    ref_iter = g["ref_conv_iter"]
    ref_ev = g["ref_eigenvalues"][ref_iter < its]
    ref_res = g["ref_residuals"][ref_iter < its] * (1.0 + np.abs(ref_ev))   # unscaled
    ev, evecs, info = jdqz(P, k=int(g["k"]), sigma=complex(g["sigma"]), tol=float(g["tol"]),
                           maxiter=its, maxsub=int(g["maxsub"]), minsub=int(g["minsub"]),
                           preconditioner="exact", v0=start_vector(P.n, int(g["v0_seed"])),
                           return_info=True)
    assert info["nconv"] == len(ref_ev) >= 1
    assert sorted(nearest(ev, ref_ev)) == list(range(len(ref_ev)))
    ci = info["device"]["conv_iters"]
    assert np.all(np.abs(ci - ref_iter[ref_iter < its][nearest(ev, ref_ev)]) <= 2), (ci, ref_iter)
    assert_eigs_match(P, ev, evecs, g["arpack"], kappas=g["arpack_kappa"])
    kap_ref = g["arpack_kappa"][nearest(ref_ev, g["arpack"])]
    assert_eigs_match(P, ev, evecs, ref_ev, ref_resid=ref_res, kappas=kap_ref)
    nA = np.sqrt(sum(np.vdot(a, a).real for a in (P.Ad, P.Al, P.Au, P.E, P.F)))
    nB = np.sqrt(np.vdot(P.Bd, P.Bd).real)
    for lam, x in zip(ev, evecs.T):
        assert unscaled_residual(P, lam, x) / (nA + abs(lam) * nB) < 1e-10
    assert np.all(info["residuals"] < 1e-10)
    assert_no_duplicates(ev)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_full_size_bench_solve_pairs_in_oracle_set(precision):
    """The benchmark solve itself (n = 1,000,064, k = 64, maxsub 200, minsub
    80, tol 1e-10, 2,000 outer iterations, both forms): every returned pair
    passes the normalised residual test on the host (numpy block product,
    independent of the device kernels), every eigenvalue lies within its
    conditioning-aware bound of one of ARPACK's 80 eigenvalues nearest sigma
    (tests/golden/bbt_n1000064.npz), no eigenvalue is returned twice, and
    the set shares all but two of its members with the reference's own run
    of the same 2,000 iterations (its distinct values), whose path parts
    from this one after a few hundred iterations."""
    g = _load("bbt_n1000064")
    P = make_pencil(int(g["b"]), int(g["nblk"]), int(g["t"]), seed=int(g["seed"]))
    ev, evecs, info = jdqz(P, k=int(g["k"]), sigma=complex(g["sigma"]), tol=float(g["tol"]),
                           maxiter=int(g["ref_maxiter"]), maxsub=int(g["maxsub"]),
                           minsub=int(g["minsub"]), preconditioner="exact",
                           v0=start_vector(P.n, int(g["v0_seed"])), return_info=True,
                           precision=precision)
    assert info["nconv"] >= 8
    nA = np.sqrt(sum(np.vdot(a, a).real for a in (P.Ad, P.Al, P.Au, P.E, P.F)))
    nB = np.sqrt(np.vdot(P.Bd, P.Bd).real)
    for lam, x in zip(ev, evecs.T):
        assert unscaled_residual(P, lam, x) / (nA + abs(lam) * nB) < 1e-10
    assert_eigs_match(P, ev, evecs, g["arpack"], kappas=g["arpack_kappa"])
    assert_no_duplicates(ev)
    ref = []
    for lam in g["ref_eigenvalues"]:
        if all(abs(lam - d) > 1e-6 * max(1.0, abs(lam)) for d in ref):
            ref.append(lam)
    same = sum(1 for lam in ev if np.min(np.abs(np.asarray(ref) - lam)) <= 1e-8 * abs(lam))
    assert same >= min(len(ev), len(ref)) - 2, (ev, ref)
