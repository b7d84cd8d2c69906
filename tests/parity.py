"""Parity criteria shared by the tests (not collected by pytest).

JDQZ is not deterministic at the iteration level (BLAS threading and
rounding change the path; the reference itself returns 383-398 iterations
on the same pencil), so parity is defined on the returned set:

1. each returned pair has a small residual, in the reference's own measure
   ``||theta_b A u - theta_a B u|| / (|theta_a| + |theta_b|)`` and in the
   normalised measure ``||Ax - lam Bx|| / ((||A||_F + |lam| ||B||_F) ||x||)``;
2. each returned eigenvalue lies within a conditioning-aware bound of an
   eigenvalue of the FP64 reference set (ARPACK shift-invert values, and the
   reference's own jdqz run): a pair with residual ``r = Ax - lam Bx`` is,
   to first order, ``|y^H r| / |y^H B x|`` away from the eigenvalue whose
   unit left and right eigenvectors are ``y`` and ``x``, so
   ``|lam - lam_ref| <= 2 kappa (||r_dev|| + ||r_ref||) / ||x|| + 1e-12 max(1, |lam|)``
   with ``kappa = 1 / |y^H B x|``: the first-order bound, doubled for the
   second-order terms and the estimate of kappa (the reference and ARPACK
   differ by up to 7e-9 on these pencils, where kappa reaches ~60: at most
   0.35 of that bound);
3. no eigenvalue is returned twice.

Where no condition number is available (pencils that are not block-
bordered) the reference suite's own flat bound 1e-8 applies
(reference tests/test_bbjd.py:257, 309).
"""
from __future__ import annotations

import numpy as np

# the reference test suite's bound against ARPACK (reference tests/test_bbjd.py:257, 309)
SUITE_ATOL = 1e-8
# slack over the first-order bound kappa ||r||, and the floor that covers the
# oracle set's own error (ARPACK at tol 1e-13 on (A - sigma B)^-1 B)
KAPPA_FACTOR = 2.0
FLOOR_REL = 1e-12


def normalized_residual(matA, matB, lam, x, normA, normB):
    r = matA(x) - lam * matB(x)
    return np.linalg.norm(r) / ((normA + abs(lam) * normB) * np.linalg.norm(x))


def match_set(got, ref):
    """For each value in got, distance to the nearest value in ref."""
    ref = np.asarray(ref)
    return np.array([np.min(np.abs(ref - g)) for g in np.asarray(got)])


def nearest(got, ref):
    """Index in ref of the nearest value, for each value in got."""
    ref = np.asarray(ref)
    return np.array([int(np.argmin(np.abs(ref - g))) for g in np.asarray(got)], dtype=int)


def assert_no_duplicates(vals, rel=1e-6):
    vals = np.asarray(vals)
    for i in range(len(vals)):
        for j in range(i + 1, len(vals)):
            assert abs(vals[i] - vals[j]) > rel * max(1.0, abs(vals[i])), \
                f"duplicate eigenvalue {vals[i]} / {vals[j]}"


def adjoint_pencil(P, lam):
    """(A - lam B)^H as a block-bordered pencil with B = 0.

    The conjugate transpose of a block-bordered matrix whose B has zero tau
    rows is again block-bordered: diagonal blocks (Ad_j - lam Bd_j)^H,
    lower blocks Au_{j-1}^H, upper blocks Al_{j+1}^H, border columns
    F[:, :nb]^H and tau rows [E^H | F[:, nb:]^H]."""
    from bbjd_b200.pencils import BBTPencil
    h = lambda a: np.conj(np.transpose(a, (0, 2, 1)))  # noqa: E731
    Ad = h(P.Ad - lam * P.Bd)
    Al = np.zeros_like(P.Al)
    Au = np.zeros_like(P.Au)
    Al[1:] = h(P.Au[:-1])
    Au[:-1] = h(P.Al[1:])
    nb = P.nb
    E = np.ascontiguousarray(np.conj(P.F[:, :nb]).T)
    F = np.ascontiguousarray(np.conj(np.concatenate([P.E, P.F[:, nb:]], axis=0)).T)
    return BBTPencil(P.b, P.nblk, P.t, np.ascontiguousarray(Ad), Al, Au, E, F,
                     np.zeros_like(P.Bd))


def eig_condition(P, lam, steps=3, seed=7):
    """kappa = 1 / |y^H B x| for unit right and left eigenvectors x, y of the
    block-bordered pencil P at its eigenvalue nearest lam, by inverse
    iteration with the exact block-bordered LU of A - lam B and of its
    conjugate transpose (oracle/c)."""
    from oracle.bbt_lu import BBTLUHost
    rng = np.random.default_rng(seed)
    lr = BBTLUHost(P, lam)
    ll = BBTLUHost(adjoint_pencil(P, lam), 0.0)
    x = rng.standard_normal(P.n) + 1j * rng.standard_normal(P.n)
    y = rng.standard_normal(P.n) + 1j * rng.standard_normal(P.n)
    for _ in range(steps):
        x = lr.solve(x)
        x /= np.linalg.norm(x)
        y = ll.solve(y)
        y /= np.linalg.norm(y)
    return 1.0 / abs(np.vdot(y, P.matvec_B(x)))


def eig_bound(lam, kappa, resid_abs):
    """Conditioning-aware bound on |lam - lam_exact| for a pair whose
    unscaled residual ||A x - lam B x|| / ||x|| is resid_abs."""
    return KAPPA_FACTOR * kappa * resid_abs + FLOOR_REL * max(1.0, abs(lam))


def unscaled_residual(P, lam, x):
    return np.linalg.norm(P.matvec_A(x) - lam * P.matvec_B(x)) / np.linalg.norm(x)


def assert_eigs_match(P, ev, evecs, ref, ref_resid=None, kappas=None):
    """Every (lam, x) in (ev, evecs) lies within eig_bound of its nearest
    value in ref.  ref_resid: the unscaled residuals of the ref values (None
    for an ARPACK set, whose error the floor covers); kappas: condition
    numbers of the ref values (computed when None).  Returns the observed
    errors and their bounds."""
    ref = np.asarray(ref)
    idx = nearest(ev, ref)
    errs, bounds = [], []
    for j, (lam, x) in enumerate(zip(ev, np.asarray(evecs).T)):
        i = idx[j]
        kap = kappas[i] if kappas is not None else eig_condition(P, lam)
        assert np.isfinite(kap), f"{lam}: no condition number cached for its oracle value {ref[i]}"
        r = unscaled_residual(P, lam, x)
        if ref_resid is not None:
            r += ref_resid[i]
        err, bnd = abs(lam - ref[i]), eig_bound(lam, kap, r)
        assert err <= bnd, f"{lam}: |lam - ref| = {err:.3e} > bound {bnd:.3e} (kappa {kap:.1f})"
        errs.append(err)
        bounds.append(bnd)
    return np.array(errs), np.array(bounds)
