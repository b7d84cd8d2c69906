"""CPU restatement of the reference JDQZ (test infrastructure, not product).

This module is the checker for the device engine: a numpy/LAPACK
restatement of the reference's ``bbjd_solve`` (``src/jd_core.c:743-1120``)
with its helpers, step by step, each citing the reference lines it follows.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  It is pinned against the reference itself
(``oracle/_ref``, built from the reference's sources by ``oracle/Makefile``)
by ``tests/test_oracle.py`` and the fixtures under ``tests/golden/``.

The projected QZ and its reordering call the same LAPACK routines as the
reference (ZGGES with an optimal workspace, then ZTGSEN with ijob = 0,
``jd_core.c:343-356, 411-422``) through scipy's bundled OpenBLAS, which is
the library the reference links (``setup.py:36-58``).
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import lapack

SUCCESS, MAX_ITER = 0, 1
ERR_ALLOC, ERR_INVALID, ERR_CALLBACK, ERR_LAPACK, ERR_BREAKDOWN = -1, -2, -3, -4, -5

TARGETS = {"nearest": 0, "LM": 1, "SM": 2, "LR": 3, "SR": 4, "LI": 5, "SI": 6}


def block_orthogonalize(Q: np.ndarray, v: np.ndarray) -> float:
    """CGS with one DGKS re-pass (``jd_core.c:207-241``); v is updated in place."""
    if Q.shape[1] == 0:
        return float(np.linalg.norm(v))
    before = np.linalg.norm(v)
    h = Q.conj().T @ v
    v -= Q @ h
    after = np.linalg.norm(v)
    if after < 0.7071 * before:                       # jd_core.c:232
        h = Q.conj().T @ v
        v -= Q @ h
        after = np.linalg.norm(v)
    return float(after)


def project_out(Q: np.ndarray, v: np.ndarray) -> None:
    """Two unconditional CGS passes (``jd_core.c:269-309``)."""
    if Q.shape[1] == 0:
        return
    for _ in range(2):
        v -= Q @ (Q.conj().T @ v)


def _target_value(lam: complex, sigma: complex, target: int) -> float:
    """The selection key of ``jd_core.c:387-396`` (smaller is better)."""
    if target == 0:
        return abs(lam - sigma)
    if target == 1:
        return -abs(lam)
    if target == 2:
        return abs(lam)
    if target == 3:
        return -lam.real
    if target == 4:
        return lam.real
    if target == 5:
        return -lam.imag
    if target == 6:
        return lam.imag
    return abs(lam - sigma)


def solve_projected(MA, MB, k, sigma, target, nkeep, conv, tol):
    """ZGGES + SELECT + ZTGSEN + target scan (``jd_core.c:319-462``).

    Returns (SA, SB, ZA, ZB, alpha, beta, target_pos) or None on a LAPACK
    failure.
    """
    SA = np.asfortranarray(MA[:k, :k].copy())
    SB = np.asfortranarray(MB[:k, :k].copy())
    sel_all = lambda a, b: 0  # noqa: E731  (sort = 'N')
    # workspace query then the call, as jd_core.c:342-354 does
    q = lapack.zgges(sel_all, SA, SB, lwork=-1)
    lwork = int(q[-2][0].real) + 1
    SA, SB, _sdim, alpha, beta, ZA, ZB, _w, info = lapack.zgges(sel_all, SA, SB, lwork=lwork)
    if info != 0:
        return None
    sel = np.zeros(k, dtype=np.int32)
    for i in range(k):                                  # jd_core.c:365-374
        if abs(beta[i]) < 1e-300:
            continue
        lam = alpha[i] / beta[i]
        for c in conv:
            if abs(lam - c) < tol * 100:
                sel[i] = 1
                break
    for _ in range(nkeep):                              # jd_core.c:379-401
        tidx, best = -1, np.inf
        for i in range(k):
            if sel[i] or abs(beta[i]) < 1e-300:
                continue
            val = _target_value(alpha[i] / beta[i], sigma, target)
            if val < best:
                best, tidx = val, i
        if tidx < 0:
            break
        sel[tidx] = 1
    if sel.sum() > 0:                                   # jd_core.c:407-425
        SA, SB, alpha, beta, ZA, ZB, _m, _pl, _pr, _dif, info = lapack.ztgsen(
            sel, SA, SB, ZA, ZB, ijob=0)
        if info != 0:
            return None
    tpos, best = 0, np.inf                              # jd_core.c:430-458
    for i in range(k):
        if abs(beta[i]) < 1e-300:
            continue
        lam = alpha[i] / beta[i]
        if any(abs(lam - c) < tol * 100 for c in conv):
            continue
        val = _target_value(lam, sigma, target)
        if val < best:
            best, tpos = val, i
    return SA, SB, ZA, ZB, alpha, beta, tpos


def zlartg_stable(f: complex, g: complex):
    """Complex Givens with real cs >= 0 (``jd_core.c:477-511``)."""
    af, ag = abs(f), abs(g)
    if ag < 1e-300:
        return 1.0, 0j, f
    if af < 1e-300:
        return 0.0, np.conj(g) / ag, complex(ag)
    scale = af + ag
    norm = scale * np.sqrt((af / scale) ** 2 + (ag / scale) ** 2)
    return af / norm, (f / af) * np.conj(g) / norm, (f / af) * norm


def correction_gmres(Qr, Ql, theta_a, theta_b, r, mvA, mvB, pc, maxiter, tol):
    """Left-preconditioned GMRES on the projected correction equation
    (``jd_core.c:568-727``).  Returns z, or None when a callback fails."""
    n = r.shape[0]
    ims = maxiter
    V = np.zeros((n, ims + 1), dtype=np.complex128)
    H = np.zeros((ims + 1, ims), dtype=np.complex128)
    cs = np.zeros(ims)
    sn = np.zeros(ims, dtype=np.complex128)
    g = np.zeros(ims + 1, dtype=np.complex128)
    t1 = -r.copy()
    project_out(Ql, t1)                                 # jd_core.c:599-600
    V[:, 0] = pc(t1) if pc is not None else t1
    beta0 = np.linalg.norm(V[:, 0])
    if beta0 < 1e-300:
        return np.zeros(n, dtype=np.complex128)
    V[:, 0] /= beta0
    g[0] = beta0
    j = 0
    while j < ims:
        t1 = V[:, j].copy()
        project_out(Qr, t1)                             # jd_core.c:628-629
        t2 = theta_b * mvA(t1) - theta_a * mvB(t1)      # jd_core.c:632-636
        project_out(Ql, t2)                             # jd_core.c:639
        w = pc(t2) if pc is not None else t2            # jd_core.c:642-646
        before = np.linalg.norm(w)
        for i in range(j + 1):                          # jd_core.c:651-657 (MGS)
            h = np.vdot(V[:, i], w)
            H[i, j] = h
            w = w - h * V[:, i]
        after = np.linalg.norm(w)
        if after < 0.7071 * before:                     # jd_core.c:660-669
            for i in range(j + 1):
                h = np.vdot(V[:, i], w)
                H[i, j] += h
                w = w - h * V[:, i]
            after = np.linalg.norm(w)
        H[j + 1, j] = after
        if after < 1e-14 * before:                      # jd_core.c:674
            j += 1
            break
        V[:, j + 1] = w / after
        for i in range(j):                              # jd_core.c:680-685
            h1, h2 = H[i, j], H[i + 1, j]
            H[i, j] = cs[i] * h1 + sn[i] * h2
            H[i + 1, j] = -np.conj(sn[i]) * h1 + cs[i] * h2
        c, s, rr = zlartg_stable(H[j, j], H[j + 1, j])  # jd_core.c:688-696
        cs[j], sn[j] = c, s
        H[j, j], H[j + 1, j] = rr, 0.0
        g1, g2 = g[j], g[j + 1]                         # jd_core.c:699-703
        g[j] = cs[j] * g1 + sn[j] * g2
        g[j + 1] = -np.conj(sn[j]) * g1 + cs[j] * g2
        if abs(g[j + 1]) < tol * beta0:                 # jd_core.c:705
            j += 1
            break
        j += 1
    m = j
    y = g.copy()
    for i in range(m - 1, -1, -1):                      # jd_core.c:711-716
        for k2 in range(i + 1, m):
            y[i] -= H[i, k2] * y[k2]
        if abs(H[i, i]) > 1e-300:
            y[i] /= H[i, i]
    z = V[:, :m] @ y[:m]                                # jd_core.c:719-721
    project_out(Qr, z)                                  # jd_core.c:724
    return z


def deflation_append(j, Qr, Ql, u, Au, Bu, nu0, mu0):
    """Column j of the deflation projectors (``jd_core.c:516-528``)."""
    qr = u.copy()
    nrm = block_orthogonalize(Qr[:, :j], qr)
    if nrm > 1e-300:
        qr /= nrm
    Qr[:, j] = qr
    ql = nu0 * Au + mu0 * Bu
    nrm = block_orthogonalize(Ql[:, :j], ql)
    if nrm > 1e-300:
        ql /= nrm
    Ql[:, j] = ql


class _Rand:
    """Stand-in for the reference's ``srand(42); rand()`` stream.

    The reference draws its start vector and breakdown vectors from the C
    library's global generator (``jd_core.c:793-799, 1040``).  This
    restatement calls the same glibc ``rand`` through ctypes so that a
    run without ``v0`` starts from the same vector.
    """

    def __init__(self):
        import ctypes
        libc = ctypes.CDLL("libc.so.6")
        self._rand = libc.rand
        self._rand.restype = ctypes.c_int
        libc.srand(42)
        self.RAND_MAX = 2147483647

    def vec(self, n):
        out = np.empty(n, dtype=np.complex128)
        for i in range(n):
            re = self._rand() / self.RAND_MAX - 0.5
            im = self._rand() / self.RAND_MAX - 0.5
            out[i] = re + 1j * im
        return out


def jdqz(n, nev, mvA, mvB, pc=None, sigma=0.0, target=0, tol=1e-10, maxiter=200,
         maxsub=0, minsub=0, inner_maxiter=0, inner_tol=1e-2, v0=None, verbose=0):
    """Restatement of ``bbjd_solve`` (``jd_core.c:743-1120``).

    Returns a dict with eigenvalues, eigenvectors (n x nconv), residuals,
    nconv, iters and status, as the reference's result struct holds them.
    """
    sigma = complex(sigma)
    maxsub_auto = max(3 * nev + 10, 40)                 # jd_core.c:95-98
    maxsub = maxsub if maxsub > 0 else min(maxsub_auto, n)
    minsub = minsub if minsub > 0 else max(2 * nev + 5, 20)   # jd_core.c:750-752
    V = np.zeros((n, maxsub), dtype=np.complex128)
    W = np.zeros_like(V)
    AV = np.zeros_like(V)
    BV = np.zeros_like(V)
    MA = np.zeros((maxsub, maxsub), dtype=np.complex128)
    MB = np.zeros_like(MA)
    Qr = np.zeros((n, nev + 1), dtype=np.complex128)
    Ql = np.zeros_like(Qr)
    evals, evecs, resid = [], [], []
    res = dict(status=SUCCESS, iters=0)

    if target == 0:                                     # jd_core.c:783-789
        sc = 1.0 / np.sqrt(1.0 + abs(sigma) ** 2)
        nu0, mu0 = sc, -sigma * sc
    elif target == 2:
        nu0, mu0 = 1.0, 0.0
    else:
        nu0, mu0 = 0.0, 1.0
    rnd = _Rand()                                       # jd_core.c:793
    if v0 is not None:
        V[:, 0] = v0
    else:
        V[:, 0] = rnd.vec(n)
    nrm = np.linalg.norm(V[:, 0])
    if nrm < 1e-300:
        return _finish(res, evals, evecs, resid, n, ERR_BREAKDOWN)
    V[:, 0] /= nrm
    AV[:, 0] = mvA(V[:, 0])                             # jd_core.c:807-810
    BV[:, 0] = mvB(V[:, 0])
    W[:, 0] = nu0 * AV[:, 0] + mu0 * BV[:, 0]           # jd_core.c:812-816
    W[:, 0] /= np.linalg.norm(W[:, 0])
    MA[0, 0] = np.vdot(W[:, 0], AV[:, 0])               # jd_core.c:818-819
    MB[0, 0] = np.vdot(W[:, 0], BV[:, 0])
    kdim, nlock = 1, 0

    for it in range(maxiter):                           # jd_core.c:823
        k, locked = kdim, nlock
        nkeep = max(minsub - locked, 1)                 # jd_core.c:830-831
        out = solve_projected(MA, MB, k, sigma, target, nkeep, evals, tol)
        if out is None:
            return _finish(res, evals, evecs, resid, n, ERR_LAPACK)
        SA, SB, ZA, ZB, alpha, beta, p = out
        ta, tb = alpha[p], beta[p]
        y = np.zeros(p + 1, dtype=np.complex128)        # jd_core.c:855-867
        y[p] = 1.0
        for i in range(p - 1, -1, -1):
            acc = 0j
            for j in range(i + 1, p + 1):
                acc += (tb * SA[i, j] - ta * SB[i, j]) * y[j]
            d = tb * SA[i, i] - ta * SB[i, i]
            y[i] = -acc / d if abs(d) > 1e-300 else 0.0
        x = ZB[:k, :p + 1] @ y                          # jd_core.c:870-871
        u = V[:, :k] @ x
        nrm = np.linalg.norm(u)
        if nrm < 1e-300:
            return _finish(res, evals, evecs, resid, n, ERR_BREAKDOWN)
        u /= nrm
        Au, Bu = mvA(u), mvB(u)                         # jd_core.c:884-888
        r = tb * Au - ta * Bu
        denom = abs(ta) + abs(tb)
        rel = np.linalg.norm(r) / (denom if denom > 1e-300 else 1.0)
        if verbose >= 2:
            lam = ta / tb if abs(tb) > 1e-300 else ta
            print(f"  iter {it:3d}  kdim {k:3d}  locked {locked:2d}  eig {lam:.6e}  res {rel:.3e}")
        if rel < tol:                                   # jd_core.c:905-932
            lam = ta / tb if abs(tb) > 1e-300 else ta
            evals.append(lam)
            evecs.append(u.copy())
            resid.append(rel)
            if len(evals) >= nev:
                res["iters"] = it + 1
                return _finish(res, evals, evecs, resid, n, SUCCESS)
            deflation_append(nlock, Qr, Ql, u, Au, Bu, nu0, mu0)
            nlock += 1
            continue
        if inner_maxiter > 0:                           # jd_core.c:945-951
            deflation_append(locked, Qr, Ql, u, Au, Bu, nu0, mu0)
            z = correction_gmres(Qr[:, :nlock + 1], Ql[:, :nlock + 1], ta, tb, r, mvA, mvB,
                                 pc, inner_maxiter, inner_tol)
        else:                                           # jd_core.c:952-972
            z = pc(r) if pc is not None else r.copy()
            s = pc(u) if pc is not None else u.copy()
            uz, us = np.vdot(u, z), np.vdot(u, s)
            if abs(us) > 1e-300:
                z = z - (uz / us) * s
        if k >= maxsub:                                 # jd_core.c:975-1030
            keep = minsub if minsub < k else k - 1
            keep = max(keep, locked + 1)
            Z = ZB[:k, :keep]
            V[:, :keep] = V[:, :k] @ Z
            AV[:, :keep] = AV[:, :k] @ Z
            BV[:, :keep] = BV[:, :k] @ Z
            for j in range(keep):                       # jd_core.c:1002-1010
                w = nu0 * AV[:, j] + mu0 * BV[:, j]
                nrm = block_orthogonalize(W[:, :j], w)
                if nrm > 1e-300:
                    w /= nrm
                W[:, j] = w
            MA[:keep, :keep] = W[:, :keep].conj().T @ AV[:, :keep]
            MB[:keep, :keep] = W[:, :keep].conj().T @ BV[:, :keep]
            kdim = k = keep
        v = z.copy()                                    # jd_core.c:1033-1048
        nrm = block_orthogonalize(V[:, :k], v)
        if nrm < 1e-14:
            v = rnd.vec(n)
            nrm = block_orthogonalize(V[:, :k], v)
            if nrm < 1e-14:
                res["iters"] = it + 1
                return _finish(res, evals, evecs, resid, n, ERR_BREAKDOWN)
        V[:, k] = v / nrm
        AV[:, k] = mvA(V[:, k])                         # jd_core.c:1051-1054
        BV[:, k] = mvB(V[:, k])
        w = nu0 * AV[:, k] + mu0 * BV[:, k]             # jd_core.c:1057-1068
        nrm = block_orthogonalize(W[:, :k], w)
        if nrm < 1e-14:
            w = AV[:, k].copy()
            nrm = block_orthogonalize(W[:, :k], w)
        if nrm > 1e-300:
            w /= nrm
        W[:, k] = w
        MA[:k + 1, k] = W[:, :k + 1].conj().T @ AV[:, k]     # jd_core.c:1090-1095
        MB[:k + 1, k] = W[:, :k + 1].conj().T @ BV[:, k]
        MA[k, :k] = W[:, k].conj() @ AV[:, :k]               # jd_core.c:1098-1103
        MB[k, :k] = W[:, k].conj() @ BV[:, :k]
        kdim = k + 1
        res["iters"] = it + 1
    status = MAX_ITER if len(evals) < nev else SUCCESS      # jd_core.c:1110
    return _finish(res, evals, evecs, resid, n, status)


def _finish(res, evals, evecs, resid, n, status):
    res["status"] = status
    res["nconv"] = len(evals)
    res["eigenvalues"] = np.asarray(evals, dtype=np.complex128)
    res["eigenvectors"] = (np.stack(evecs, axis=1) if evecs
                           else np.zeros((n, 0), dtype=np.complex128))
    res["residuals"] = np.asarray(resid, dtype=np.float64)
    return res
