"""Generate the full-size golden fixture (n = 1,000,064) by running the reference.

The benchmark pencil (b = 32, 31,250 blocks, t = 64, sigma = 3, k = 64,
maxsub = 200, minsub = 80, tol = 1e-10, seed 0, start vector seed 1) is
solved on the CPU by:

* the reference's own C core (``oracle/_ref``, built from the reference's
  ``src/jd_core.c`` and ``src/_bbjd_c.c`` by ``oracle/Makefile``), driven
  through its extension function ``jdqz_c`` with numpy block products and
  the C block-bordered LU (``oracle/c``) as its operators, for ``--maxiter``
  outer iterations.  It runs in a child process at verbose level 2; this
  process timestamps every per-iteration line the child prints, so the
  fixture holds the reference's own convergence history (which value
  converged at which iteration, returned duplicates included) and its
  wall time per outer iteration against the subspace dimension;
* ARPACK shift-invert (``scipy.sparse.linalg.eigs`` on
  ``(A - sigma B)^-1 B`` through the same LU), the ``--n-arpack`` eigenvalues
  nearest sigma;
* the condition number ``1 / |y^H B x|`` of each ARPACK eigenvalue (unit
  left and right eigenvectors by inverse iteration with the exact LU of
  ``A - lam B`` and of its conjugate transpose), which sets the parity
  tests' conditioning-aware eigenvalue bound.

Both take hours on a few cores, so their output is cached as
``tests/golden/bbt_n1000064.npz``; the GPU tests and ``bench.py`` read it.

    python tests/golden/make_golden_n1e6.py [--maxiter 2000] [--threads 6] [--procs 3]
                                            [--kappa-count 24]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASE = dict(b=32, nblk=31250, t=64, sigma=3.0, k=64, maxsub=200, minsub=80, tol=1e-10)
OUT = os.path.join(HERE, "bbt_n1000064.npz")

_ITER = re.compile(r"iter\s+(\d+)\s+kdim\s+(\d+)\s+locked\s+(\d+)\s+eig \(([-+.\deE]+), ([-+.\deE]+)\)"
                   r"\s+res ([-+.\deE]+)")
_CONV = re.compile(r"converged #(\d+): \(([-+.\deE]+), ([-+.\deE]+)\)\s+res ([-+.\deE]+)\s+iter (\d+)")


def child(maxiter: int, out: str) -> None:
    """Run the reference's C core on the pencil (stderr: its verbose log)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import _bbjd_c  # the reference's C core, built from its sources

    from bbjd_b200.pencils import make_pencil, start_vector
    from oracle.bbt_lu import BBTLUHost
    c = CASE
    P = make_pencil(c["b"], c["nblk"], c["t"], seed=0)
    lu = BBTLUHost(P, c["sigma"])
    v0 = start_vector(P.n, 1)
    sys.stderr.write("START\n")
    sys.stderr.flush()
    t0 = time.time()
    ev, _, resid, nconv, iters, status = _bbjd_c.jdqz_c(
        n=P.n, nev=c["k"], sigma=c["sigma"], target=0, matvec_A=P.matvec_A,
        matvec_B=P.matvec_B, precond_solve=lu.solve, tol=c["tol"], maxiter=maxiter,
        maxsub=c["maxsub"], minsub=c["minsub"], inner_maxiter=0, inner_tol=1e-2, verbose=2, v0=v0)
    np.savez(out, eigenvalues=np.asarray(ev)[:nconv], residuals=np.asarray(resid)[:nconv],
             nconv=nconv, iters=iters, status=status, seconds=time.time() - t0)


def run_reference(maxiter: int, threads: int) -> dict:
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads))
    tmp = tempfile.mktemp(suffix=".npz")
    proc = subprocess.Popen([sys.executable, os.path.abspath(__file__), "--child", tmp,
                             "--maxiter", str(maxiter)], env=env, stderr=subprocess.PIPE,
                            text=True, bufsize=1)
    rows, convs, t_start = [], [], [None]

    def reader():
        for line in proc.stderr:
            now = time.monotonic()
            if line.startswith("START"):
                t_start[0] = now
                continue
            m = _ITER.search(line)
            if m:
                rows.append((int(m[1]), int(m[2]), int(m[3]), float(m[4]), float(m[5]),
                             float(m[6]), now))
                if len(rows) % 100 == 0:
                    print(f"  reference iteration {m[1]} kdim {m[2]} locked {m[3]} "
                          f"{now - t_start[0]:.0f} s", flush=True)
                continue
            m = _CONV.search(line)
            if m:
                convs.append((int(m[1]), float(m[2]), float(m[3]), float(m[4]), int(m[5])))
                print("  " + line.strip(), flush=True)

    th = threading.Thread(target=reader, daemon=True)
    th.start()
    rc = proc.wait()
    th.join()
    if rc != 0:
        raise RuntimeError(f"reference child exited {rc}")
    d = dict(np.load(tmp))
    os.unlink(tmp)
    it = np.array([r[0] for r in rows], dtype=np.int64)
    tt = np.array([r[6] for r in rows]) - t_start[0]
    return dict(ref_eigenvalues=d["eigenvalues"], ref_residuals=d["residuals"],
                ref_nconv=int(d["nconv"]), ref_iters=int(d["iters"]), ref_status=int(d["status"]),
                ref_seconds=float(d["seconds"]), ref_threads=threads,
                ref_conv_iter=np.array([c[4] for c in convs], dtype=np.int64),
                ref_iter=it, ref_kdim=np.array([r[1] for r in rows], dtype=np.int64),
                ref_locked=np.array([r[2] for r in rows], dtype=np.int64),
                ref_res=np.array([r[5] for r in rows]), ref_time=tt)


def run_arpack(n_arpack: int, threads: int) -> dict:
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    from scipy.sparse.linalg import LinearOperator, eigs

    from bbjd_b200.pencils import make_pencil
    from oracle.bbt_lu import BBTLUHost
    c = CASE
    P = make_pencil(c["b"], c["nblk"], c["t"], seed=0)
    lu = BBTLUHost(P, c["sigma"])
    op = LinearOperator((P.n, P.n), matvec=lambda x: lu.solve(P.matvec_B(np.asarray(x).ravel())),
                        dtype=np.complex128)
    t0 = time.time()
    mu, X = eigs(op, k=n_arpack, which="LM", tol=1e-13, v0=np.ones(P.n, np.complex128))
    lam = c["sigma"] + 1.0 / mu
    order = np.argsort(np.abs(lam - c["sigma"]))
    lam, X = lam[order], X[:, order]
    # residual of each ARPACK pair in the normalised measure
    nA = np.sqrt(sum(np.linalg.norm(a) ** 2 for a in (P.Ad, P.Al, P.Au, P.E, P.F)))
    nB = np.linalg.norm(P.Bd)
    res = np.array([np.linalg.norm(P.matvec_A(X[:, j]) - lam[j] * P.matvec_B(X[:, j]))
                    / ((nA + abs(lam[j]) * nB) * np.linalg.norm(X[:, j])) for j in range(len(lam))])
    print(f"  arpack: {len(lam)} values in {time.time() - t0:.0f} s, max residual {res.max():.2e}",
          flush=True)
    return dict(arpack=lam, arpack_residuals=res, arpack_seconds=time.time() - t0)


def _kappa_chunk(lams):
    from bbjd_b200.pencils import make_pencil
    from tests.parity import eig_condition
    c = CASE
    P = make_pencil(c["b"], c["nblk"], c["t"], seed=0)
    return [eig_condition(P, lam) for lam in lams]


def run_kappa(lams, threads: int, procs: int = 1, count: int = 0) -> dict:
    """Condition numbers of `lams` (the first `count` of them when count > 0,
    NaN for the rest: ARPACK's values come sorted by distance to sigma, and
    each costs two factorisations of ~2 minutes), split over `procs`
    processes (spawned: each builds the pencil and factors its own LUs,
    ~10 GB each)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    t0 = time.time()
    lams = np.asarray(lams)
    rest = None
    if 0 < count < len(lams):
        rest = np.full(len(lams) - count, np.nan)
        lams = lams[:count]
    if procs <= 1:
        kap = np.array(_kappa_chunk(lams))
    else:
        import multiprocessing as mp
        chunks = [c for c in np.array_split(lams, procs) if len(c)]
        with mp.get_context("spawn").Pool(len(chunks)) as pool:
            kap = np.concatenate([np.asarray(k) for k in pool.map(_kappa_chunk, chunks)])
    if rest is not None:
        kap = np.concatenate([kap, rest])
    print(f"  kappa of {len(lams)} values in {time.time() - t0:.0f} s: "
          f"{np.nanmin(kap):.1f} .. {np.nanmax(kap):.1f}", flush=True)
    return dict(arpack_kappa=kap)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--maxiter", type=int, default=2000)
    ap.add_argument("--threads", type=int, default=6)
    ap.add_argument("--n-arpack", type=int, default=80)
    ap.add_argument("--procs", type=int, default=1, help="processes for the condition numbers")
    ap.add_argument("--kappa-count", type=int, default=0,
                    help="condition numbers for the nearest this many ARPACK values only (0: all)")
    ap.add_argument("--only", choices=["reference", "arpack", "kappa"], default=None)
    ap.add_argument("--child", default=None)
    args = ap.parse_args()
    if args.child:
        child(args.maxiter, args.child)
        return
    out = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    out.update({k: v for k, v in CASE.items()}, seed=0, v0_seed=1)
    if args.only in (None, "reference"):
        out.update(run_reference(args.maxiter, args.threads), ref_maxiter=args.maxiter)
        np.savez(OUT, **out)
    if args.only in (None, "arpack"):
        out.update(run_arpack(args.n_arpack, args.threads))
        np.savez(OUT, **out)
    if args.only in (None, "kappa"):
        out.update(run_kappa(out["arpack"], args.threads, args.procs, args.kappa_count))
        np.savez(OUT, **out)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
