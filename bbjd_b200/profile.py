"""Short device JDQZ run of a block-bordered pencil, for profilers.

    python -m bbjd_b200.profile [--b 32] [--nblk 31250] [--t 64] [--k 64]
                                [--iters 30] [--maxsub 200] [--minsub 80]
                                [--preconditioner exact|block_jacobi]
                                [--inner-maxiter 0] [--inner-tol 1e-2]
                                [--projected auto|qz|schur] [--lock robust|reference]
                                [--precision fp64|mixed] [--verbose 0|1|2]
                                [--ritz-estimate auto|fp64|fp32]
    python -m bbjd_b200.profile --sweep 32 [--threads 16] [--maxiter 2000]

Builds the seeded pencil, uploads it, factors the exact LU (or the block
Jacobi preconditioner) of A - 3 B on the device, runs `iters` outer JDQZ
iterations and prints the per-kernel-class CUDA-event times and algorithmic
bandwidths.  The defaults are the n = 1,000,064 benchmark pencil; a smaller
--nblk gives a case small enough for multi-pass ncu captures; with
--inner-maxiter > 0 the correction equation is solved by GMRES.  --sweep N
runs the batched sweep of N pencils instead (sweep() below).
"""
from __future__ import annotations

import argparse
import time

from . import DevicePencil, DevicePreconditioner, jdqz, make_pencil, start_vector


def sweep(count: int, threads: int, precision: str, maxiter: int, seed: int = 7):
    """The batched sweep: `count` pencils with b = t = 16 and n drawn
    uniformly in [5e4, 3e5], sigma_j = 3 + i U[-40, 40], k = 16, maxsub 80,
    minsub 32, solved concurrently on one GPU."""
    import numpy as np

    from . import jdqz_batch
    rng = np.random.default_rng(seed)
    ns = rng.uniform(5e4, 3e5, size=count)
    sig = rng.uniform(-40.0, 40.0, size=count)
    t0 = time.time()
    pencils = [make_pencil(16, int((n - 16) // 16), 16, seed=1000 + i) for i, n in enumerate(ns)]
    gen = time.time() - t0
    out, wall = jdqz_batch(pencils, [complex(3.0, s) for s in sig], k=16, tol=1e-10,
                           maxiter=maxiter, maxsub=80, minsub=32, precision=precision,
                           threads=threads)
    pairs = sum(o[2]["nconv"] for o in out)
    slow = max(o[2]["seconds"] for o in out)
    print(f"sweep count={count} threads={threads} precision={precision} gen={gen:.1f}s "
          f"wall={wall:.2f}s pairs={pairs} eigenpairs/s={pairs / wall:.2f} slowest_solve={slow:.2f}s "
          f"iters={[o[2]['iters'] for o in out]}")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sweep", type=int, default=0, help="run the batched sweep of this many pencils")
    ap.add_argument("--threads", type=int, default=16)
    ap.add_argument("--maxiter", type=int, default=2000)
    ap.add_argument("--b", type=int, default=32)
    ap.add_argument("--nblk", type=int, default=31250)
    ap.add_argument("--t", type=int, default=64)
    ap.add_argument("--k", type=int, default=64)
    ap.add_argument("--iters", type=int, default=30)
    ap.add_argument("--maxsub", type=int, default=200)
    ap.add_argument("--minsub", type=int, default=80)
    ap.add_argument("--projected", default="auto")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--preconditioner", default="exact", choices=["exact", "block_jacobi"])
    ap.add_argument("--inner-maxiter", type=int, default=0)
    ap.add_argument("--inner-tol", type=float, default=1e-2)
    ap.add_argument("--verbose", type=int, default=0)
    ap.add_argument("--lock", default="robust", choices=["robust", "reference"])
    ap.add_argument("--ritz-estimate", default="auto", choices=["auto", "fp64", "fp32"])
    a = ap.parse_args(argv)
    if a.sweep:
        return sweep(a.sweep, a.threads, a.precision, a.maxiter)
    P = make_pencil(a.b, a.nblk, a.t, seed=0)
    dev = DevicePencil(P)
    pc = DevicePreconditioner(dev, 3.0, a.preconditioner, precision=a.precision)
    t0 = time.time()
    ev, _, info = jdqz(dev, k=a.k, sigma=3.0, tol=1e-10, maxiter=a.iters, maxsub=a.maxsub,
                       minsub=a.minsub, inner_maxiter=a.inner_maxiter, inner_tol=a.inner_tol,
                       preconditioner=pc, v0=start_vector(P.n, 1), verbose=a.verbose,
                       return_info=True, timing=True, projected=a.projected, lock=a.lock,
                       precision=a.precision, ritz_estimate=a.ritz_estimate)
    wall = time.time() - t0
    d = info["device"]
    print(f"n={P.n} iters={info['iters']} nconv={info['nconv']} wall={wall:.2f}s "
          f"host_qz={d['seconds_qz']:.2f}s device={d['seconds_device']:.2f}s "
          f"launches={d['kernel_launches']} factor={pc.factor_seconds:.3f}s "
          f"refinement_lus={d['ritz_refinements']} fp64_fallbacks={d['ritz_fallbacks']}")
    for name, v in d["kernels"].items():
        if v["calls"]:
            print(f"  {name:8s} calls {v['calls']:6d}  ms {v['ms']:9.2f}  "
                  f"GB {v['bytes'] / 1e9:9.2f}  GB/s {v['bytes'] / max(v['ms'], 1e-9) / 1e6:8.1f}")


if __name__ == "__main__":
    main()
