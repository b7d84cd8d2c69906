"""Short device JDQZ run of a block-bordered pencil, for profilers.

    python -m bbjd_b200.profile [--b 32] [--nblk 31250] [--t 64] [--k 64]
                                [--iters 30] [--maxsub 200] [--minsub 80]

Builds the seeded pencil, uploads it, factors the exact LU of A - 3 B on the
device, runs `iters` outer JDQZ iterations and prints the per-kernel-class
CUDA-event times and algorithmic bandwidths.  The defaults are the
n = 1,000,064 benchmark pencil; a smaller --nblk gives a case small enough
for multi-pass ncu captures.
"""
from __future__ import annotations

import argparse
import time

from . import DevicePencil, DevicePreconditioner, jdqz, make_pencil, start_vector


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--b", type=int, default=32)
    ap.add_argument("--nblk", type=int, default=31250)
    ap.add_argument("--t", type=int, default=64)
    ap.add_argument("--k", type=int, default=64)
    ap.add_argument("--iters", type=int, default=30)
    ap.add_argument("--maxsub", type=int, default=200)
    ap.add_argument("--minsub", type=int, default=80)
    ap.add_argument("--projected", default="auto")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    a = ap.parse_args(argv)
    P = make_pencil(a.b, a.nblk, a.t, seed=0)
    dev = DevicePencil(P)
    pc = DevicePreconditioner(dev, 3.0, "exact", precision=a.precision)
    t0 = time.time()
    ev, _, info = jdqz(dev, k=a.k, sigma=3.0, tol=1e-10, maxiter=a.iters, maxsub=a.maxsub,
                       minsub=a.minsub, preconditioner=pc, v0=start_vector(P.n, 1),
                       return_info=True, timing=True, projected=a.projected,
                       precision=a.precision)
    wall = time.time() - t0
    d = info["device"]
    print(f"n={P.n} iters={info['iters']} nconv={info['nconv']} wall={wall:.2f}s "
          f"host_qz={d['seconds_qz']:.2f}s device={d['seconds_device']:.2f}s "
          f"launches={d['kernel_launches']} factor={pc.factor_seconds:.3f}s")
    for name, v in d["kernels"].items():
        if v["calls"]:
            print(f"  {name:8s} calls {v['calls']:6d}  ms {v['ms']:9.2f}  "
                  f"GB {v['bytes'] / 1e9:9.2f}  GB/s {v['bytes'] / max(v['ms'], 1e-9) / 1e6:8.1f}")


if __name__ == "__main__":
    main()
