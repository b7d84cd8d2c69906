"""Eigenspectrum sweep over shifts sigma: the launcher the reference's
deployment describes but does not ship (reference README.md:59-83: "each
MPI rank runs jdqz independently on one guess eigenvalue sigma").

One process per GPU (torchrun); the shifts are partitioned over the ranks
(bbjd_b200.sweep.partition: largest first, deterministic), each rank solves
its shifts on its GPU in batches of ``--threads`` concurrent solves that
share one device copy of the pencil (bbjd_solve_batch: one host thread and
CUDA stream per solve, so one solve's host-side projected eigenproblem
overlaps the others' device work), and rank 0 gathers every result and
writes them to ``--out``.  Nothing is exchanged while the ranks solve.

    python -m torch.distributed.run --nproc-per-node 8 -m bbjd_b200.eigensweep \\
        --pencil pencil.npz --sigmas "3+0j,3+10j,3-10j" --k 16 --out sweep.npz
    python -m bbjd_b200.eigensweep --synthetic 16,4096,16 --sigma-grid 3,-40,40,32

``--pencil`` is an ``.npz`` with scipy-sparse ``A`` and ``B`` saved as
``A_data, A_indices, A_indptr, A_shape`` (CSR) and the same for ``B``;
they must have the block-bordered form (bbjd_b200.structure).
``--synthetic b,nblk,t[,seed]`` builds the seeded test pencil instead.
Memory: each concurrent solve holds its LU factors and an n x maxsub
workspace (about 26 GB at n = 10^6, k = 64, maxsub = 200), so choose
``--threads`` to fit the GPU.
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np


def _load_pencil(args):
    from .pencils import make_pencil
    if args.synthetic:
        parts = [int(x) for x in args.synthetic.split(",")]
        b, nblk, t = parts[:3]
        seed = parts[3] if len(parts) > 3 else 0
        return make_pencil(b, nblk, t, seed=seed)
    import scipy.sparse as sp

    from .structure import pencil_from_sparse
    z = np.load(args.pencil)

    def csr(name):
        return sp.csr_matrix((z[f"{name}_data"], z[f"{name}_indices"], z[f"{name}_indptr"]),
                             shape=tuple(z[f"{name}_shape"]))
    P = pencil_from_sparse(csr("A"), csr("B"), b_is_identity=False)
    if P is None:
        raise SystemExit("the pencil does not have the block-bordered form")
    return P


def _sigmas(args) -> list[complex]:
    if args.sigmas:
        return [complex(s.replace(" ", "")) for s in args.sigmas.split(",")]
    if args.sigma_file:
        with open(args.sigma_file) as f:
            return [complex(line.strip()) for line in f if line.strip()]
    re_part, lo, hi, count = args.sigma_grid.split(",")
    return [complex(float(re_part), float(v)) for v in np.linspace(float(lo), float(hi), int(count))]


def solve_share(P, sigmas, idx, args):
    """Solve sigmas[i] for i in idx on this rank's GPU, `threads` at a time;
    returns {i: (eigenvalues, residuals, iters, status, eigenvectors|None)}."""
    from . import DevicePencil, jdqz_batch
    from .pencils import start_vector
    dev = DevicePencil(P)
    out = {}
    for c0 in range(0, len(idx), args.threads):
        chunk = idx[c0:c0 + args.threads]
        res, _ = jdqz_batch([dev] * len(chunk), [sigmas[i] for i in chunk], k=args.k, tol=args.tol,
                            maxiter=args.maxiter, maxsub=args.maxsub, minsub=args.minsub,
                            precision=args.precision, threads=len(chunk),
                            v0s=[start_vector(P.n, 1 + i) for i in chunk],
                            ritz_estimate=args.ritz_estimate)
        for i, (ev, evecs, info) in zip(chunk, res):
            out[i] = (ev, info["residuals"], info["iters"], info["status"],
                      evecs if args.vectors else None)
    dev.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    src = ap.add_mutually_exclusive_group(required=True)
    src.add_argument("--pencil", help=".npz with CSR A and B")
    src.add_argument("--synthetic", help="b,nblk,t[,seed]: the seeded test pencil")
    sig = ap.add_mutually_exclusive_group(required=True)
    sig.add_argument("--sigmas", help="comma-separated complex shifts, e.g. 3+10j,3-10j")
    sig.add_argument("--sigma-file", help="one complex shift per line")
    sig.add_argument("--sigma-grid", help="re,im_lo,im_hi,count: shifts re + i linspace(lo, hi)")
    ap.add_argument("--k", type=int, default=16)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--maxiter", type=int, default=2000)
    ap.add_argument("--maxsub", type=int, default=0)
    ap.add_argument("--minsub", type=int, default=0)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--ritz-estimate", default="auto", choices=["auto", "fp64", "fp32"],
                    help="projected eigenvalues between restarts: complex64 estimates with "
                         "an FP64-refined target (auto, fp32) or all in FP64")
    ap.add_argument("--threads", type=int, default=4, help="concurrent solves per GPU")
    ap.add_argument("--vectors", action="store_true", help="also gather the eigenvectors")
    ap.add_argument("--out", default="sweep.npz")
    args = ap.parse_args(argv)

    import torch
    from .sweep import partition
    rank, local, world = (int(os.environ.get(v, d)) for v, d in
                          (("RANK", 0), ("LOCAL_RANK", 0), ("WORLD_SIZE", 1)))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(hours=6))
    t0 = time.time()
    P = _load_pencil(args)
    sigmas = _sigmas(args)
    from .sweep import SweepItem
    items = [SweepItem(key=s, n=P.n, k=args.k) for s in sigmas]
    mine = partition(items, world)[rank]
    t_setup = time.time() - t0
    results = solve_share(P, sigmas, mine, args)
    if world > 1:
        gathered = [None] * world
        dist.all_gather_object(gathered, results)
        results = {}
        for g in gathered:
            results.update(g)
    wall = time.time() - t0
    if rank == 0:
        order = range(len(sigmas))
        payload = {
            "sigmas": np.array(sigmas),
            "nconv": np.array([len(results[i][0]) for i in order]),
            "iters": np.array([results[i][2] for i in order]),
            "status": np.array([results[i][3] for i in order]),
            "wall_seconds": wall,
            "setup_seconds": t_setup,
        }
        for i in order:
            payload[f"eigenvalues_{i}"] = results[i][0]
            payload[f"residuals_{i}"] = results[i][1]
            if results[i][4] is not None:
                payload[f"eigenvectors_{i}"] = results[i][4]
        np.savez(args.out, **payload)
        total = int(payload["nconv"].sum())
        solve = wall - t_setup
        print(f"{len(sigmas)} shifts on {world} GPU(s): {total} eigenpairs in {wall:.1f} s "
              f"({t_setup:.1f} s building the pencil, {solve:.1f} s solving: "
              f"{total / max(solve, 1e-9):.2f} eigenpairs/s) -> {args.out}")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
