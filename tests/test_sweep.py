"""The sigma-sweep driver's host logic: partition and gather, with two
gloo ranks on the CPU (the N > 1 path has no collective but the final
gather).  The solve function is the CPU oracle on tiny pencils, so the
results can be checked."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bbjd_b200.sweep import SweepItem, partition, run_sweep


def test_partition_covers_and_balances():
    items = [SweepItem(key=i, n=n, k=16) for i, n in
             enumerate([50000, 300000, 120000, 80000, 250000, 60000, 90000])]
    for world in (1, 2, 3, 4, 8):
        parts = partition(items, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(items)))
        loads = [sum(items[i].estimate() for i in p) for p in parts]
        # LPT: the heaviest rank carries at most the mean plus the largest item
        assert max(loads) <= sum(loads) / world + max(it.estimate() for it in items)
        assert partition(items, world) == parts          # deterministic


def _solve(item):
    import scipy.sparse as sp
    from scipy.sparse.linalg import splu
    from bbjd_b200.pencils import make_pencil, start_vector
    from oracle import jdqz_np
    P = make_pencil(8, item.payload["nblk"], 2, seed=item.payload["seed"])
    A, B = P.to_csc("A"), P.to_csc("B")
    s = complex(item.key)
    lu = splu((A - s * B).tocsc())
    out = jdqz_np.jdqz(P.n, item.k, lambda x: A @ x, lambda x: B @ x, lu.solve, sigma=s,
                       tol=1e-10, maxiter=300, maxsub=24, minsub=10, v0=start_vector(P.n, 1))
    return (item.key, out["nconv"], np.sort_complex(out["eigenvalues"]).tolist())


def _items():
    return [SweepItem(key=complex(3.0, im), n=8 * nblk + 2, k=2,
                      payload={"nblk": nblk, "seed": i})
            for i, (im, nblk) in enumerate([(-10.0, 16), (0.0, 24), (10.0, 20), (-5.0, 12),
                                            (5.0, 18)])]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = run_sweep(_items(), _solve, rank=rank, world=world)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_rank_sweep_matches_single_rank():
    serial = run_sweep(_items(), _solve)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank holds every item's result, in item order, equal to the serial run
    for r in (0, 1):
        assert [g[0] for g in got[r]] == [s[0] for s in serial]
        for a, b in zip(got[r], serial):
            assert a[1] == b[1]
            assert np.allclose(a[2], b[2], atol=1e-8)
