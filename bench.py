#!/usr/bin/env python
"""Benchmark: JDQZ eigenpairs/s on the n = 1,000,064 block-bordered pencil,
mixed-precision form against the plain FP64 form.

Workload (the configuration the headline metric is quoted on): the seeded
block-bordered pencil with b = 32, 31,250 diagonal blocks, t = 64 tau rows
(n = 1,000,064), complex128, sigma = 3, k = 64 eigenpairs, maxsub = 200,
minsub = 80, tol = 1e-10, maxiter = 2000, exact block-bordered LU of
A - sigma B factored once on the device (factor time reported separately).

One step = one complete jdqz solve.  Both forms of the engine solve the same
pencil from the same start vector (--precision both, the default): the
mixed form (complex64 LU factors and a complex64 first CGS pass against V;
second pass, DGKS, residuals, projected pencil and QZ in FP64) gives
`value` and `e2e`; the FP64 form's numbers, the per-eigenvalue distance
between the two forms' sets and the change in iterations per converged
pair are in `detail`.  `value` = converged eigenpairs / solve time with the
pencil and its LU already in HBM (CUDA events around the call, max over
ranks); `e2e` = the same through the public API from pinned host buffers:
upload of the pencil, device LU factorisation, the solve, and the copy of
the eigenvectors back to the host, all inside the timed region.  Inputs are
larger than L2 (4.1 GB pencil), so no flush is needed.  `detail` also
times a window of outer iterations of the inner-GMRES configuration on the
same pencil (k = 32, maxsub 120, minsub 48, block-Jacobi preconditioner,
GMRES 50 steps to 1e-3) in both forms.

Multi-GPU (torchrun, one process per GPU): rank r solves its own pencil of
the sigma-sweep (generator seed r); nothing is exchanged (weak scaling).

--impl reference: the reference's own CPU implementation (its C core built
from its sources into oracle/_ref) on the same pencil, with the C
restatement of the exact block-bordered LU (oracle/c) as its
preconditioner, timed on the host cores over its first outer iterations;
run_reference() says how that sample and the reference's own full
2,000-iteration run (cached in tests/golden/bbt_n1000064.npz) give its
eigenpairs/s.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = dict(b=32, nblk=31250, t=64, sigma=3.0, k=64, maxsub=200, minsub=80, tol=1e-10,
                maxiter=2000)
WORKLOAD_NAME = "bbt_n1000064_k64"
# The reference's own run on this pencil: its C core for 2,000 outer
# iterations from the same start vector, with per-iteration timestamps
# (written by tests/golden/make_golden_n1e6.py).
REF_RUN = os.path.join(ROOT, "tests", "golden", "bbt_n1000064.npz")
# DRAM traffic (read + write bytes) of each kernel class per call, from ncu
# captures on B200 (profiles/): the fused A,B product per launch, and the
# ratio of measured DRAM bytes to algorithmic bytes for the CGS classes
# (all their launches over 150 outer iterations, selected by NVTX range).
SPMV_TRAFFIC_BYTES = 4.117e9   # launch list, n = 1,000,064: 317.04 GB over 77 launches
TRAFFIC_RATIO = {"pencil": 916.86 / 918.04, "orth": 546.50 / 548.07}   # GB measured / algorithmic


def _env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # the raw samples go to $BBJD_CLOCKS_DIR (default: the temp dir); the
        # JSON line carries their summary
        out = os.environ.get("BBJD_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out, f"clocks_rank{index}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        mx = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


_REF_STATE = {}


def reference_sample(iters: int, threads: int, P=None):
    """Run the reference's jdqz (oracle/_ref: its C core built from its own
    sources, linked to the same OpenBLAS) on the workload pencil for
    `iters` outer iterations and return its seconds per outer iteration.

    Operators: the reference takes A x, B x and M^-1 r from its caller
    (reference include/bbjd.h:101-109); here they are the numpy block
    product of the pencil (2x faster than the scipy CSC product the
    reference's wrapper builds, whose assembly alone takes ~100 s at this
    size) and the C restatement of the exact block-bordered LU.
    Every outer iteration before the first lock calls the preconditioner
    twice (the correction z = M^-1 r and s = M^-1 u, reference
    jd_core.c:952-965), so the first of each pair of calls marks an
    iteration; the sample is the time from the first iteration's mark to the
    last one's, over iters - 1 iterations (the n x maxsub workspace's
    first touch and the start-up products fall outside it).
    """
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(threads))
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import _bbjd_c  # the reference's C core, built from its sources
    from bbjd_b200.pencils import make_pencil, start_vector
    from oracle.bbt_lu import BBTLUHost
    w = WORKLOAD
    if "lu" not in _REF_STATE:
        t0 = time.time()
        if P is None:
            P = make_pencil(w["b"], w["nblk"], w["t"], seed=0)
        _REF_STATE["P"] = P
        _REF_STATE["lu"] = BBTLUHost(P, w["sigma"])
        _REF_STATE["setup_s"] = time.time() - t0
    P, lu = _REF_STATE["P"], _REF_STATE["lu"]
    v0 = start_vector(P.n, 1)
    marks = []

    def solve(r):
        marks.append(time.time())
        return lu.solve(r)

    t1 = time.time()
    out = _bbjd_c.jdqz_c(n=P.n, nev=w["k"], sigma=w["sigma"], target=0, matvec_A=P.matvec_A,
                         matvec_B=P.matvec_B, precond_solve=solve, tol=w["tol"], maxiter=iters,
                         maxsub=w["maxsub"], minsub=w["minsub"], inner_maxiter=0, inner_tol=1e-2,
                         verbose=0, v0=v0)
    t2 = time.time()
    done = int(out[4])
    it_marks = marks[0::2][:done]
    span = len(it_marks) - 1
    dt = (it_marks[-1] - it_marks[0]) if span > 0 else t2 - t1
    return {"s_per_iter": dt / max(span, 1), "iters": done, "span": max(span, 1), "seconds": dt,
            "seconds_call": t2 - t1, "setup_s": _REF_STATE["setup_s"], "threads": threads,
            "nconv": int(out[3])}


def reference_run_record():
    """The reference's own full run on this pencil (its C core, 2,000 outer
    iterations from the same start vector, per-iteration timestamps; cached
    in tests/golden/bbt_n1000064.npz): its distinct converged pairs (the
    reference can return one eigenvalue more than once; values within
    1e-6 |lambda| of an earlier one count once), its iteration count, and
    its per-iteration wall times."""
    g = dict(np.load(REF_RUN))
    ev = np.asarray(g["ref_eigenvalues"])
    distinct = []
    for lam in ev:
        if all(abs(lam - d) > 1e-6 * max(1.0, abs(lam)) for d in distinct):
            distinct.append(lam)
    return {"pairs": len(distinct), "returned": int(g["ref_nconv"]), "iters": int(g["ref_iters"]),
            "time": np.asarray(g["ref_time"], dtype=np.float64), "threads": int(g["ref_threads"])}


def reference_rate(sample: dict, rec: dict):
    """Eigenpairs/s of the reference on this box's host cores.

    The box times the reference's first outer iterations (`sample`); the
    cached full run (`rec`, timed on the build machine with the same code)
    gives the ratio of its mean seconds per iteration over all iterations
    to its mean over the same first iterations (later iterations work on
    subspaces of 80..200 columns and cost more).  The full run's time on
    this box is then estimated as sample s/iteration x that ratio x the full
    run's iteration count, and the reference's rate is its own distinct
    converged pairs over that time."""
    t = rec["time"]
    m = min(sample["span"], len(t) - 1)
    first = (t[m] - t[0]) / m
    full = (t[-1] - t[0]) / (len(t) - 1)
    ratio = full / first
    est_s = sample["s_per_iter"] * ratio * rec["iters"]
    return rec["pairs"] / est_s, ratio, est_s


def run_reference(args):
    rank, _, world = _env_rank()
    if rank != 0:
        return 0
    # all host cores (on the 16-core B200 box its seconds per outer iteration
    # are the same with 4, 8 and 16 threads: 2.09, 2.04, 2.05 s)
    threads = max(1, os.cpu_count() or 1)
    if not os.path.exists(REF_RUN):
        print(json.dumps({"impl": "reference", "unavailable": "the reference's cached full run "
                          "(tests/golden/bbt_n1000064.npz) is missing"}), flush=True)
        return 0
    rec = reference_run_record()
    steps = []
    for i in range(args.warmup + args.steps):
        warm = i < args.warmup
        # the warm-up steps only page in the pencil, the LU and the thread pools
        s = reference_sample(min(args.ref_iters, 4) if warm else args.ref_iters, threads)
        if not warm:
            steps.append(s)
    spi = sum(s["seconds"] for s in steps) / sum(s["span"] for s in steps)
    value, ratio, est_s = reference_rate({"s_per_iter": spi, "span": steps[0]["span"]}, rec)
    sample = (f"reference jdqz (C core built from its sources, scipy OpenBLAS, {threads} threads) "
              f"on the n=1,000,064 pencil, numpy block products and the C block-bordered LU as "
              f"its operators: outer iterations 1..{steps[0]['span']} timed per step, "
              f"{spi:.3f} s/iteration; x {ratio:.3f} (its full 2,000-iteration run's mean "
              f"s/iteration over its mean over the same first iterations, cached run on "
              f"{rec['threads']} threads) x {rec['iters']} iterations = {est_s:.0f} s for its "
              f"{rec['pairs']} distinct converged pairs ({rec['returned']} returned)")
    line = {"metric": "eigenpairs/s", "value": value, "unit": "eigenpairs/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(s["seconds"] for s in steps) / len(steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "complex128", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, **WORKLOAD, "preconditioner": "exact LU (C, host)"},
            "cpu_baseline": {"value": value, "unit": "eigenpairs/s", "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "eigenpairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "s_per_iter_sample": spi, "full_run_ratio": ratio, "estimated_full_run_s": est_s,
            "setup_s": steps[0]["setup_s"]}
    print(json.dumps(line), flush=True)
    return 0


def _form_summary(results, secs_max):
    """Pairs, iterations and device statistics of one form's timed solves."""
    info = results[-1][1][2]
    d = info["device"]
    kern = {k: {"ms": round(v["ms"], 2), "calls": v["calls"],
                "GBps": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6, 1)}
            for k, v in d["kernels"].items() if v["calls"]}
    steps = len(results)
    return {"value": sum(r[1][2]["nconv"] for r in results) / secs_max,
            "ms_per_step": 1e3 * secs_max / steps,
            "nconv": info["nconv"], "iters": sum(r[1][2]["iters"] for r in results) // steps,
            "conv_iters": [int(c) for c in d["conv_iters"]],
            "seconds_qz_host": round(d["seconds_qz"], 3),
            "seconds_qz_exposed": round(d["seconds_qz_exposed"], 3),
            "seconds_device_timed": round(d["seconds_device"], 3),
            "guess_hits": d["guess_hits"], "guess_misses": d["guess_misses"],
            "dgks_passes": d["dgks_passes"], "restarts": d["restarts"],
            "ritz_refinement_lus": d["ritz_refinements"], "ritz_fp64_fallbacks": d["ritz_fallbacks"],
            "device_GB": round(d["bytes_device"] / 1e9, 1),
            "gpu_launches": int(sum(r[1][2]["device"]["kernel_launches"] for r in results)),
            "kernels": kern}


def _compare_forms(ev_a, ev_b):
    """Per-eigenvalue distance from each value of set a to the nearest value
    of set b, and how many values of a lie within 1e-8 |lambda| of one in b
    (the same eigenvalue; the eigenvalues near sigma are ~1e-2 apart)."""
    ev_a, ev_b = np.asarray(ev_a), np.asarray(ev_b)
    if not len(ev_a) or not len(ev_b):
        return [], 0
    d = [float(np.min(np.abs(ev_b - lam))) for lam in ev_a]
    same = sum(1 for lam, x in zip(ev_a, d) if x <= 1e-8 * max(1.0, abs(lam)))
    return d, same


GMRES_CONFIG = dict(k=32, maxsub=120, minsub=48, inner_maxiter=50, inner_tol=1e-3)


def gmres_window(dev, v0, iters, form, timed):
    """The inner-GMRES configuration on the same pencil: block-Jacobi
    preconditioner (b x b diagonal-block LU of A - sigma B), left-
    preconditioned GMRES of at most 50 steps to 1e-3 with the projectors in
    FP64 (complex64 Arnoldi basis in the mixed form), k = 32, maxsub 120,
    minsub 48, for a fixed window of outer iterations (a full solve to 32
    pairs takes thousands): seconds per outer iteration, pairs converged in
    the window, and the device classes."""
    from bbjd_b200 import DevicePreconditioner, jdqz
    w = WORKLOAD
    pc = DevicePreconditioner(dev, w["sigma"], "block_jacobi", precision=form)
    kw = dict(sigma=w["sigma"], tol=w["tol"], maxiter=iters, v0=v0, return_info=True,
              precision=form, **GMRES_CONFIG)
    jdqz(dev, preconditioner=pc, timing=False, **dict(kw, maxiter=3))      # warm-up
    dt, out = timed(lambda: jdqz(dev, preconditioner=pc, timing=True, **kw))
    pc.close()
    info = out[2]
    d = info["device"]
    return {"form": form, "outer_iters": info["iters"], "seconds": round(dt, 3),
            "s_per_iter": round(dt / max(info["iters"], 1), 4), "nconv": info["nconv"],
            "seconds_device_timed": round(d["seconds_device"], 3),
            "seconds_qz_host": round(d["seconds_qz"], 3),
            "kernels": {k: {"ms": round(v["ms"], 1),
                            "GBps": round(v["bytes"] / max(v["ms"], 1e-9) / 1e6, 1)}
                        for k, v in d["kernels"].items() if v["calls"]}}


def run_ours(args):
    import torch
    import torch.distributed as dist

    from bbjd_b200 import DevicePencil, DevicePreconditioner, jdqz, make_pencil, start_vector

    rank, local, world = _env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        # short enough that ranks waiting on a dead peer end with an error;
        # one solve takes about 25 s, a rank's whole run about 6 minutes
        dist.init_process_group("nccl", timeout=timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    w = WORKLOAD
    seed = rank
    t0 = time.time()
    P = make_pencil(w["b"], w["nblk"], w["t"], seed=seed)
    host = P.device_arrays()     # flat, in the order the kernels read
    # pinned copies of the C-ABI layout: the inputs of the end-to-end steps
    pinned = {k: torch.from_numpy(v.view(np.float64)).pin_memory() for k, v in host.items()}
    del host
    v0 = start_vector(P.n, seed + 1)
    gen_s = time.time() - t0
    forms = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    head = forms[0]

    def solve_kw(form):
        return dict(k=w["k"], sigma=w["sigma"], tol=w["tol"], maxiter=w["maxiter"],
                    maxsub=w["maxsub"], minsub=w["minsub"], v0=v0, return_info=True,
                    projected=args.projected, precision=form, ritz_estimate=args.ritz_estimate,
                    host_overlap=args.host_overlap)

    dims = dict(b=w["b"], nblk=w["nblk"], t=w["t"])
    dev = DevicePencil(arrays=pinned, **dims)

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn):
        barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        out = fn()
        b.record()
        torch.cuda.synchronize()
        barrier()
        return a.elapsed_time(b) * 1e-3, out

    # device-resident steps, each form after its own warm-up
    timed_res, clocks, factor_s = {}, {}, {}
    for form in forms:
        pc = DevicePreconditioner(dev, w["sigma"], "exact", precision=form)
        factor_s[form] = pc.factor_seconds
        for _ in range(args.warmup):
            jdqz(dev, preconditioner=pc, timing=False, **solve_kw(form))
        res = []
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                res.append(timed(lambda: jdqz(dev, preconditioner=pc, timing=True,
                                              **solve_kw(form))))
        clocks[form] = clk.summary()
        timed_res[form] = res
        pc.close()

    # end-to-end steps of the headline form through the public API from
    # pinned host buffers
    e2e = []
    for _ in range(args.steps):
        def full():
            d = DevicePencil(arrays=pinned, **dims)
            p = DevicePreconditioner(d, w["sigma"], "exact", precision=head)
            r = jdqz(d, preconditioner=p, timing=False, **solve_kw(head))
            p.close()
            d.close()
            return r
        e2e.append(timed(full))

    gmres = [gmres_window(dev, v0, args.gmres_iters, f, timed) for f in forms] \
        if args.gmres_iters > 0 else []

    # max over ranks of the seconds, sum of the pairs
    secs = [sum(r[0] for r in timed_res[f]) for f in forms] + [sum(r[0] for r in e2e)]
    pairs = [sum(r[1][2]["nconv"] for r in timed_res[f]) for f in forms] + \
        [sum(r[1][2]["nconv"] for r in e2e)]
    t_local = torch.tensor(secs, dtype=torch.float64, device="cuda")
    c_local = torch.tensor(pairs, dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
        dist.all_reduce(c_local, op=dist.ReduceOp.SUM)
    secs_max, pairs_all = t_local.tolist(), c_local.tolist()
    summ = {f: _form_summary(timed_res[f], secs_max[i]) for i, f in enumerate(forms)}
    for i, f in enumerate(forms):
        summ[f]["value"] = pairs_all[i] / secs_max[i]
        summ[f]["factor_s"] = round(factor_s[f], 3)
    e_secs_max, e_pairs_all = secs_max[-1], pairs_all[-1]
    hs = summ[head]

    info = timed_res[head][-1][1][2]
    d = info["device"]
    # dominant kernel class by device time
    dom = max(d["kernels"].items(), key=lambda kv: kv[1]["ms"])
    peak, peak_kind = _peaks()
    roof = None
    if dom[1]["calls"] and dom[1]["ms"] > 0:
        per_launch_bytes = dom[1]["bytes"] / dom[1]["calls"]
        per_launch_s = dom[1]["ms"] * 1e-3 / dom[1]["calls"]
        ach = per_launch_bytes / per_launch_s / 1e9
        roof = {"bound": "hbm", "kernel": dom[0], "achieved": round(ach, 1), "peak": peak,
                "unit": "GB/s", "frac": round(ach / peak, 4), "peak_kind": peak_kind,
                "traffic": (SPMV_TRAFFIC_BYTES if dom[0] == "spmv" else
                            round(TRAFFIC_RATIO[dom[0]] * per_launch_bytes) if dom[0] in TRAFFIC_RATIO
                            else None),
                "algorithmic_bytes_per_launch": per_launch_bytes}
    n = P.n
    h2d = sum(v.numel() * 8 for v in pinned.values()) + 16 * n
    d2h = 16 * n * (e_pairs_all / max(1, world * len(e2e))) + 24 * w["k"]
    detail = {"form": head, **{k: v for k, v in hs.items() if k not in ("value", "ms_per_step")},
              "setup_s": round(gen_s, 1)}
    if len(forms) == 2:
        other = forms[1]
        ev_h = timed_res[head][-1][1][0]
        ev_o = timed_res[other][-1][1][0]
        dist_h, same = _compare_forms(ev_h, ev_o)
        o = summ[other]
        detail[other] = {k: v for k, v in o.items() if k != "kernels"}
        detail[other]["kernels"] = o["kernels"]
        detail["clocks_" + other] = clocks[other]
        detail[f"{head}_vs_{other}"] = {
            "eigenpairs_per_s_ratio": hs["value"] / o["value"] if o["value"] else None,
            "solve_seconds": [hs["ms_per_step"] / 1e3, o["ms_per_step"] / 1e3],
            "device_seconds": [hs["seconds_device_timed"], o["seconds_device_timed"]],
            "iters_per_pair": [hs["iters"] / max(hs["nconv"], 1), o["iters"] / max(o["nconv"], 1)],
            "pairs_in_both": same,
            "eigenvalue_distance_to_nearest_in_other": [float(f"{x:.3e}") for x in dist_h],
            "max_distance_same_eigenvalue": max([x for x, lam in zip(dist_h, ev_h)
                                                 if x <= 1e-8 * max(1.0, abs(lam))], default=None)}
    if gmres:
        detail["gmres_block_jacobi"] = {"config": {"workload": WORKLOAD_NAME, **GMRES_CONFIG,
                                                   "preconditioner": "block Jacobi (device)"},
                                        "forms": gmres}
    line = {
        "metric": "eigenpairs/s", "value": hs["value"], "unit": "eigenpairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": hs["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "complex128" if head == "fp64" else "complex128+complex64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, **WORKLOAD, "precision": head,
                   "forms": forms, "projected": args.projected,
                   "ritz_estimate": args.ritz_estimate, "host_overlap": args.host_overlap,
                   "preconditioner": "exact block-bordered LU (device)",
                   "l2": "inputs larger than L2 (4.1 GB pencil), no flush"},
        "e2e": {"value": e_pairs_all / e_secs_max, "unit": "eigenpairs/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": hs["gpu_launches"],
        "roofline": roof,
        "clocks": clocks[head],
        "detail": detail,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_RUN):
        threads = max(1, os.cpu_count() or 1)
        s = reference_sample(args.ref_iters, threads, P=P)
        rec = reference_run_record()
        val, ratio, est_s = reference_rate(s, rec)
        line["cpu_baseline"] = {
            "value": val, "unit": "eigenpairs/s", "cores": threads, "kind": "reference",
            "sample": (f"reference jdqz (its C core built from its sources) on this pencil: "
                       f"outer iterations 1..{s['span']} from the same start vector timed here, "
                       f"{s['s_per_iter']:.3f} s/iteration, x {ratio:.3f} (its cached full "
                       f"run's mean over its first-iteration mean) x {rec['iters']} iterations "
                       f"= {est_s:.0f} s for its {rec['pairs']} distinct converged pairs")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--projected", default="auto", choices=["auto", "qz", "schur"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: the mixed form (headline) and the plain FP64 form on the same "
                         "pencil; fp64 or mixed: that form alone")
    ap.add_argument("--ritz-estimate", default="auto", choices=["auto", "fp64", "fp32"],
                    help="projected eigenvalues between restarts: fp32 estimates + FP64 "
                         "refinement of the target (auto), or all in fp64")
    ap.add_argument("--host-overlap", default="auto", choices=["auto", "off"],
                    help="auto: the projected eigenvalue estimates run on a second host thread "
                         "while the device iterates on the guessed target; off: serially")
    ap.add_argument("--ref-iters", type=int, default=16,
                    help="reference outer iterations per CPU sample step")
    ap.add_argument("--gmres-iters", type=int, default=100,
                    help="outer iterations of the inner-GMRES configuration reported in detail "
                         "(0: skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
