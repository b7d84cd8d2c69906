"""Host-side arithmetic of bench.py: how the reference's sampled seconds
per iteration and its cached full run become eigenpairs/s, and how the
mixed and FP64 forms' eigenvalue sets are compared."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_rate_scales_the_sample_by_the_full_runs_own_profile():
    # a full run of 2,000 iterations whose first 10 take 1 s each and whose
    # later ones take 3 s: mean over all = (10 * 1 + 1990 * 3) / 2000
    t = np.concatenate([[0.0], np.cumsum(np.r_[np.ones(10), 3 * np.ones(1989)])])
    rec = {"pairs": 10, "returned": 12, "iters": 2000, "time": t, "threads": 5}
    # the box measured 2 s per iteration over the same first 10 iterations
    value, ratio, est_s = bench.reference_rate({"s_per_iter": 2.0, "span": 10}, rec)
    full = (t[-1] - t[0]) / (len(t) - 1)
    assert np.isclose(ratio, full / 1.0)
    assert np.isclose(est_s, 2.0 * ratio * 2000)
    assert np.isclose(value, 10 / est_s)


def test_reference_rate_with_a_sample_longer_than_the_record():
    t = np.arange(6, dtype=float)          # 5 iterations of 1 s
    rec = {"pairs": 1, "returned": 1, "iters": 5, "time": t, "threads": 1}
    value, ratio, est_s = bench.reference_rate({"s_per_iter": 1.0, "span": 50}, rec)
    assert np.isclose(ratio, 1.0) and np.isclose(est_s, 5.0) and np.isclose(value, 0.2)


def test_compare_forms():
    a = np.array([3.0 + 0.1j, 3.2 - 0.05j, 2.9 + 0.3j])
    b = np.array([3.2 - 0.05j + 1e-11, 3.0 + 0.1j - 2e-12, 3.5 + 0j])
    d, same = bench._compare_forms(a, b)
    assert same == 2
    assert np.isclose(d[0], 2e-12) and np.isclose(d[1], 1e-11)
    assert d[2] > 0.1
    assert bench._compare_forms([], b) == ([], 0)


def test_reference_run_record_counts_distinct_pairs():
    rec = bench.reference_run_record()
    assert rec["iters"] >= 200 and len(rec["time"]) >= 200
    assert 1 <= rec["pairs"] <= rec["returned"]
    assert np.all(np.diff(rec["time"]) >= 0)


def test_reference_arm_reports_unavailable_without_its_cached_run(monkeypatch, capsys):
    import json
    import types
    monkeypatch.setattr(bench, "REF_RUN", "/nonexistent/bbt_n1000064.npz")
    monkeypatch.delenv("RANK", raising=False)
    args = types.SimpleNamespace(warmup=3, steps=1, ref_iters=16)
    assert bench.run_reference(args) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_reference_arm_other_ranks_do_nothing(monkeypatch, capsys):
    import types
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.run_reference(types.SimpleNamespace(warmup=3, steps=1, ref_iters=16)) == 0
    assert capsys.readouterr().out == ""
