"""The reference arm of bench.py (the reference's own CPU path on a bounded sample) prints one JSON
line with the keys the benchmark contract names; it needs no GPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--cpu-budget", "2"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["workload"]
    # the reference arm builds its inputs from the oracle and never loads the product library
    assert d["product_library_mapped"] is False
    assert len(d["config"]["complexes"]) == 8  # the default workload: the batched eight complexes


def test_work_per_pose_weighted_by_swarms():
    """The brute-force work per scored pose averages Nr x Nl over the poses of every complex, so a
    complex with more swarms counts for more (the batched workload's complexes differ in both)."""
    sys.path.insert(0, ROOT)
    import bench
    cfg = {"complexes": [(100, 10, 1), (1000, 20, 3)]}
    assert bench.brute_pairs_per_pose(cfg) == (100 * 10 * 1 + 1000 * 20 * 3) / 4
    c1 = bench.CONFIGS["c1"]
    nr, nl, _ = c1["complexes"][0]
    assert bench.brute_pairs_per_pose(c1) == nr * nl


def test_roofline_follows_the_precision():
    """The roofline object rooflines a mixed run against the FP32 vector peak with the mixed scorer's
    issue ceiling beside it, and an FP64 run against the FP64 vector peak without that ceiling."""
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    m = {"run": {"stats": {"pairs_in_cutoff": 5.7e9, "pairs_evaluated": 2.7e10, "scored_poses": 1e5}},
         "t_ms": 1000.0, "pairs_all": 5.7e9, "scored": 1e5, "value": 1e5}
    args = argparse.Namespace(steps=10)
    peaks = {"sm_max_mhz": 1965.0, "hbm_gbs": 7000.0}
    for prec, bound, lanes in (("mixed", "fp32", 128), ("fp64", "fp64", 64)):
        cfg = dict(bench.CONFIGS["c1"], precision=prec)
        r = bench.roofline_of(cfg, "c1", m, args, peaks, "measured")
        assert r["bound"] == bound
        assert abs(r["peak"] - 148 * lanes * 2 * 1.965e9 / 1e12) < 1e-9
        assert abs(r["achieved"] - 8 * 5.7e9 / 1e12) < 1e-12 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-15
        assert ("issue_bound" in r) == (prec == "mixed") and ("l1_bound" in r) == (prec == "mixed")
        if prec == "mixed":
            assert abs(r["l1_bound"]["ceiling_pairs_per_s"] - 148 * 1.965e9 / bench.L1_WAVEFRONTS_PER_PAIR) < 1.0
