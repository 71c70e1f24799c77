"""bench.py's host-side pieces that need no GPU: the JSON line of the reference arm (IMPACT's CPU
algorithm, the oracle restatement, on a small case), the peak and traffic tables the roofline
object is computed from, and the whole-job rate."""
import json
import os
import subprocess
import sys

import bench  # the repository root is on sys.path (conftest.py)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CONTRACT = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config", "e2e", "cpu_baseline"}


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--size", "32",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600, check=True)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and CONTRACT <= set(line)
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1
    assert line["config"]["workload"] == "stenosed-vessel-32x32x64"
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]


def test_roofline_tables():
    peaks, note = bench.measured_peaks()
    assert peaks["hbm_gbs"] > 0 and note in ("of measured", "of fallback")
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert note == "of measured"
    ratios = bench.traffic_ratio()
    for kind in ("mg_post_smooth", "mg_pre_smooth", "div_grad_dot", "nl_rhs"):
        assert 0.8 < ratios[kind] < 1.2, (kind, ratios[kind])


def test_whole_job_rate_counts_every_replica():
    # 2 replicas x 1e6 cells x 4 steps in 2 s (the slowest replica's time) = 4 Mcell-steps/s
    assert bench.whole_job_rate(2, 1_000_000, 4, 2000.0) == 4.0
