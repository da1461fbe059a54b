"""bench.py on a small case: one run of every leg, and the JSON line's keys
and units as the measurement contract states them."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_on_a_small_block():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--block-dims", "64,32,16", "--steps", "1",
           "--warmup", "3", "--cycles-per-step", "8", "--profile-cycles", "4", "--accuracy-cycles", "16",
           "--e2e-steps", "1", "--sweep-instances", "4", "--sweep-cycles", "16", "--sweep-fp64-sample", "2",
           "--serve-requests", "4", "--serve-seq-sample", "2", "--batched-block-cycles", "8", "--no-cpu-baseline"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-3000:]
    lines = [x for x in res.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, res.stdout[-3000:]
    d = json.loads(lines[0])
    assert d["metric"] == d["unit"] == "element-cycles/s"
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 3
    assert d["higher_is_better"] is True and d["scaling"] == "weak" and d["vs_baseline"] is None
    assert d["ms_per_step"] > 0 and d["data"] == "synthetic" and "workload" in d["config"]
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] > 0
    assert r["achieved"] > 0 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    e = d["e2e"]
    assert e["value"] > 0 and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(d["clocks"])
    acc = d["fp64_vs_mixed"]
    assert acc["mixed_max_rel_disp_err"] <= 1e-5 and acc["mixed_energy_drift"] <= 5e-3
    assert d["batched_block"]["mixed"]["element_cycles_per_s"] > 0
    sw = d["batched_sweep"]
    assert sw["failed"] == 0 and sw["solves_per_s"] > 0 and sw["cycle_roofline"]["mixed_frac"] > 0
    sv = d["serving"]
    assert sv["failed"] == 0 and sv["requests"] == 4 and sv["p99_latency_s"] >= sv["p50_latency_s"] > 0
    assert sv["deck_read"]["identical"] is True
