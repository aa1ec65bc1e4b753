"""One short run of bench.py's GPU arm: every key of the JSON contract, with
consistent values.  Collected after the GPU parity tests (and before the
no-allocation test, which is collected last), so a benchmark problem never
hides a kernel result."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


@pytest.mark.gpu
def test_main_arm_prints_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "1", "--warmup", "3", "--no-cpu",
                        "--no-accuracy", "--no-c3", "--meshes", "12"], capture_output=True, text=True, timeout=900,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "roofline",
                "cpu_baseline", "clocks", "plain_loop", "batched_over_plain", "latency_ms", "hausdorff_rel"):
        assert key in line, key
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] == 3
    cfg = line["config"]
    assert cfg["workload"] == "batched_12_meshes" and cfg["meshes"] == 12
    n, iters = cfg["sites_total"], cfg["iters"]
    assert abs(line["value"] - n * iters / (line["ms_per_step"] / 1e3)) < 1e-6 * line["value"]
    assert line["gpu_launches"] >= 10 * iters
    clk = line["clocks"]
    assert clk["sm_mhz"] or clk["sm_max_mhz"], clk
    e2e = line["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert e2e["same_sites_as_engine"] is True
    assert line["plain_loop"]["identical_results"] is True
    assert line["batched_over_plain"] > 0
    rf = line["roofline"]
    assert rf["bound"] == "hbm" and rf["unit"] == "GB/s" and abs(rf["frac"] - rf["achieved"] / rf["peak"]) < 1e-9
    assert rf["traffic"] is not None and "recorded" in rf["traffic_source"], rf
    ir = line["issue_roofline"]
    assert ir is not None, f"issue_roofline missing although a clock is known: clocks={clk}"
    assert "recorded" in ir["counts"] and len(ir["kernels"]) == 3, ir
    assert all(0.0 < k["frac"] < 1.5 for k in ir["kernels"].values()), ir
    assert set(line["tiles"]) == {"knn_block", "clip_block", "proj_block"}
    assert 0 < line["hausdorff_rel"]["max"] < 1e-2
