"""bench.py's JSON contract where it runs without a GPU: the reference arm
(the oracle port of the reference's CPU path, timed on the host cores) on a
bounded sample, and the issue-roofline arithmetic."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def test_reference_arm_prints_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--ref-seconds", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"].startswith("sites")
    assert line["unit"] == "sites*iters/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["n_gpus"] == 1
    assert line["config"]["workload"] == "torus_100k" and line["config"]["sites"] == 100_000
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_issue_roofline_arithmetic():
    sys.path.insert(0, ROOT)
    import bench
    with open(os.path.join(ROOT, "profiles", "instructions.json")) as fh:
        counts = json.load(fh)["warp_instructions_per_remesh"]
    prof = {"grid": 0.03, "knn": 0.08, "clip": 0.06, "proj": 0.1}
    out = bench.issue_roofline(prof, 100, 1965.0, sms=148)
    assert out["bound"] == "issue" and out["peak"] == 148 * 4 * 1965e6
    for kernel, group in (("k_site_knn", "knn"), ("k_site_clip", "clip"), ("k_site_proj", "proj")):
        k = out["kernels"][kernel]
        assert abs(k["achieved"] - counts[kernel] / (prof[group] * 1e-3 * 100)) < 1e-6 * k["achieved"]
        assert abs(k["frac"] - k["achieved"] / out["peak"]) < 1e-12
        assert 0.0 < k["frac"] < 1.0
    assert bench.issue_roofline(prof, 100, None, sms=148) is None


@pytest.mark.gpu
def test_main_arm_prints_contract_line():
    """One short run of the benchmark's own arm on the GPU: every key the
    JSON contract asks for, with consistent values."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "1", "--warmup", "3", "--no-cpu",
                        "--no-accuracy"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "roofline",
                "issue_roofline", "cpu_baseline", "clocks"):
        assert key in line, key
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] == 3 and line["scaling"] == "weak"
    n, iters = line["config"]["sites"], line["config"]["iters"]
    assert abs(line["value"] - n * iters / (line["ms_per_step"] / 1e3)) < 1e-6 * line["value"]
    assert line["gpu_launches"] >= 10 * iters
    e2e = line["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert e2e["same_sites_as_engine"] is True
    rf = line["roofline"]
    assert rf["bound"] == "hbm" and rf["unit"] == "GB/s" and abs(rf["frac"] - rf["achieved"] / rf["peak"]) < 1e-9
    assert set(line["issue_roofline"]["kernels"]) == {"k_site_knn", "k_site_clip", "k_site_proj"}
    assert set(line["config"]["tiles"]) == {"knn_block", "clip_block", "proj_block"}
