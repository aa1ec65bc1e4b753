"""bench.py's JSON contract where it runs without a GPU: the reference arm
(the oracle port of the reference's CPU path, timed on the host cores) on a
bounded sample of the batched workload, its configuration identical to the
GPU arm's, and the issue-roofline arithmetic."""
import json
import os
import subprocess
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)


def test_reference_arm_prints_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--ref-seconds", "1", "--meshes", "6"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"].startswith("sites")
    assert line["unit"] == "sites*iters/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["n_gpus"] == 1
    cfg = line["config"]
    assert cfg["workload"] == "batched_6_meshes" and cfg["meshes"] == 6 and cfg["iters"] == 100 and cfg["k"] == 24
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert "whole remeshes" in cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_both_arms_share_one_config():
    """The GPU arm and the reference arm build their config dicts with the
    same function, so the dicts are identical for the same flags."""
    import bench
    _, a, _ = bench.batched_workload(4, 1)
    _, b, _ = bench.batched_workload(4, 1)
    assert a == b and a["parallelism"] == "single GPU"
    assert "tiles" not in a                       # run-dependent values stay outside config
    _, c, _ = bench.batched_workload(4, 2)
    assert c["parallelism"] != a["parallelism"]


def test_issue_roofline_arithmetic():
    """Issue rate = recorded warp instructions of a kernel group, scaled by
    sites from the captured case, over the group's event time per remesh."""
    import bench
    with open(os.path.join(ROOT, "profiles", "instructions.json")) as fh:
        rec = json.load(fh)["workloads"]["batched_12_meshes"]
    counts = rec["warp_instructions_per_remesh"]
    prof = {"grid": 0.12, "knn": 2.9, "clip": 0.9, "proj": 2.0}
    sites = 3 * rec["sites"]
    out = bench.issue_roofline("batched_256_meshes", prof, 100, 1965.0, sites, sms=148)
    assert out["bound"] == "issue" and out["peak"] == 148 * 4 * 1965e6
    assert "recorded" in out["counts"]
    assert set(out["kernels"]) == {" + ".join(ks) for ks in rec["groups"].values()}
    for group, kernels in rec["groups"].items():
        k = out["kernels"][" + ".join(kernels)]
        want = 3 * sum(counts[x] for x in kernels) / (prof[group] * 1e-3 * 100)
        assert abs(k["achieved"] - want) < 1e-6 * want
        assert abs(k["frac"] - k["achieved"] / out["peak"]) < 1e-12
        assert 0.0 < k["frac"] < 1.0
    assert bench.issue_roofline("batched_256_meshes", prof, 100, None, sites, sms=148) is None
    assert bench.issue_roofline("no_such_workload", prof, 100, 1965.0, sites, sms=148) is None


def test_traffic_recorded_scaling():
    """Recorded DRAM bytes of the site-KNN group (verify + search) scale with
    the launch's sites; unknown workloads and groups give no figure."""
    import bench
    with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
        rec = json.load(fh)["workloads"]["batched_12_meshes"]
    b, src = bench.traffic_recorded("batched_256_meshes", bench.KNN_GROUP, 2 * rec["sites"])
    want = 2 * (rec["bytes_per_launch"]["k_knn_verify"] + rec["bytes_per_launch"]["k_knn_search"])
    assert abs(b - want) < 1e-6 * want and "recorded" in src
    assert bench.traffic_recorded("torus_100k", bench.KNN_GROUP, 100000) == (None, None)
    assert bench.traffic_recorded("batched_256_meshes", "k_frame_vertex", 100000) == (None, None)


def test_clock_fallback_without_samples(monkeypatch):
    """A timed region shorter than the sampling period still reports a clock
    (one-shot queries around it), never None when any source answers."""
    import bench
    c = bench.Clocks(0)
    c.before = (1965.0, 1965.0)
    monkeypatch.setattr(bench, "_smi_once", lambda gpu: (1950.0, 1965.0))
    out = c.stop()
    assert out["samples"] == 0 and out["sm_mhz"] == (1965.0 + 1950.0) / 2 and out["sm_max_mhz"] == 1965.0
    assert "one-shot" in out["source"]
    c2 = bench.Clocks(0)
    monkeypatch.setattr(bench, "_smi_once", lambda gpu: None)
    monkeypatch.setattr(bench, "_nvml_max_clock", lambda gpu: 1965.0)
    out2 = c2.stop()
    assert out2["sm_mhz"] is None and out2["sm_max_mhz"] == 1965.0 and "NVML" in out2["source"]
