#!/usr/bin/env python
"""Benchmark: restricted-Voronoi CVT remeshing throughput on B200.

One *step* = one complete remesh of the workload: 100 Lloyd iterations of
100,000 area-uniform sites on the noisy (R=1, r=0.3, 200x100) torus, K=24,
freezing on (mode 1), mixed FP32/FP64 profile.  ``value`` is sites x
Lloyd-iterations per second over the whole job with the mesh and initial
sites resident in HBM; ``e2e`` is the same metric through the one-call C ABI
(``cvt_remesh``: host arrays in, upload + iterate + download).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (launched by torch.distributed.run) runs independent replicas, one per
GPU (the path shards at mesh granularity; there is no exchange step), and
reports the aggregate over ranks with the max-over-ranks device time.
``--impl reference`` times the CPU implementation of the same path (the
oracle port of the reference's algorithm) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sites·Lloyd-iters/s and p50/p99 remesh latency, batched/served vs plain, equal Hausdorff"
UNIT = "sites*iters/s"
PROFILE = "mixed"


def workload():
    from gpu_cvt_b200 import meshgen as mg
    m, S, p = mg.workload_mesh("torus_100k")
    cfg = {"workload": "torus_100k",
           "mesh": "torus R=1 r=0.3, 200x100 grid (20,000 V / 40,000 F), N(0,0.002) normal noise, seed 1",
           "sites": int(S.shape[0]), "site_seed": 1, "k": p["k"], "iters": p["iters"], "mode": p["mode"],
           "profile": PROFILE, "kproj": 5, "l2": "flushed (256 MiB write) before every timed step"}
    return m, S, p, cfg


# ---------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# algorithmic bytes per site and launch (fp32 positions, uint32 ids; the
# mesh arrays are gathered from L2 and not counted, like the neighbours'
# positions, which are the sites' own positions read again)
def knn_bytes_per_site(K):
    # own position 12 + neighbour ids written 4K (the frame vertex is
    # written by the separate frame-vertex kernel)
    return 12 + 4 * K


def clip_bytes_per_site(K):
    # position 12 + neighbour ids read 4K + frame vertex id 4 + its normal 12
    # + frozen flag 1 + centroid written 12
    return 12 + 4 * K + 4 + 12 + 1 + 12


def proj_bytes_per_site(K):
    # centroid 12 + position 12 + vertex ids written 20 + new position 12 +
    # flags read 4 (frozen, same, streak, tier) and written 2
    return 12 + 12 + 20 + 12 + 4 + 2


def traffic_from_profiles(kernel_key):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        d = json.load(fh)
    return d.get(kernel_key)


def issue_roofline(prof, iters, sm_mhz, sms=None):
    """Warp-instruction issue rate of the site kernels against the B200's
    issue peak (SMs x 4 schedulers x SM clock), the bound these kernels meet
    long before HBM.  Warp instructions per remesh of this workload come from
    profiles/instructions.json (ncu smsp__inst_executed.sum over the launches
    of one remesh), the kernel times from this run's CUDA events (the
    projection group includes the deferred-site kernel and the bookkeeping)."""
    path = os.path.join(ROOT, "profiles", "instructions.json")
    if not os.path.exists(path) or not sm_mhz:
        return None
    with open(path) as fh:
        counts = json.load(fh)["warp_instructions_per_remesh"]
    if sms is None:
        import torch
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    peak = sms * 4 * sm_mhz * 1e6
    out = {"bound": "issue", "unit": "warp instructions/s", "peak": peak,
           "peak_from": f"{sms} SMs x 4 schedulers x {sm_mhz:.0f} MHz (median SM clock of the timed region)",
           "counts": "profiles/instructions.json", "kernels": {}}
    for kernel, group in (("k_site_knn", "knn"), ("k_site_clip", "clip"), ("k_site_proj", "proj")):
        if kernel in counts and prof.get(group, 0) > 0:
            achieved = counts[kernel] / (prof[group] * 1e-3 * iters)
            out["kernels"][kernel] = {"achieved": achieved, "frac": achieved / peak}
    return out


# ---------------------------------------------------------------------------
def cpu_baseline(m, S, p, budget_s=15.0):
    """The oracle port of the reference's algorithm on the host cores."""
    from oracle import oracle as O
    threads = O.max_threads()
    n = S.shape[0]
    t0 = time.perf_counter()
    O.lloyd_run(m.V, m.F, S, p["k"], p["mode"], 2, profile=O.P_MIXED)
    t2 = time.perf_counter() - t0
    it = int(max(2, min(p["iters"], budget_s / max(t2 / 2, 1e-6))))
    t0 = time.perf_counter()
    O.lloyd_run(m.V, m.F, S, p["k"], p["mode"], it, profile=O.P_MIXED)
    dt = time.perf_counter() - t0
    return {"value": n * it / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} sites x the first {it} of {p['iters']} Lloyd iterations (mode {p['mode']}, "
                      f"mixed profile), {dt:.1f} s"}


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    m, S, p, cfg = workload()
    from oracle import oracle as O
    threads = O.max_threads()
    n = S.shape[0]
    # size each step so that warmup + steps end within a few minutes
    t0 = time.perf_counter()
    O.lloyd_run(m.V, m.F, S, p["k"], p["mode"], 1, profile=O.P_MIXED)
    t1 = time.perf_counter() - t0
    per_step_budget = args.ref_seconds / max(args.steps + args.warmup, 1)
    it = int(max(1, min(p["iters"], per_step_budget / max(t1, 1e-6))))
    for _ in range(args.warmup):
        O.lloyd_run(m.V, m.F, S, p["k"], p["mode"], 1, profile=O.P_MIXED)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.lloyd_run(m.V, m.F, S, p["k"], p["mode"], it, profile=O.P_MIXED)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = n * it * args.steps / tot
    sample = f"{n} sites x the first {it} of {p['iters']} Lloyd iterations per step, mixed profile"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    from gpu_cvt_b200 import engine as E
    from gpu_cvt_b200 import _lib

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    m, S, p, cfg = workload()
    n, iters = S.shape[0], p["iters"]
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    mesh = E.Mesh(m.V, m.F)
    cells = E.grid_cells(mesh, n, p["k"])
    # launch shapes from the autotuner (untimed; results do not depend on them)
    prm, tune_ms = E.autotune(mesh, S, E.params(k=p["k"], mode=p["mode"], profile=PROFILE), iters=4)
    cfg = dict(cfg, tiles=E.tiles(prm))
    eng = E.Engine(prm, 1, n, cells)
    S_dev = torch.from_numpy(S).cuda()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    state = {"seg": None}

    def reset():
        if state["seg"] is not None:
            eng.remove(state["seg"])
        state["seg"] = eng.add(mesh, S_dev, sp)

    def step(timed_list, launches):
        reset()
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.run(iters, sp)
        e1.record(stream)
        e1.synchronize()
        timed_list.append(e0.elapsed_time(e1))
        launches.append(eng.last_launches())

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()

    warm, wl = [], []
    for _ in range(max(args.warmup, 3)):
        step(warm, wl)
    barrier()
    clocks = Clocks(local)
    clocks.start()
    times, launches = [], []
    for _ in range(args.steps):
        step(times, launches)
    barrier()
    clk = clocks.stop()
    tot = float(sum(times))
    if ws > 1:
        t = torch.tensor([tot], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot = float(t.item())
    value = ws * n * iters * args.steps / (tot / 1e3)
    lat = sorted(times)
    p50 = float(np.percentile(lat, 50))
    p99 = float(np.percentile(lat, 99))
    seg = state["seg"]
    final = eng.sites(seg)
    frozen = int(eng.state(seg)["frozen"].sum())

    # ---- e2e through the one-call C ABI with host buffers ----------------
    V, F = m.V, m.F
    e2e_t = []
    for k in range(3):
        out = np.empty_like(S)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(torch.cuda.default_stream())
        out, _ = E.remesh(V, F, S, iters=iters, with_counts=True, prm=prm)
        e1.record(torch.cuda.default_stream())
        e1.synchronize()
        if k > 0:
            e2e_t.append(e0.elapsed_time(e1))
    e2e_ms = float(np.mean(e2e_t))
    if ws > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    same_as_engine = bool(np.array_equal(out, final))
    h2d = int(V.nbytes + F.nbytes + S.nbytes)
    d2h = int(S.nbytes + 16 * iters)

    # ---- per-kernel timing (CUDA events on the launching stream) over one
    # whole remesh: average per launch of each kernel group --------------
    reset()
    prof = eng.profile(iters, sp)
    K = p["k"]
    # the KNN kernel runs for the sites not yet frozen at the start of each
    # iteration (frozen counts from the engine's per-iteration statistics)
    newly = np.array([eng.stats(state["seg"], i)["newly_frozen"] for i in range(iters)], np.float64)
    active_mean = float(np.mean(n - np.concatenate([[0.0], np.cumsum(newly)[:-1]])))
    groups = {"k_site_knn": (prof["knn"], active_mean * knn_bytes_per_site(K)),
              "k_site_clip": (prof["clip"], n * clip_bytes_per_site(K)),
              "k_site_proj": (prof["proj"], n * proj_bytes_per_site(K))}
    dom = max(groups, key=lambda g: groups[g][0])
    ms, alg_bytes = groups[dom]
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    tr = traffic_from_profiles(dom)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": tr, "kernel": dom, "algorithmic_bytes_per_launch": alg_bytes,
                "ms_per_launch": ms, "peak_source": peak_kind,
                "stage_ms_per_iter": {k: round(v, 5) for k, v in prof.items()}}

    # ---- accuracy: drift of the mixed profile vs FP64 state ----------------
    acc = None
    if not args.no_accuracy and rank == 0:
        e64 = E.Engine(E.params(k=K, mode=p["mode"], profile="fp64"), 1, n, cells)
        g = e64.add(mesh, S_dev, sp)
        e64.run(iters, sp)
        S64 = e64.sites_f64(g)
        e64.close()
        d = np.linalg.norm(final.astype(np.float64) - S64, axis=1)
        acc = {"max_site_drift_vs_fp64": float(d.max() / mesh.diag), "mean_site_drift_vs_fp64": float(d.mean() / mesh.diag),
               "unit": "fraction of bbox diagonal", "fp64": "same engine, FP64 state and arithmetic"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(m, S, p, budget_s=args.cpu_seconds)

    eng.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": tot / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(cfg, parallelism=f"replicas x{ws}" if ws > 1 else "single GPU"),
                "latency_ms": {"p50": p50, "p99": p99, "what": "one full remesh (100 iterations), device time"},
                "frozen_sites_at_end": frozen,
                "e2e": {"value": ws * n * iters / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "api": "cvt_remesh (host buffers)",
                        "same_sites_as_engine": same_as_engine},
                "gpu_launches": int(sum(launches)),
                "roofline": roofline,
                "issue_roofline": issue_roofline(prof, iters, clk.get("sm_mhz") or clk.get("sm_max_mhz")),
                "cpu_baseline": cpu, "accuracy": acc, "clocks": clk,
                "libgpucvt_launches_total": _lib.launch_count()}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batched(args):
    """256 procedural meshes (spheres, tori, superquadrics; 4.8k-200k
    triangles, ~3.1M sites in total, K=24, 100 iterations) as segments of one
    engine vs the plain per-mesh loop (same kernels, one mesh at a time)."""
    import torch
    from gpu_cvt_b200 import workloads
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    r = workloads.batched_vs_plain(n_meshes=args.meshes, iters=100, k=24, mode=0, profile="ref", seed=3)
    line = {"metric": METRIC, "value": r["batched_sites_iters_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": r["batched_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched_{args.meshes}_meshes", "seed": 3, "k": 24, "iters": 100, "mode": 0,
                       "profile": "ref", "sites_total": r["sites_total"],
                       "tris_per_mesh": [r["tris_min"], r["tris_max"]], "tiles": r["tiles"]},
            "plain_loop": {"value": r["plain_sites_iters_per_s"], "ms": r["plain_loop_s"] * 1e3},
            "batched_over_plain": r["speedup"], "identical_results": r["identical_results"],
            "mesh_generation_s": r["mesh_generation_s"]}
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """A Poisson request stream (64 requests, rate 200/s, seed 4) over
    procedural meshes, 2k-2M sites per request, each iterated until no site
    moves more than 1e-4 of the bbox diagonal (cap 150 iterations); continuous
    batching vs first-come-first-served one at a time."""
    import copy
    import torch
    from gpu_cvt_b200 import server
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    meshes, reqs = server.request_stream(n_requests=args.requests, rate=200.0, site_lo=2_000, site_hi=2_000_000,
                                         n_meshes=8, seed=4)
    gen_s = time.perf_counter() - t0
    # launch shapes tuned on the largest request (untimed), used by both loops
    from gpu_cvt_b200 import engine as E, meshgen as mg, workloads
    big = max(reqs, key=lambda r: r.n)
    Vb, Fb = meshes[big.mesh]
    prm, tune_ms = workloads.tune_for(Vb, Fb, mg.sample_sites(Vb, Fb, big.n, seed=big.seed % (2**31)), k=24, mode=1,
                                      profile="mixed")
    # warm-up: graph capture and first-touch costs on a tiny stream
    wm, wr = server.request_stream(n_requests=4, rate=1000.0, site_lo=1000, site_hi=5000, n_meshes=1, seed=5)
    srv = server.RemeshServer(meshes, hbm_budget=args.hbm_gb << 30, max_segments=64, prm=prm)
    srv_w = server.RemeshServer(wm, hbm_budget=64 << 20, max_segments=4, prm=prm)
    srv_w.run(wr)
    srv_w.close()
    plain_reqs = [copy.copy(r) for r in reqs]
    served = srv.run(reqs)
    srv.close()
    plain = server.serve_plain(srv.M, plain_reqs, prm=prm)
    line = {"metric": METRIC, "value": served["sites_iters_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": served["makespan_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "serve_poisson", "requests": args.requests, "rate_per_s": 200.0, "seed": 4,
                       "sites_per_request": [2000, 2000000], "stop": "max motion < 1e-4 bbox diag, cap 150",
                       "k": 24, "mode": 1, "profile": "mixed", "hbm_budget_gb": args.hbm_gb,
                       "sites_total": int(sum(r.n for r in reqs)), "tiles": E.tiles(prm)},
            "latency_s": {"p50": served["latency_p50_s"], "p99": served["latency_p99_s"],
                          "mean": served["latency_mean_s"]},
            "served": served, "plain_fifo": plain,
            "served_over_plain": served["sites_iters_per_s"] / plain["sites_iters_per_s"],
            "request_generation_s": gen_s}
    print(json.dumps(line), flush=True)
    return 0


def run_precision(args):
    """1M sites on the jittered rounded box |x|^8+|y|^8+|z|^8=1 (~2M
    triangles), K=32, 200 iterations in the FP32, mixed and FP64 profiles."""
    import torch
    from gpu_cvt_b200 import workloads
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    r = workloads.precision_study(iters=200, k=32, mode=1)
    line = {"metric": METRIC, "value": r["mixed"]["sites_iters_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": r["mixed"]["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "superellipsoid_1m", "mesh": r["mesh"], "sites": r["sites"], "k": 32,
                       "iters": 200, "mode": 1, "profile": "mixed"},
            "profiles": {p: r[p] for p in ("ref", "mixed", "fp64")}, "generation_s": r["generation_s"]}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=120.0,
                    help="reference arm: seconds of CPU work to size the steps for")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--workload", choices=["torus_100k", "batched", "serve", "superellipsoid_1m"],
                    default="torus_100k")
    ap.add_argument("--meshes", type=int, default=256)
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--hbm-gb", type=int, default=4)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "superellipsoid_1m":
        return run_precision(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
