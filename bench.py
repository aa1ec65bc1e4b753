#!/usr/bin/env python
"""Benchmark: restricted-Voronoi CVT remeshing throughput on B200.

Default workload (``--workload batched``): 256 seeded procedural meshes
(spheres, tori, superquadrics; 5k-200k triangles each) with log-uniform site
counts in [1k, 50k] (about 3.1M sites in total), K=24, 100 Lloyd iterations,
freezing off (every site is recomputed in every iteration), mixed FP32/FP64
profile.  One *step* = one complete remesh of all 256 meshes as segments of
one engine.  ``value`` is sites x Lloyd-iterations per second over the timed
steps with the meshes and initial sites resident in HBM; beside it the line
carries the plain per-mesh loop (the same meshes one after another, as the
reference's driver runs them) with the batched/plain ratio, p50/p99 per-mesh
latency of both, per-mesh Hausdorff / bbox diagonal, the 1M-site rounded-box
figures (KNN + clip time per iteration and HBM fraction), and ``e2e``: the
same remesh through the one-call C ABI ``cvt_remesh_batch`` with pinned host
buffers (upload + iterate + download inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload batched|torus_100k|superellipsoid_1m|serve]

N > 1 (launched by torch.distributed.run): the meshes are partitioned over
the ranks by site count (the path shards at mesh granularity, with no
exchange step); value = all ranks' sites x iterations / the max-over-ranks
device time.  ``--impl reference`` times the CPU implementation of the same
path (the oracle port of the reference's algorithm, all host threads) on the
same configuration: every step runs whole remeshes (all 100 iterations) of
meshes drawn from a seeded permutation of the 256, and the rate of that
sample stands for the whole job.
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
L2_NOTE = "flushed (256 MiB write) before every timed step"


# ---------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _smi_once(gpu: int):
    """One read-only nvidia-smi query: (sm MHz, max sm MHz) or None."""
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=clocks.sm,clocks.max.sm", "--format=csv,noheader,nounits",
                              "-i", str(gpu)], capture_output=True, text=True, timeout=20).stdout
        a, b = [float(x) for x in out.strip().splitlines()[0].split(",")[:2]]
        return a, b
    except Exception:
        return None


def _nvml_max_clock(gpu: int):
    """The device's maximum SM clock from NVML (read-only), or None."""
    try:
        import pynvml
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByIndex(gpu)
            return float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        finally:
            pynvml.nvmlShutdown()
    except Exception:
        return None


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region.

    A timed region shorter than the 200 ms sampling period can end before
    the first sample; the clock then comes from one-shot queries taken just
    before and just after the region, or, failing those, from the device's
    maximum SM clock (NVML).  ``source`` says which."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None
        self.before = None

    def start(self):
        self.before = _smi_once(self.gpu)
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
        if self.proc is not None:
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
        if sm:
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                    "reasons": sorted(reasons), "source": "nvidia-smi -lms 200 during the timed region"}
        once = [x for x in (self.before, _smi_once(self.gpu)) if x]
        if once:
            return {"sm_mhz": statistics.median([a for a, _ in once]), "sm_max_mhz": max(b for _, b in once),
                    "samples": 0, "reasons": [],
                    "source": "no sample inside the timed region (shorter than the sampling period): "
                              "one-shot nvidia-smi queries just before and after it"}
        mx = _nvml_max_clock(self.gpu)
        return {"sm_mhz": None, "sm_max_mhz": mx, "samples": 0, "reasons": [],
                "source": "nvidia-smi unavailable; sm_max_mhz from NVML" if mx else "no clock source available"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s, earlier measurement on this pool)"


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


def _recorded(name):
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        return json.load(fh)


KNN_GROUP = "site_knn (k_knn_verify + k_knn_search)"
PROJ_GROUP = "projection (k_site_vsearch + k_site_proj)"


def _recorded_workload(name, workload):
    """The entry of a recorded capture for a workload: its own entry, else
    the entry recorded on a smaller case of the same family (`stands_for`
    is the family's name prefix)."""
    d = _recorded(name)
    ws = (d or {}).get("workloads", {})
    if workload in ws:
        return ws[workload]
    for w in ws.values():
        if w.get("stands_for") and workload.startswith(w["stands_for"]):
            return w
    return None


def traffic_recorded(workload, group, sites_in_launch):
    """DRAM read + write bytes per launch of a kernel group from a recorded
    ncu capture (profiles/traffic.json: dram__bytes_read.sum +
    dram__bytes_write.sum averaged over the launches of one remesh), scaled
    from the captured case's sites to this launch's sites.  (None, None)
    when nothing is recorded for the workload's family."""
    w = _recorded_workload("traffic.json", workload)
    if not w or group not in w.get("groups", {}):
        return None, None
    b = sum(float(w["bytes_per_launch"][k]) for k in w["groups"][group])
    return b * sites_in_launch / float(w["sites"]), \
        f"recorded ncu capture on {w['sites']} sites: {w['command']} (scaled by sites per launch)"


def issue_roofline(workload, prof, iters, sm_mhz, sites, sms=None):
    """Warp-instruction issue rate of the site kernels against the B200's
    issue peak (SMs x 4 schedulers x SM clock), the bound these kernels meet
    long before HBM.  Warp instructions per remesh come from a recorded ncu
    capture (profiles/instructions.json: smsp__inst_executed.sum summed over
    the launches of one remesh, scaled from the captured case's sites to
    `sites`); the kernel times come from this run's CUDA events.  None when
    no count is recorded for the workload's family or no clock is known."""
    w = _recorded_workload("instructions.json", workload)
    if not w or not sm_mhz:
        return None
    counts = w["warp_instructions_per_remesh"]
    if sms is None:
        import torch
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    peak = sms * 4 * sm_mhz * 1e6
    scale = sites / float(w["sites"])
    out = {"bound": "issue", "unit": "warp instructions/s", "peak": peak,
           "peak_from": f"{sms} SMs x 4 schedulers x {sm_mhz:.0f} MHz",
           "counts": f"recorded ncu capture on {w['sites']} sites, scaled to {sites}: {w['command']}; not this run",
           "kernels": {}}
    for group, kernels in w["groups"].items():
        if prof.get(group, 0) > 0:
            achieved = sum(counts[k] for k in kernels) * scale / (prof[group] * 1e-3 * iters)
            out["kernels"][" + ".join(kernels)] = {"achieved": achieved, "frac": achieved / peak}
    return out


# ---------------------------------------------------------------------------
# workloads and their configuration (identical in both arms)
# ---------------------------------------------------------------------------
def parallelism(ws):
    return "single GPU" if ws == 1 else f"{ws} GPUs, meshes partitioned over ranks by site count (no exchange)"


def batched_workload(n_meshes, ws):
    from gpu_cvt_b200 import workloads
    t0 = time.perf_counter()
    meshes = workloads.batched_set(seed=3, n_meshes=n_meshes)
    gen_s = time.perf_counter() - t0
    sizes = [int(S.shape[0]) for *_, S in meshes]
    tris = [int(F.shape[0]) for _, _, F, _ in meshes]
    cfg = {"workload": f"batched_{n_meshes}_meshes",
           "meshes": n_meshes, "seed": 3, "families": "spheres, tori, superquadrics (random parameters)",
           "tris_per_mesh": [min(tris), max(tris)], "sites_per_mesh": "log-uniform in [1000, 50000]",
           "sites_total": int(sum(sizes)), "k": 24, "iters": 100, "mode": 0, "freezing": "off",
           "profile": PROFILE, "kproj": 5, "l2": L2_NOTE, "parallelism": parallelism(ws)}
    return meshes, cfg, gen_s


def rank_share(meshes, ws, rank):
    """Indices of the meshes rank `rank` of `ws` remeshes: a size-balanced
    partition by site count, the same on every rank without communication."""
    from gpu_cvt_b200 import replicas
    sizes = [int(S.shape[0]) for *_, S in meshes]
    return replicas.partition(sizes, ws, rank) if ws > 1 else list(range(len(meshes)))


def torus_workload(ws):
    from gpu_cvt_b200 import meshgen as mg
    m, S, p = mg.workload_mesh("torus_100k")
    cfg = {"workload": "torus_100k",
           "mesh": "torus R=1 r=0.3, 200x100 grid (20,000 V / 40,000 F), N(0,0.002) normal noise, seed 1",
           "sites": int(S.shape[0]), "site_seed": 1, "k": p["k"], "iters": p["iters"], "mode": p["mode"],
           "freezing": "on", "profile": PROFILE, "kproj": 5, "l2": L2_NOTE, "parallelism": parallelism(ws)}
    return m, S, p, cfg


def cpu_sample(meshes, k, mode, iters, budget_s, seed=11, start=0, min_meshes=1):
    """The oracle port (all host threads) on whole remeshes of meshes drawn
    in a seeded order, until budget_s of CPU time is spent.  Returns
    (site-iterations, seconds, meshes used, next start)."""
    from oracle import oracle as O
    order = np.random.default_rng(seed).permutation(len(meshes))
    done, secs, used, i = 0, 0.0, 0, start
    while (secs < budget_s or used < min_meshes) and used < len(meshes):
        _, V, F, S = meshes[int(order[i % len(meshes)])]
        t0 = time.perf_counter()
        O.lloyd_run(V, F, S, k, mode, iters, profile=O.P_MIXED)
        secs += time.perf_counter() - t0
        done += int(S.shape[0]) * iters
        used += 1
        i += 1
    return done, secs, used, i


# ---------------------------------------------------------------------------
def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from oracle import oracle as O
    threads = O.max_threads()
    if args.workload == "batched":
        meshes, cfg, _ = batched_workload(args.meshes, ws)
        k, mode, iters = cfg["k"], cfg["mode"], cfg["iters"]
    elif args.workload == "torus_100k":
        m, S, p, cfg = torus_workload(ws)
        meshes = [("torus", m.V, m.F, S)]
        k, mode, iters = p["k"], p["mode"], p["iters"]
    else:
        print(json.dumps({"impl": "reference", "unavailable": f"no CPU arm for --workload {args.workload}"}))
        return 0
    per_step = args.ref_seconds / max(args.steps + args.warmup, 1)
    # warm-up steps: the smallest mesh, two iterations each (page-in, thread start-up)
    small = min(meshes, key=lambda x: x[3].shape[0])
    for _ in range(args.warmup):
        O.lloyd_run(small[1], small[2], small[3], k, mode, 2, profile=O.P_MIXED)
    tot_si, tot_s, used, nxt = 0, 0.0, 0, 0
    times = []
    for _ in range(args.steps):
        si, secs, u, nxt = cpu_sample(meshes, k, mode, iters, per_step, start=nxt)
        tot_si += si
        tot_s += secs
        used += u
        times.append(secs)
    value = tot_si / tot_s
    sample = (f"{used} whole remeshes ({iters} iterations each, {tot_si / iters:.0f} sites) of meshes drawn in a "
              f"seeded order from the {len(meshes)} of the workload, {tot_s:.1f} s; the sample's rate stands for "
              f"the whole job (extrapolated)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
            "higher_is_better": True, "scaling": "strong" if args.workload == "batched" else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def _init_dist(ws, local):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))


def _max_over_ranks(x, ws):
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws):
    import torch
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def run_ours_batched(args):
    import torch
    from gpu_cvt_b200 import _lib, workloads
    from gpu_cvt_b200 import engine as E

    ws, rank, local = dist_setup()
    _init_dist(ws, local)
    meshes_all, cfg, gen_s = batched_workload(args.meshes, ws)
    sizes = [int(S.shape[0]) for *_, S in meshes_all]
    mine = rank_share(meshes_all, ws, rank)
    meshes = [meshes_all[i] for i in mine]
    K, mode, iters = cfg["k"], cfg["mode"], cfg["iters"]
    n_mine = sum(int(S.shape[0]) for *_, S in meshes)
    n_all = int(sum(sizes))
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    # launch shapes from the autotuner on this rank's largest mesh (untimed;
    # results never depend on them)
    _, Vb, Fb, Sb = max(meshes, key=lambda x: x[3].shape[0])
    prm, tune_ms = workloads.tune_for(Vb, Fb, Sb, k=K, mode=mode, profile=PROFILE)
    if args.no_reuse:
        prm.knn_reuse = 0
    M = [E.Mesh(V, F) for _, V, F, _ in meshes]
    cells = sum(E.grid_cells(m, S.shape[0], K) for m, (*_, S) in zip(M, meshes))
    eng = E.Engine(prm, len(M), n_mine, cells)
    S_dev = [torch.from_numpy(S).cuda() for *_, S in meshes]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    segs = []

    def reset():
        for g in segs:
            eng.remove(g)
        segs.clear()
        segs.extend(eng.add(m, s, sp) for m, s in zip(M, S_dev))

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

    warm, wl = [], []
    for _ in range(max(args.warmup, 3)):
        step(warm, wl)
    _barrier(ws)
    clocks = Clocks(local)
    clocks.start()
    times, launches = [], []
    for _ in range(args.steps):
        step(times, launches)
    _barrier(ws)
    clk = clocks.stop()
    tot = _max_over_ranks(float(sum(times)), ws)
    value = n_all * iters * args.steps / (tot / 1e3)
    finals = [eng.sites(g) for g in segs]
    evals = [eng.evaluate(g) for g in segs]
    dH_rel = np.array([ev["dH_rel"] for ev in evals], np.float64)

    # ---- the plain per-mesh loop: same meshes, same kernels, one at a time --
    plain = None
    if not args.no_plain:
        tp, pfinals, each = workloads.run_plain_loop(meshes, k=K, mode=mode, profile=PROFILE, iters=iters,
                                                     prm=prm, per_mesh=True)
        tp = _max_over_ranks(tp, ws)
        each_ms = np.array(each) * 1e3
        done_ms = np.cumsum(each_ms)
        plain = {"value": n_all * iters / tp, "unit": UNIT, "ms": tp * 1e3,
                 "latency_ms": {"p50": float(np.percentile(each_ms, 50)), "p99": float(np.percentile(each_ms, 99)),
                                "what": "device time of one mesh's remesh, meshes run one after another"},
                 "completion_ms": {"p50": float(np.percentile(done_ms, 50)),
                                   "p99": float(np.percentile(done_ms, 99)),
                                   "what": "time from the job's start until the mesh's result is ready"},
                 "identical_results": bool(all(np.array_equal(a, b) for a, b in zip(finals, pfinals)))}

    # ---- e2e through the one-call batched C ABI with pinned host buffers ----
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    Vh = [pin(V) for _, V, _, _ in meshes]
    Fh = [pin(F) for _, _, F, _ in meshes]
    Sh = [pin(S) for *_, S in meshes]
    Oh = [torch.empty((int(S.shape[0]), 3), dtype=torch.float32).pin_memory() for *_, S in meshes]
    e2e_t, e2e_wall = [], []
    for r in range(3):
        ds = torch.cuda.default_stream()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e0.record(ds)
        E.remesh_batch(Vh, Fh, Sh, prm, iters, outs=Oh)
        e1.record(ds)
        e1.synchronize()
        if r > 0:   # the first call is the warm-up
            e2e_t.append(e0.elapsed_time(e1))
            e2e_wall.append((time.perf_counter() - w0) * 1e3)
    e2e_ms = _max_over_ranks(float(np.mean(e2e_t)), ws)
    same_as_engine = bool(all(np.array_equal(o.numpy(), f) for o, f in zip(Oh, finals)))
    h2d = int(sum(v.numel() * 4 + f.numel() * 4 + s.numel() * 4 for v, f, s in zip(Vh, Fh, Sh)))
    d2h = int(sum(o.numel() * 4 for o in Oh))

    # ---- per-kernel timing over one whole batched remesh ----------------
    reset()
    prof = eng.profile(iters, sp)
    big = sorted(range(len(segs)), key=lambda j: -int(meshes[j][3].shape[0]))[:8]
    reuse = knn_reuse_share(eng, [segs[j] for j in big], iters)
    reuse["over"] = "the 8 meshes with the most sites, one whole remesh"
    groups = {KNN_GROUP: (prof["knn"], n_mine * knn_bytes_per_site(K)),
              "k_site_clip": (prof["clip"], n_mine * clip_bytes_per_site(K)),
              PROJ_GROUP: (prof["proj"], n_mine * proj_bytes_per_site(K))}
    dom = max(groups, key=lambda g: groups[g][0])
    ms, alg_bytes = groups[dom]
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    tr, tr_src = traffic_recorded(cfg["workload"], dom, n_mine)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": tr, "traffic_source": tr_src, "kernel": dom,
                "algorithmic_bytes_per_launch": alg_bytes, "ms_per_launch": ms, "peak_source": peak_kind,
                "stage_ms_per_iter": {k: round(v, 5) for k, v in prof.items()},
                "knn_clip": {"ms_per_iter": prof["knn"] + prof["clip"],
                             "achieved_gbs": n_mine * (knn_bytes_per_site(K) + clip_bytes_per_site(K))
                             / ((prof["knn"] + prof["clip"]) * 1e-3) / 1e9}}
    roofline["knn_clip"]["frac"] = roofline["knn_clip"]["achieved_gbs"] / peak
    sm_clock = clk.get("sm_mhz") or clk.get("sm_max_mhz")
    ir = issue_roofline(cfg["workload"], prof, iters, sm_clock, n_mine)

    # ---- accuracy: the same remesh with FP64 state and arithmetic ---------
    acc = None
    if not args.no_accuracy:
        e64 = E.Engine(E.params(k=K, mode=mode, profile="fp64"), len(M), n_mine, cells)
        g64 = [e64.add(m, s, sp) for m, s in zip(M, S_dev)]
        e64.run(iters, sp)
        drift = []
        ddH = []
        for j, g in enumerate(g64):
            S64 = e64.sites_f64(g)
            drift.append(np.linalg.norm(finals[j].astype(np.float64) - S64, axis=1) / M[j].diag)
            ddH.append(abs(evals[j]["dH"] - e64.evaluate(g)["dH"]) / M[j].diag)
        e64.close()
        d = np.concatenate(drift)
        acc = {"site_drift_vs_fp64": {"max": float(d.max()), "p99": float(np.percentile(d, 99)),
                                      "mean": float(d.mean())},
               "hausdorff_minus_fp64_max": float(max(ddH)),
               "unit": "fraction of each mesh's bbox diagonal",
               "fp64": "same engine, FP64 state and arithmetic (bit-identical to the FP64 oracle)"}

    # ---- 1M sites on the jittered rounded box (rank 0) ---------------------
    c3 = None
    if rank == 0 and not args.no_c3:
        c3 = c3_figures(peak, peak_kind, reuse=not args.no_reuse)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        si, secs, used, _ = cpu_sample(meshes_all, K, mode, iters, args.cpu_seconds)
        from oracle import oracle as O
        cpu = {"value": si / secs, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
               "sample": f"{used} whole remeshes ({iters} iterations each, {si / iters:.0f} sites) of meshes drawn "
                         f"in a seeded order, mixed profile, {secs:.1f} s"}

    eng.close()
    for m in M:
        m.close()
    if rank == 0:
        batched_lat = float(np.percentile(times, 50)), float(np.percentile(times, 99))
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": tot / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
                "latency_ms": {"p50": batched_lat[0], "p99": batched_lat[1],
                               "what": "batched: every mesh's result is ready when the step ends, so a mesh's "
                                       "latency is the step's device time (p50/p99 over the timed steps)"},
                "plain_loop": plain,
                "batched_over_plain": (value / plain["value"]) if plain else None,
                "hausdorff_rel": {"p50": float(np.median(dH_rel)), "max": float(dH_rel.max()),
                                  "what": "per mesh, one-sided (dual mesh -> input), / bbox diagonal"},
                "e2e": {"value": n_all * iters / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "wall_ms_per_step": float(np.mean(e2e_wall)),
                        "api": "cvt_remesh_batch (pinned host buffers; mesh ingest, upload, iterations, download)",
                        "same_sites_as_engine": same_as_engine},
                "gpu_launches": int(sum(launches)),
                "roofline": roofline, "issue_roofline": ir, "knn_reuse": reuse, "superellipsoid_1m": c3,
                "cpu_baseline": cpu, "accuracy": acc, "clocks": clk,
                "tiles": E.tiles(prm), "tune_ms_per_iter": tune_ms, "mesh_generation_s": gen_s,
                "libgpucvt_launches_total": _lib.launch_count()}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def knn_reuse_share(eng, segs, iters):
    """Share of the site KNN lists taken from the kept candidate lists (the
    rest were full searches) over the segments' last `iters` iterations."""
    r = s = 0
    for g in segs:
        for i in range(iters):
            st = eng.stats(g, i)
            r += st["knn_reused"]
            s += st["knn_searched"]
    return {"reused": r, "searched": s, "share": r / max(r + s, 1)}


def c3_figures(peak, peak_kind, iters=200, k=32, reuse=True):
    """1M area-uniform sites on the rounded box |x|^8+|y|^8+|z|^8=1 (~2M
    triangles, 1% jittered by 1e-3), K=32, 200 iterations, freezing on,
    mixed profile: remesh time, KNN + clip time per iteration and its HBM
    fraction (while every site is active, and averaged over the run)."""
    import torch
    from gpu_cvt_b200 import engine as E, meshgen as mg
    m = mg.superellipsoid(8.0, 2_000_000, 0.01, 1e-3, seed=2)
    S0 = mg.sample_sites(m.V, m.F, 1_000_000, seed=2)
    n = S0.shape[0]
    M = E.Mesh(m.V, m.F)
    cells = E.grid_cells(M, n, k)
    eng = E.Engine(E.params(k=k, mode=1, profile=PROFILE, knn_reuse=reuse), 1, n, cells)
    st = torch.cuda.current_stream()
    sp = st.cuda_stream
    g = eng.add(M, S0, sp)
    eng.run(2, sp)                     # graph capture (untimed)
    torch.cuda.synchronize()
    eng.remove(g)
    g = eng.add(M, S0, sp)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    eng.run(iters, sp)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ev = eng.evaluate(g)
    eng.remove(g)
    g = eng.add(M, S0, sp)
    first = eng.profile(3, sp)          # iterations 0-2: every site active
    eng.remove(g)
    g = eng.add(M, S0, sp)
    whole = eng.profile(iters, sp)
    reuse = knn_reuse_share(eng, [g], iters)
    eng.close()
    M.close()
    b = n * (knn_bytes_per_site(k) + clip_bytes_per_site(k))
    kc_first = first["knn"] + first["clip"]
    kc_avg = whole["knn"] + whole["clip"]
    return {"mesh": f"superellipsoid p=8, {m.nF} triangles, 1% jittered by 1e-3 (seed 2)", "sites": n, "k": k,
            "iters": iters, "mode": 1, "profile": PROFILE, "ms_per_remesh": ms,
            "sites_iters_per_s": n * iters / (ms / 1e3), "dH_rel": ev["dH_rel"],
            "knn_clip_ms_per_iter": {"all_sites_active": kc_first, "run_average": kc_avg},
            "knn_clip_hbm_frac_all_active": b / (kc_first * 1e-3) / 1e9 / peak,
            "knn_clip_bytes_per_site": knn_bytes_per_site(k) + clip_bytes_per_site(k),
            "peak_gbs": peak, "peak_source": peak_kind,
            "stage_ms_per_iter_all_active": {k_: round(v, 5) for k_, v in first.items()},
            "stage_ms_per_iter_run_average": {k_: round(v, 5) for k_, v in whole.items()},
            "knn_reuse": reuse}


def run_ours_torus(args):
    import torch
    from gpu_cvt_b200 import engine as E
    from gpu_cvt_b200 import _lib

    ws, rank, local = dist_setup()
    _init_dist(ws, local)
    m, S, p, cfg = torus_workload(ws)
    n, iters = S.shape[0], p["iters"]
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    mesh = E.Mesh(m.V, m.F)
    cells = E.grid_cells(mesh, n, p["k"])
    prm, tune_ms = E.autotune(mesh, S, E.params(k=p["k"], mode=p["mode"], profile=PROFILE), iters=4)
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

    warm, wl = [], []
    for _ in range(max(args.warmup, 3)):
        step(warm, wl)
    _barrier(ws)
    clocks = Clocks(local)
    clocks.start()
    times, launches = [], []
    for _ in range(args.steps):
        step(times, launches)
    _barrier(ws)
    clk = clocks.stop()
    tot = _max_over_ranks(float(sum(times)), ws)
    value = ws * n * iters * args.steps / (tot / 1e3)
    seg = state["seg"]
    final = eng.sites(seg)
    frozen = int(eng.state(seg)["frozen"].sum())

    V, F = m.V, m.F
    e2e_t = []
    for r in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(torch.cuda.default_stream())
        out, _ = E.remesh(V, F, S, iters=iters, with_counts=True, prm=prm)
        e1.record(torch.cuda.default_stream())
        e1.synchronize()
        if r > 0:
            e2e_t.append(e0.elapsed_time(e1))
    e2e_ms = _max_over_ranks(float(np.mean(e2e_t)), ws)
    same_as_engine = bool(np.array_equal(out, final))
    h2d = int(V.nbytes + F.nbytes + S.nbytes)
    d2h = int(S.nbytes + 16 * iters)

    reset()
    prof = eng.profile(iters, sp)
    K = p["k"]
    newly = np.array([eng.stats(state["seg"], i)["newly_frozen"] for i in range(iters)], np.float64)
    active_mean = float(np.mean(n - np.concatenate([[0.0], np.cumsum(newly)[:-1]])))
    groups = {KNN_GROUP: (prof["knn"], active_mean * knn_bytes_per_site(K)),
              "k_site_clip": (prof["clip"], n * clip_bytes_per_site(K)),
              PROJ_GROUP: (prof["proj"], n * proj_bytes_per_site(K))}
    dom = max(groups, key=lambda g: groups[g][0])
    ms, alg_bytes = groups[dom]
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    tr, tr_src = traffic_recorded(cfg["workload"], dom, n)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": tr, "traffic_source": tr_src, "kernel": dom,
                "algorithmic_bytes_per_launch": alg_bytes, "ms_per_launch": ms, "peak_source": peak_kind,
                "stage_ms_per_iter": {k: round(v, 5) for k, v in prof.items()}}

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
        si, secs, used, _ = cpu_sample([("torus", m.V, m.F, S)], K, p["mode"], iters, args.cpu_seconds)
        from oracle import oracle as O
        cpu = {"value": si / secs, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
               "sample": f"{used} whole remesh(es) of {n} sites x {iters} iterations, mixed profile, {secs:.1f} s"}

    eng.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": tot / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
                "latency_ms": {"p50": float(np.percentile(times, 50)), "p99": float(np.percentile(times, 99)),
                               "what": "one full remesh (100 iterations), device time"},
                "frozen_sites_at_end": frozen,
                "e2e": {"value": ws * n * iters / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "api": "cvt_remesh (host buffers)",
                        "same_sites_as_engine": same_as_engine},
                "gpu_launches": int(sum(launches)),
                "roofline": roofline,
                "issue_roofline": issue_roofline(cfg["workload"], prof, iters, clk.get("sm_mhz") or clk.get("sm_max_mhz"), n),
                "cpu_baseline": cpu, "accuracy": acc, "clocks": clk, "tiles": E.tiles(prm),
                "libgpucvt_launches_total": _lib.launch_count()}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
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
    classes = server.size_classes(plain_reqs)
    ceiling = server.batching_ceiling(plain_reqs, plain["makespan_s"])
    line = {"metric": METRIC, "value": served["sites_iters_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": served["makespan_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "serve_poisson", "requests": args.requests, "rate_per_s": 200.0, "seed": 4,
                       "sites_per_request": [2000, 2000000], "stop": "max motion < 1e-4 bbox diag, cap 150",
                       "k": 24, "mode": 1, "profile": "mixed", "hbm_budget_gb": args.hbm_gb,
                       "sites_total": int(sum(r.n for r in reqs))},
            "tiles": E.tiles(prm),
            "latency_s": {"p50": served["latency_p50_s"], "p99": served["latency_p99_s"],
                          "mean": served["latency_mean_s"]},
            "served": served, "plain_fifo": plain,
            "served_over_plain": served["sites_iters_per_s"] / plain["sites_iters_per_s"],
            "plain_by_request_size": classes, "batching_ceiling": ceiling,
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


def run_options(args):
    """The projection (one-ring / BVH) and frame (vertex normal / PCA)
    options on the 100k-site torus and the 1M-site rounded box: mixed
    profile against FP64 with the same options."""
    import torch
    from gpu_cvt_b200 import workloads
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    res = [workloads.options_study(c) for c in ("torus_100k", "superellipsoid_1m")]
    print(json.dumps({"workload": "options", "studies": res}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["batched", "torus_100k", "serve", "superellipsoid_1m", "options"],
                    default="batched")
    ap.add_argument("--meshes", type=int, default=256, help="batched workload: number of meshes (256)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-seconds", type=float, default=120.0,
                    help="reference arm: seconds of CPU work to size the steps for")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="batched: skip the plain per-mesh loop")
    ap.add_argument("--no-c3", action="store_true", help="batched: skip the 1M-site rounded-box figures")
    ap.add_argument("--no-reuse", action="store_true", help="full KNN searches every iteration (knn_reuse off)")
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--hbm-gb", type=int, default=4)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_ours_batched(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "superellipsoid_1m":
        return run_precision(args)
    if args.workload == "options":
        return run_options(args)
    return run_ours_torus(args)


if __name__ == "__main__":
    sys.exit(main())
