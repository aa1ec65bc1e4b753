"""Remesh serving with continuous batching.

Requests (mesh, site count, seed, arrival time) stream in.  Meshes stay
resident (vertex grid, CSR, BVH on the device).  Every request becomes a
segment of one engine as soon as it has arrived and fits: its sites are
sampled on the device, its stop rule (max site motion below `tol` times the
mesh's bbox diagonal, at most `max_iters` iterations) is applied on the device
after every iteration, and all admitted requests iterate together, one CUDA
graph replay per Lloyd iteration.  Finished segments free their slots and
capacity for the next arrivals.  Admission is by an HBM budget: the engine's
site and grid-cell capacity is derived from it, and a request waits until its
sites and cells fit.

`serve_plain` is the baseline: the same requests one at a time, first come
first served, through a one-segment engine.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import engine as E
from . import meshgen as mg
from ._lib import CvtError

# device bytes per site held by an engine (positions x2, list, flags, grid
# build arrays, sorted copy) and per grid cell, for budget-derived capacity
BYTES_PER_SITE_BASE = 150
BYTES_PER_CELL = 8


@dataclass
class Request:
    rid: int
    mesh: int
    n: int
    seed: int
    arrival: float
    admitted: float = -1.0
    done: float = -1.0
    service: float = -1.0   # plain loop: seconds from admission to done
    iters: int = 0
    result: np.ndarray | None = field(default=None, repr=False)


def request_stream(n_requests=100, rate=200.0, site_lo=2_000, site_hi=2_000_000, n_meshes=8, seed=4):
    """Poisson arrivals (rate per second) over a pool of procedural meshes,
    log-uniform site counts.  Returns (meshes as (V,F) arrays, requests)."""
    rng = np.random.default_rng(seed)
    meshes = []
    for _ in range(n_meshes):
        m = mg.procedural_family(rng, 20_000, 200_000)
        meshes.append((m.V, m.F))
    t = 0.0
    reqs = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(round(math.exp(rng.uniform(math.log(site_lo), math.log(site_hi)))))
        reqs.append(Request(i, int(rng.integers(0, n_meshes)), n, int(rng.integers(0, 2**62)), t))
    return meshes, reqs


def _percentile(x, q):
    return float(np.percentile(np.asarray(x, np.float64), q)) if len(x) else float("nan")


class RemeshServer:
    def __init__(self, meshes, k=24, mode=1, profile="mixed", hbm_budget=4 << 30, max_segments=64, tol=1e-4,
                 max_iters=150, chunk=5, keep_results=False, prm=None):
        import torch
        self.torch = torch
        self.M = [m if isinstance(m, E.Mesh) else E.Mesh(*m) for m in meshes]
        self.k, self.tol, self.max_iters, self.chunk = k, tol, max_iters, chunk
        per_site = BYTES_PER_SITE_BASE + 4 * k
        # sites and their grid cells (a segment reserves at most 4 per site)
        self.max_sites = int(hbm_budget // (per_site + 4 * BYTES_PER_CELL))
        self.max_cells = int(4 * self.max_sites + 65 * max_segments)
        self.max_segments = max_segments
        self.engine = E.Engine(prm if prm is not None else E.params(k=k, mode=mode, profile=profile), max_segments,
                               self.max_sites, self.max_cells)
        self.keep_results = keep_results
        self.stream = torch.cuda.current_stream()
        self.sp = C.c_void_p(self.stream.cuda_stream)

    def _fits(self, r):
        return r.n <= self.max_sites

    def _admit(self, r, now):
        m = self.M[r.mesh]
        S = self.torch.empty((r.n, 3), dtype=self.torch.float32, device="cuda")
        m.sample_sites(S, r.seed, self.sp)
        try:
            seg = self.engine.add(m, S, self.sp)
        except CvtError as e:
            if e.status == 5:      # capacity: wait for running requests to finish
                return None
            raise
        self.engine.set_stop(seg, self.tol * m.diag, self.max_iters)
        r.admitted = now
        return seg

    def run(self, requests):
        """Serve `requests` (arrival times relative to the start).  Returns a
        dict of latency / throughput figures; requests are updated in place."""
        torch = self.torch
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        active = {}
        launches = 0
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now and len(active) < self.max_segments:
                r = pending[0]
                if not self._fits(r):
                    raise ValueError(f"request {r.rid} ({r.n} sites) exceeds the HBM budget")
                seg = self._admit(r, now)
                if seg is None:
                    break
                active[seg] = r
                pending.popleft()
            if not active:
                if pending:
                    time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - t0)))
                continue
            self.engine.run(self.chunk, self.sp)
            launches += self.engine.last_launches()
            iters, state = self.engine.poll(self.max_segments, self.sp)
            now = time.perf_counter() - t0
            for seg in [s for s in active if state[s] == 2]:
                r = active.pop(seg)
                r.done = now
                r.iters = int(iters[seg])
                if self.keep_results:
                    r.result = self.engine.sites(seg)
                self.engine.remove(seg)
        torch.cuda.synchronize()
        makespan = time.perf_counter() - t0
        lat = [r.done - r.arrival for r in requests]
        work = sum(r.n * r.iters for r in requests)
        return {"requests": len(requests), "makespan_s": makespan, "sites_iters": int(work),
                "sites_iters_per_s": work / makespan, "latency_p50_s": _percentile(lat, 50),
                "latency_p99_s": _percentile(lat, 99), "latency_mean_s": float(np.mean(lat)),
                "iters_mean": float(np.mean([r.iters for r in requests])), "gpu_launches": launches}

    def close(self):
        self.engine.close()


def serve_plain(meshes, requests, k=24, mode=1, profile="mixed", tol=1e-4, max_iters=150, chunk=5,
                keep_results=False, prm=None):
    """The baseline: one request at a time, first come first served."""
    import torch
    M = [m if isinstance(m, E.Mesh) else E.Mesh(*m) for m in meshes]
    nmax = max(r.n for r in requests)
    cells = max(E.grid_cells(M[r.mesh], r.n, k) for r in requests)
    eng = E.Engine(prm if prm is not None else E.params(k=k, mode=mode, profile=profile), 1, nmax, cells)
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    launches = 0
    t0 = time.perf_counter()
    for r in sorted(requests, key=lambda r: r.arrival):
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        m = M[r.mesh]
        S = torch.empty((r.n, 3), dtype=torch.float32, device="cuda")
        m.sample_sites(S, r.seed, sp)
        seg = eng.add(m, S, sp)
        eng.set_stop(seg, tol * m.diag, max_iters)
        r.admitted = time.perf_counter() - t0
        while True:
            eng.run(chunk, sp)
            launches += eng.last_launches()
            iters, state = eng.poll(1, sp)
            if state[seg] == 2:
                break
        r.done = time.perf_counter() - t0
        r.service = r.done - r.admitted
        r.iters = int(iters[seg])
        if keep_results:
            r.result = eng.sites(seg)
        eng.remove(seg)
    torch.cuda.synchronize()
    makespan = time.perf_counter() - t0
    lat = [r.done - r.arrival for r in requests]
    work = sum(r.n * r.iters for r in requests)
    eng.close()
    return {"requests": len(requests), "makespan_s": makespan, "sites_iters": int(work),
            "sites_iters_per_s": work / makespan, "latency_p50_s": _percentile(lat, 50),
            "latency_p99_s": _percentile(lat, 99), "latency_mean_s": float(np.mean(lat)),
            "iters_mean": float(np.mean([r.iters for r in requests])), "gpu_launches": launches}


def size_classes(requests, bounds=(20_000, 200_000)):
    """Per request-size class of a plain (one at a time) run: requests, share
    of the stream's site-iterations, and the sites x iterations per second
    each class reached alone (its work over its service time)."""
    out = []
    lo = 0
    for hi in list(bounds) + [None]:
        cls = [r for r in requests if r.n >= lo and (hi is None or r.n < hi)]
        work = sum(r.n * r.iters for r in cls)
        svc = sum(r.service for r in cls)
        out.append({"sites": [lo, hi], "requests": len(cls), "work_share": 0.0, "site_iters": int(work),
                    "plain_rate": work / svc if svc > 0 else None})
        lo = hi if hi is not None else lo
    tot = sum(c["site_iters"] for c in out)
    for c in out:
        c["work_share"] = c["site_iters"] / tot if tot else 0.0
    return out


def batching_ceiling(requests, plain_makespan):
    """Upper bound of the served/plain throughput ratio: even with perfect
    overlap, the stream's work takes at least its site-iterations divided by
    the best rate any single request reached in the plain loop (a large
    request already fills the GPU), and no earlier than the last arrival."""
    best = max(r.n * r.iters / r.service for r in requests if r.service > 0)
    work = sum(r.n * r.iters for r in requests)
    t_min = max(work / best, max(r.arrival for r in requests))
    return {"best_single_request_rate": best, "min_makespan_s": t_min, "max_ratio": plain_makespan / t_min}
