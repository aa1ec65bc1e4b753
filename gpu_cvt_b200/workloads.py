"""The multi-mesh workloads: batched (many meshes in one engine) and the
plain per-mesh loop it is measured against.

Batched: a seeded set of procedural meshes (spheres, tori, superquadrics,
5k-200k triangles each) with log-uniform site counts, all placed as segments
of ONE engine, so every Lloyd iteration of every mesh is one pass of the fused
kernels replayed from a CUDA graph.  Plain loop: the same meshes one after
another through the same engine type (one segment at a time) -- the way the
reference's driver handles one mesh per process run.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import engine as E
from . import meshgen as mg


def batched_set(seed: int = 3, n_meshes: int = 256, tri_lo: int = 5_000, tri_hi: int = 200_000,
                site_lo: int = 1_000, site_hi: int = 50_000):
    """[(name, V, F, sites)] for the batched workload (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_meshes):
        m = mg.procedural_family(rng, tri_lo, tri_hi)
        n = int(round(math.exp(rng.uniform(math.log(site_lo), math.log(site_hi)))))
        S = mg.sample_sites(m.V, m.F, n, seed=int(rng.integers(0, 2**31 - 1)))
        out.append((m.name, m.V, m.F, S))
    return out


def _sync():
    import torch
    torch.cuda.synchronize()


def run_batched(meshes, k=24, mode=0, profile="ref", iters=100, stream=None, prm=None):
    """All meshes as segments of one engine; returns (seconds, engine, segs).
    Mesh upload/preprocessing is outside the timed region.  prm (e.g. from
    tune_for) replaces the default parameters."""
    import torch
    M = [E.Mesh(V, F) for _, V, F, _ in meshes]
    n_tot = sum(S.shape[0] for *_, S in meshes)
    cells = sum(E.grid_cells(m, S.shape[0], k) for m, (*_, S) in zip(M, meshes))
    eng = E.Engine(prm if prm is not None else E.params(k=k, mode=mode, profile=profile), len(meshes), n_tot, cells)
    segs = [eng.add(m, S) for m, (*_, S) in zip(M, meshes)]
    eng.run(1, stream)          # graph capture + first iteration (untimed warm-up)
    _sync()
    for s in list(segs):        # restart every segment from its initial sites
        eng.remove(s)
    segs = [eng.add(m, S) for m, (*_, S) in zip(M, meshes)]
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    eng.run(iters, C_stream(st))
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, eng, segs, M


def run_plain_loop(meshes, k=24, mode=0, profile="ref", iters=100, prm=None, per_mesh=False):
    """One mesh at a time through one engine sized for the largest; every
    mesh's 100 iterations replayed from the same CUDA graphs.  Returns
    (total seconds, final sites per mesh[, device seconds per mesh])."""
    import torch
    M = [E.Mesh(V, F) for _, V, F, _ in meshes]
    nmax = max(S.shape[0] for *_, S in meshes)
    cells = max(E.grid_cells(m, S.shape[0], k) for m, (*_, S) in zip(M, meshes))
    eng = E.Engine(prm if prm is not None else E.params(k=k, mode=mode, profile=profile), 1, nmax, cells)
    st = torch.cuda.current_stream()
    g = eng.add(M[0], meshes[0][3])
    eng.run(2, C_stream(st))    # graph capture (untimed)
    _sync()
    eng.remove(g)
    total = 0.0
    finals, each = [], []
    for m, (*_, S) in zip(M, meshes):
        g = eng.add(m, S)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        eng.run(iters, C_stream(st))
        e1.record(st)
        e1.synchronize()
        each.append(e0.elapsed_time(e1) / 1e3)
        total += each[-1]
        finals.append(eng.sites(g))
        eng.remove(g)
    eng.close()
    for m in M:
        m.close()
    return (total, finals, each) if per_mesh else (total, finals)


def C_stream(st):
    import ctypes
    return ctypes.c_void_p(st.cuda_stream)


def tune_for(V, F, sites, k=24, mode=0, profile="ref", iters=4):
    """Launch shapes from the autotuner (cvt_autotune) on one mesh and site
    set: (tuned params, their per-iteration ms).  Results do not depend on
    the shapes, only the time does."""
    m = E.Mesh(V, F)
    try:
        return E.autotune(m, sites, E.params(k=k, mode=mode, profile=profile), iters=iters)
    finally:
        m.close()


def batched_vs_plain(n_meshes=256, iters=100, k=24, mode=0, profile="ref", seed=3, check=True):
    t0 = time.perf_counter()
    meshes = batched_set(seed=seed, n_meshes=n_meshes)
    gen_s = time.perf_counter() - t0
    n_tot = sum(S.shape[0] for *_, S in meshes)
    # launch shapes tuned on the mesh with the most sites (untimed), used by
    # both the batched engine and the plain loop
    _, Vb, Fb, Sb = max(meshes, key=lambda x: x[3].shape[0])
    prm, tune_ms = tune_for(Vb, Fb, Sb, k=k, mode=mode, profile=profile)
    tb, eng, segs, M = run_batched(meshes, k=k, mode=mode, profile=profile, iters=iters, prm=prm)
    batched_sites = [eng.sites(s) for s in segs]
    eng.close()
    for m in M:
        m.close()
    tp, finals = run_plain_loop(meshes, k=k, mode=mode, profile=profile, iters=iters, prm=prm)
    same = all(np.array_equal(a, b) for a, b in zip(batched_sites, finals)) if check else None
    tris = [F.shape[0] for _, _, F, _ in meshes]
    return {"meshes": n_meshes, "sites_total": int(n_tot), "tris_min": int(min(tris)), "tris_max": int(max(tris)),
            "k": k, "mode": mode, "profile": profile, "iters": iters,
            "batched_s": tb, "plain_loop_s": tp,
            "batched_sites_iters_per_s": n_tot * iters / tb, "plain_sites_iters_per_s": n_tot * iters / tp,
            "speedup": tp / tb, "identical_results": same, "mesh_generation_s": gen_s,
            "tiles": E.tiles(prm), "tune_ms_per_iter": tune_ms}


def precision_study(iters=200, k=32, mode=1, n_sites=1_000_000, tris=2_000_000, seed=2):
    """Rounded box |x|^8+|y|^8+|z|^8=1 (~2M triangles, 1% jittered by 1e-3),
    1M area-uniform sites, K=32: the same run in the ref (FP32), mixed and
    fp64 profiles; Hausdorff of each result and per-site drift against FP64."""
    import torch
    t0 = time.perf_counter()
    m = mg.superellipsoid(8.0, tris, 0.01, 1e-3, seed=seed)
    S0 = mg.sample_sites(m.V, m.F, n_sites, seed=seed)
    gen_s = time.perf_counter() - t0
    M = E.Mesh(m.V, m.F)
    cells = E.grid_cells(M, n_sites, k)
    out = {"mesh": f"superellipsoid p=8, {m.nF} triangles, 1% jittered by 1e-3 (seed {seed})",
           "sites": n_sites, "k": k, "mode": mode, "iters": iters, "generation_s": gen_s}
    sites = {}
    for prof in ("ref", "mixed", "fp64"):
        eng = E.Engine(E.params(k=k, mode=mode, profile=prof), 1, n_sites, cells)
        g = eng.add(M, S0)
        eng.run(1)                      # graph capture, first iteration
        _sync()
        eng.remove(g)
        g = eng.add(M, S0)
        st = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        eng.run(iters, C_stream(st))
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        ev = eng.evaluate(g)
        sites[prof] = eng.sites_f64(g) if prof == "fp64" else eng.sites(g).astype(np.float64)
        nfz = int(eng.state(g)["frozen"].sum())
        eng.close()
        out[prof] = {"ms": ms, "sites_iters_per_s": n_sites * iters / (ms / 1e3), "dH": ev["dH"],
                     "dH_rel": ev["dH_rel"], "n_faces": ev["n_faces"], "Qavg": ev["Qavg"], "Qmin": ev["Qmin"],
                     "frozen_end": nfz, "nan_sites": int(np.isnan(sites[prof]).any(axis=1).sum())}
    for prof in ("ref", "mixed"):
        d = np.linalg.norm(sites[prof] - sites["fp64"], axis=1) / M.diag
        d = d[np.isfinite(d)]
        out[prof]["drift_vs_fp64"] = {"max": float(d.max()), "mean": float(d.mean()),
                                      "p99": float(np.percentile(d, 99))}
        out[prof]["dH_minus_fp64_rel"] = (out[prof]["dH"] - out["fp64"]["dH"]) / M.diag
    M.close()
    return out


def options_study(case="torus_100k", combos=(("onering", "vertex"), ("bvh", "vertex"), ("onering", "pca"),
                                             ("bvh", "pca"))):
    """The projection and frame options on one workload: for each (proj,
    frame) combination the mixed-profile run against the FP64 run with the
    same options (per-site drift, Hausdorff difference), its Hausdorff and
    time.  case: "torus_100k" (100k sites, K=24, 100 iterations, mode 1) or
    "superellipsoid_1m" (1M sites on the jittered rounded box, K=32, 200
    iterations, mode 1)."""
    import torch
    if case == "torus_100k":
        m, S0, p = mg.workload_mesh("torus_100k")
        k, iters = p["k"], p["iters"]
    else:
        m = mg.superellipsoid(8.0, 2_000_000, 0.01, 1e-3, seed=2)
        S0 = mg.sample_sites(m.V, m.F, 1_000_000, seed=2)
        k, iters = 32, 200
    M = E.Mesh(m.V, m.F)
    cells = E.grid_cells(M, S0.shape[0], k)
    out = {"case": case, "sites": int(S0.shape[0]), "k": k, "iters": iters, "mode": 1, "rows": []}
    for proj, frame in combos:
        res = {}
        for prof in ("mixed", "fp64"):
            eng = E.Engine(E.params(k=k, mode=1, profile=prof, proj=proj, frame=frame), 1, S0.shape[0], cells)
            g = eng.add(M, S0)
            eng.run(1)
            _sync()
            eng.remove(g)
            g = eng.add(M, S0)
            st = torch.cuda.current_stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            eng.run(iters, C_stream(st))
            e1.record(st)
            e1.synchronize()
            ev = eng.evaluate(g)
            res[prof] = {"ms": e0.elapsed_time(e1), "dH": ev["dH"],
                         "S": eng.sites_f64(g) if prof == "fp64" else eng.sites(g).astype(np.float64)}
            eng.close()
        d = np.linalg.norm(res["mixed"]["S"] - res["fp64"]["S"], axis=1) / M.diag
        d = d[np.isfinite(d)]
        out["rows"].append({"proj": proj, "frame": frame, "ms_mixed": res["mixed"]["ms"], "ms_fp64": res["fp64"]["ms"],
                            "dH_rel_mixed": res["mixed"]["dH"] / M.diag, "dH_rel_fp64": res["fp64"]["dH"] / M.diag,
                            "dH_minus_fp64_rel": (res["mixed"]["dH"] - res["fp64"]["dH"]) / M.diag,
                            "drift_vs_fp64": {"mean": float(d.mean()), "p99": float(np.percentile(d, 99)),
                                              "max": float(d.max())}})
    M.close()
    return out
