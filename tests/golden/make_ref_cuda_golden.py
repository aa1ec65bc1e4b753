"""Fixtures from the reference's own CUDA build (GPU box only).

    make -C oracle ref                      # in a container with the reference checkout
    python tests/golden/make_ref_cuda_golden.py [out_dir]

Runs oracle/_ref/ref_harness -- the reference's unmodified stage kernels
(site_knn.cuh, 2dClip.cuh, near_project.cuh, site_normals.cuh,
freezetest.cuh, buildmesh.cuh, evaluate.cuh) driven like main.cu:669-974 --
on seeded workloads and stores small .npz fixtures (the oracle tests compare
against them) plus ref_cuda_summary.json: the torus workload (100k sites,
K=24, 100 iterations, mode 1) run by the reference kernels and by libgpucvt,
with timings, Hausdorff figures and the site drift between the two.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from gpu_cvt_b200 import meshgen as mg  # noqa: E402
from oracle import ref_runner  # noqa: E402


def small_cases(out):
    m, S, _ = mg.workload_mesh("icosphere_2k")
    # the reference's own hub KNN (knn_mode 0): neighbour lists of iteration 0
    h = ref_runner.run(m.V, m.F, S, 20, 0, 1, knn_mode=0)
    np.savez_compressed(os.path.join(out, "ref_cuda_hubknn_icosphere_2k.npz"), S0=S, knn0=h["knn0"])
    # every other stage by the reference's kernels, exact KNN (knn_mode 1)
    r = ref_runner.run(m.V, m.F, S, 20, 0, 50, dump=[1, 2, 5, 10, 50])
    np.savez_compressed(os.path.join(out, "ref_cuda_icosphere_2k.npz"), S0=S, **{k: v for k, v in r.items()
                                                                               if k not in ("stage_ms",)})
    t = mg.torus(1.0, 0.3, 80, 40, noise_sigma=0.002, seed=1)
    St = mg.sample_sites(t.V, t.F, 4000, seed=1)
    for mode, dump in ((1, [1, 5, 30]), (2, [30])):
        r = ref_runner.run(t.V, t.F, St, 24, mode, 30, dump=dump)
        np.savez_compressed(os.path.join(out, f"ref_cuda_torus4k_mode{mode}.npz"), S0=St,
                            **{k: v for k, v in r.items() if k not in ("stage_ms",)})


def torus_100k(out):
    import torch
    from gpu_cvt_b200 import engine as E
    m, S, p = mg.workload_mesh("torus_100k")
    K, mode, iters = p["k"], p["mode"], p["iters"]
    # timing of the reference's own pipeline (hub KNN included); its neighbour
    # lists are corrupted on this GPU, so only the clock is kept from this run
    t0 = time.perf_counter()
    h = ref_runner.run(m.V, m.F, S, K, mode, iters, knn_mode=0)
    hub_wall = time.perf_counter() - t0
    t0 = time.perf_counter()
    r = ref_runner.run(m.V, m.F, S, K, mode, iters, dump=[1, iters])
    ref_wall = time.perf_counter() - t0
    diag = mg.bbox_diag(m.V)
    summ = {"workload": "torus_100k", "sites": int(S.shape[0]), "k": K, "mode": mode, "iters": iters,
            "reference_cuda_hub_knn_timing": {
                "loop_wall_ms": h["wall_ms"], "process_wall_s": hub_wall,
                "stage_ms_per_iter_mean": [float(x) for x in h["stage_ms"].mean(0)],
                "iter_remesh_ms_total": float(h["stage_ms"].sum()),
                "sites_iters_per_s_loop": S.shape[0] * iters / (h["wall_ms"] / 1e3),
                "note": "hub KNN returns corrupted ids on B200; timing only"},
            "reference_cuda": {"knn": "exact brute force (harness), all other stages the reference kernels",
                               "loop_wall_ms": r["wall_ms"], "process_wall_s": ref_wall,
                               "stage_ms_sum": float(r["stage_ms"].sum()),
                               "stage_ms_per_iter_mean": [float(x) for x in r["stage_ms"].mean(0)],
                               "stage_names": ["knn_sites", "knn_site_to_mesh", "uv", "centroids",
                                               "knn_centroid_to_mesh", "project"],
                               "sites_iters_per_s_loop": S.shape[0] * iters / (r["wall_ms"] / 1e3),
                               "frozen_end": int(r["frozen"].sum()), "dH": r["dH"], "dH_rel": r["dH"] / diag,
                               "quality": [float(x) for x in r["quality"]], "n_faces": r["nfaces"],
                               "counts_last": r["counts"][-1].tolist()}}
    M = E.Mesh(m.V, m.F)
    cells = E.grid_cells(M, S.shape[0], K)
    for prof in ("ref", "mixed", "fp64"):
        e = E.Engine(E.params(k=K, mode=mode, profile=prof), 1, S.shape[0], cells)
        g = e.add(M, S)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.run(iters)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        Sg = e.sites_f64(g) if prof == "fp64" else e.sites(g).astype(np.float64)
        ev = e.evaluate(g)
        st = e.state(g)
        summ[f"gpucvt_{prof}"] = {"run_wall_ms": dt * 1e3, "frozen_end": int(st["frozen"].sum()), "dH": ev["dH"],
                                  "dH_rel": ev["dH"] / diag, "n_faces": ev["n_faces"], "Qavg": ev["Qavg"],
                                  "sites": Sg}
        e.close()
    ref_final = r["S"][-1].astype(np.float64)
    ref_it1 = r["S"][0].astype(np.float64)
    S64 = summ["gpucvt_fp64"]["sites"]
    for prof in ("ref", "mixed", "fp64"):
        Sg = summ[f"gpucvt_{prof}"].pop("sites")
        d = np.linalg.norm(Sg - ref_final, axis=1) / diag
        summ[f"gpucvt_{prof}"]["drift_vs_reference_cuda"] = {"max": float(d.max()), "mean": float(d.mean()),
                                                            "p99": float(np.percentile(d, 99))}
        d64 = np.linalg.norm(Sg - S64, axis=1) / diag
        summ[f"gpucvt_{prof}"]["drift_vs_fp64"] = {"max": float(d64.max()), "mean": float(d64.mean())}
    d = np.linalg.norm(ref_final - S64, axis=1) / diag
    summ["reference_cuda"]["drift_vs_fp64"] = {"max": float(d.max()), "mean": float(d.mean())}
    # first iteration: all profiles start from identical sites
    e = E.Engine(E.params(k=K, mode=mode, profile="ref"), 1, S.shape[0], cells)
    g = e.add(M, S)
    e.run(1)
    d1 = np.linalg.norm(e.sites(g).astype(np.float64) - ref_it1, axis=1) / diag
    summ["gpucvt_ref"]["drift_vs_reference_cuda_iter1"] = {"max": float(d1.max()), "mean": float(d1.mean())}
    e.close()
    with open(os.path.join(out, "ref_cuda_summary.json"), "w") as fh:
        json.dump(summ, fh, indent=1)
    print(json.dumps(summ, indent=1))


def torus_100k_iters(out, r=None, ours=None):
    """The 100k-site torus (K=24, mode 1), iterations 1-10 by the reference's
    kernels against the engine's ref and mixed profiles: positions at
    iterations 1, 2, 5, 10 of every 20th site and of every site that strays
    more than 1e-6 of the diagonal in either profile, and, for those sites,
    whether the reference's first-iteration centroid is a projection tie
    (the best two faces of its one-rings within 1e-3 in squared distance).
    r / ours: results already computed (the harness run, {profile: sites per
    iteration}); run here when None."""
    import torch
    from gpu_cvt_b200 import engine as E
    from oracle import oracle as O
    m, S, p = mg.workload_mesh("torus_100k")
    diag = mg.bbox_diag(m.V)
    if r is None:
        r = ref_runner.run(m.V, m.F, S, p["k"], p["mode"], 10, dump=list(range(1, 11)))
    if ours is None:
        ours = {}
        M = E.Mesh(m.V, m.F)
        for prof in ("ref", "mixed"):
            e = E.Engine(E.params(k=p["k"], mode=p["mode"], profile=prof), 1, S.shape[0],
                         E.grid_cells(M, S.shape[0], p["k"]))
            g = e.add(M, S)
            arr = []
            for _ in range(10):
                e.run(1)
                arr.append(e.sites(g))
            ours[prof] = np.stack(arr)
            e.close()
        torch.cuda.synchronize()
    far = np.zeros(S.shape[0], bool)
    for prof in ("ref", "mixed"):
        d = np.linalg.norm(ours[prof].astype(np.float64) - r["S"].astype(np.float64), axis=2) / diag
        far |= (d > 1e-6).any(0)
    idx = np.union1d(np.arange(0, S.shape[0], 20), np.flatnonzero(far)).astype(np.int32)
    off, fcs = O.build_vf(m.nV, m.F)
    tie = np.zeros(idx.size, bool)
    for k, i in enumerate(idx):
        c = r["cent0"][i]
        d2 = sorted(float(((O.closest_point_tri(c, *m.V[m.F[f]]).astype(np.float64) - c) ** 2).sum())
                    for f in {int(f) for v in r["knnv0"][i] if v >= 0 for f in fcs[off[v]:off[v + 1]]})
        tie[k] = len(d2) > 1 and d2[1] - d2[0] <= 1e-3 * d2[1]
    iters = np.array([1, 2, 5, 10], np.int32)
    np.savez_compressed(os.path.join(out, "ref_cuda_torus100k_iters.npz"), idx=idx, iters=iters,
                        S=r["S"][iters - 1][:, idx], tie=tie, diag=np.float64(diag))


def superellipsoid_1m(out, iters=10):
    """The 1M-site rounded box (K=32, mode 1): iterations 1..iters by the
    reference's kernels against the engine's ref and mixed profiles (per
    iteration max / p99 / mean drift and sites above 1e-5 of the diagonal)
    and the one-sided Hausdorff figure after them; added to
    ref_cuda_summary.json as "superellipsoid_1m"."""
    from gpu_cvt_b200 import engine as E
    m = mg.superellipsoid(8.0, 2_000_000, 0.01, 1e-3, seed=2)
    S = mg.sample_sites(m.V, m.F, 1_000_000, seed=2)
    diag = mg.bbox_diag(m.V)
    r = ref_runner.run(m.V, m.F, S, 32, 1, iters, dump=list(range(1, iters + 1)), timeout=3000)
    M = E.Mesh(m.V, m.F)
    res = {"sites": int(S.shape[0]), "k": 32, "mode": 1, "iters": iters,
           "reference_cuda_dH_rel": r["dH"] / diag, "reference_frozen_end": int(r["frozen"].sum())}
    for prof in ("ref", "mixed"):
        e = E.Engine(E.params(k=32, mode=1, profile=prof), 1, S.shape[0], E.grid_cells(M, S.shape[0], 32))
        g = e.add(M, S)
        rows = []
        for it in range(iters):
            e.run(1)
            d = np.linalg.norm(e.sites(g).astype(np.float64) - r["S"][it].astype(np.float64), axis=1) / diag
            d = d[np.isfinite(d)]
            rows.append({"iter": it + 1, "max": float(d.max()), "p99": float(np.percentile(d, 99)),
                         "mean": float(d.mean()), "n_over_1e-5": int((d > 1e-5).sum())})
        res[prof] = {"drift_vs_reference_cuda": rows, "dH_rel": e.evaluate(g)["dH_rel"],
                     "frozen_end": int(e.state(g)["frozen"].sum())}
        e.close()
    path = os.path.join(out, "ref_cuda_summary.json")
    summ = json.load(open(path)) if os.path.exists(path) else {}
    summ["superellipsoid_1m"] = res
    with open(path, "w") as fh:
        json.dump(summ, fh, indent=1)


def main(out):
    os.makedirs(out, exist_ok=True)
    if not ref_runner.available():
        raise SystemExit("oracle/_ref/ref_harness is missing: build it with `make -C oracle ref`")
    small_cases(out)
    torus_100k(out)
    torus_100k_iters(out)
    superellipsoid_1m(out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
