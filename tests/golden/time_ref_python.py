"""Time the reference's own CPU path: ``lloyd_iter_sites_only`` of
Harper-Yan/GPU_CVT ``scripts/testfreeze.py`` (freezing off, as run by
``testfreeze2.py:172-195``) and ``hausdorff_bvh`` of ``scripts/evaluate.py``,
on this machine's host cores.

    python tests/golden/time_ref_python.py /path/to/reference

The reference's Python cannot travel to a GPU box, so this runs where the
checkout is; ``bench.py`` times the C++ restatement of the same algorithm on
the GPU box's host instead.  Workloads (seeded, gpu_cvt_b200.meshgen):

* icosphere level 5, 2,000 sites, K=20: 3 iterations;
* the torus of the bench (200x100 grid, N(0,0.002) noise), a 10,000-site
  sample of its 100,000 sites, K=24: 2 iterations.  The per-site work does
  not depend on the site count (the KNN is a KD-tree query), so the figure
  extrapolates per site-iteration;
* hausdorff_bvh between the icosphere level 3 and a perturbed level 2.

Prints one JSON line: sites*iterations/s per workload, the core count and
how cKDTree was threaded (workers=-1 in the reference: all cores).
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
sys.path.insert(0, HERE)

from gpu_cvt_b200 import meshgen as mg  # noqa: E402
from make_golden import _load, _stub  # noqa: E402


def lloyd_rate(tf, m, S, K, iters):
    from scipy.spatial import cKDTree
    from oracle import oracle as O
    N0 = O.vertex_normals(m.V, m.F).astype(np.float64)
    P0 = m.V.astype(np.float64)
    F0 = m.F.astype(np.int64)
    vf = [[] for _ in range(m.nV)]
    for fi, (a, b, c) in enumerate(m.F):
        vf[int(a)].append(fi)
        vf[int(b)].append(fi)
        vf[int(c)].append(fi)
    treeP0 = cKDTree(P0)
    S_it = S.astype(np.float64)
    _, idx0 = cKDTree(S_it).query(S_it, k=K + 1)
    idx0 = np.sort(idx0[:, 1:], axis=1)
    ntier = len(tf.TIERS)
    fs = {
        "frozen": np.zeros(len(S_it), dtype=bool),
        "low_streak": np.zeros(len(S_it), dtype=np.int64),
        "knn_hist": [idx0.copy()],
        "idxn_cached": idx0.copy(),
        "tier_id": np.zeros(len(S_it), dtype=np.int64),
        "disp_thr_arr": np.array([t[1] for t in tf.TIERS], dtype=np.float64),
        "streak_arr": np.full(ntier, 999999, dtype=np.int64),
        "neigh_win_arr": np.array([t[3] for t in tf.TIERS], dtype=np.int64),
        "jacc_thr_arr": np.array([t[4] for t in tf.TIERS], dtype=np.float64),
    }
    t0 = time.perf_counter()
    for _ in range(iters):
        S_it, fs, _ = tf.lloyd_iter_sites_only(S_it, P0, F0, N0, vf, treeP0, fs, k_neigh=K, k_proj=5)
    dt = time.perf_counter() - t0
    return {"sites": int(S.shape[0]), "k": K, "iters": iters, "seconds": dt, "sites_iters_per_s": S.shape[0] * iters / dt}


def main(ref_root: str) -> None:
    _stub("trimesh")
    _stub("open3d")
    tf = _load(os.path.join(ref_root, "scripts", "testfreeze.py"), "ref_testfreeze")
    ev = _load(os.path.join(ref_root, "scripts", "evaluate.py"), "ref_evaluate")
    out = {"cores": os.cpu_count(), "kdtree_workers": "-1 (all cores, as in the reference)"}
    ico = mg.icosphere(5)
    out["icosphere_2k"] = lloyd_rate(tf, ico, mg.sample_sites(ico.V, ico.F, 2000, seed=0), 20, 3)
    m, S, prm = mg.workload_mesh("torus_100k")
    out["torus_100k_10k_sample"] = lloyd_rate(tf, m, S[:10_000], 24, 2)
    mc = mg.icosphere(2)
    Vc = (mc.V * np.float32(1.01)).astype(np.float64)
    r = mg.icosphere(3)
    t0 = time.perf_counter()
    ev.hausdorff_bvh(Vc, mc.F.astype(np.int64), r.V.astype(np.float64), r.F.astype(np.int64), leaf_size=8)
    dt = time.perf_counter() - t0
    probes = (mc.nV + 4 * mc.nF) + (r.nV + 4 * r.nF)
    out["hausdorff_bvh"] = {"probes": probes, "seconds": dt, "probes_per_s": probes / dt}
    print(json.dumps(out))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPU_CVT_REF")
    if not ref:
        sys.exit(f"usage: {sys.argv[0]} <reference checkout>  (or set GPU_CVT_REF)")
    main(ref)
