"""Generate the golden fixtures under tests/golden/ from the reference's own
Python code (Harper-Yan/GPU_CVT ``scripts/testfreeze.py`` and
``scripts/evaluate.py``).

Run once, in a container that has the reference checkout:

    python tests/golden/make_golden.py /path/to/reference

``testfreeze.py`` imports ``trimesh`` and ``open3d`` at module level
(testfreeze.py:8-9) although the functions used here never touch them, so
empty stand-in modules are registered before the import.  Everything else is
the reference code unmodified.  The inputs are seeded procedural meshes and
site sets (gpu_cvt_b200.meshgen).  The fixtures are small .npz files; the
tests read them without needing the reference.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from gpu_cvt_b200 import meshgen as mg  # noqa: E402


def _load(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _stub(name):
    if name not in sys.modules:
        sys.modules[name] = types.ModuleType(name)


def main(ref_root: str) -> None:
    _stub("trimesh")
    _stub("open3d")
    tf = _load(os.path.join(ref_root, "scripts", "testfreeze.py"), "ref_testfreeze")
    ev = _load(os.path.join(ref_root, "scripts", "evaluate.py"), "ref_evaluate")
    rng = np.random.default_rng(1234)

    # ---- tangent frames (testfreeze.py:136-144) --------------------------------
    n = rng.normal(size=(512, 3))
    n[:64, 2] = np.sign(n[:64, 2]) * 10.0  # |n_z| > 0.9 branch
    n = n.astype(np.float32)
    U, V = tf.tangent(n.astype(np.float64))
    np.savez_compressed(os.path.join(HERE, "frames.npz"), n=n, U=U, V=V)

    # ---- closest point on a triangle (testfreeze.py:199-232) --------------------
    T = rng.normal(size=(600, 4, 3)).astype(np.float32)
    # degenerate-ish and region-specific cases
    T[:50, 3] = T[:50, 0] + rng.normal(scale=1e-3, size=(50, 3)).astype(np.float32)
    cp = np.array([tf.closest_point_tri(t[0].astype(np.float64), t[1].astype(np.float64),
                                        t[2].astype(np.float64), t[3].astype(np.float64)) for t in T])
    np.savez_compressed(os.path.join(HERE, "closest_point.npz"), tris=T, cp=cp)

    # ---- clip + centroid (testfreeze.py:146-197) on icosphere sites -------------
    m = mg.icosphere(5)
    S = mg.sample_sites(m.V, m.F, 2000, seed=0)
    from scipy.spatial import cKDTree
    tree = cKDTree(S.astype(np.float64))
    _, idx = tree.query(S.astype(np.float64), k=21)
    nb = idx[:, 1:].astype(np.uint32)            # distance order (the GPU order)
    N = S / np.linalg.norm(S, axis=1, keepdims=True)   # sphere normals
    Uc, Vc = tf.tangent(N.astype(np.float64))
    R = 2.0
    sel = np.arange(0, 2000, 7)
    cent = np.zeros((sel.size, 3))
    npoly = np.zeros(sel.size, np.int32)
    S64 = S.astype(np.float64)
    for t, i in enumerate(sel):
        poly = tf.cell_poly2d(int(i), S64, Uc, Vc, nb[i].astype(np.int64), R)
        _, c2 = tf.poly_area_centroid_2d(poly)
        cent[t] = S64[i] + c2[0] * Uc[i] + c2[1] * Vc[i]
        npoly[t] = poly.shape[0]
    np.savez_compressed(os.path.join(HERE, "clip_centroid.npz"), S=S, knn=nb, U=Uc, V=Vc, R=R, sel=sel,
                        cent=cent, npoly=npoly)

    # ---- one-ring projection (testfreeze.py:234-251, 413-425) --------------------
    c3 = S64[:300] * 1.05 + rng.normal(scale=0.01, size=(300, 3))
    treeV = cKDTree(m.V.astype(np.float64))
    _, vnn = treeV.query(c3, k=5)
    vf = [[] for _ in range(m.nV)]
    for fi, (a, b, c) in enumerate(m.F):
        vf[int(a)].append(fi)
        vf[int(b)].append(fi)
        vf[int(c)].append(fi)
    proj = np.zeros_like(c3)
    for i in range(c3.shape[0]):
        faces = sorted({f for v in vnn[i] for f in vf[int(v)]})
        proj[i] = tf.update_to_mesh(c3[i], m.F[np.array(faces)].astype(np.int64), m.V.astype(np.float64))
    np.savez_compressed(os.path.join(HERE, "project.npz"), cent=c3.astype(np.float32), knnv=vnn.astype(np.int32),
                        proj=proj)

    # ---- Lloyd iterations, freezing off (testfreeze.py:376-446 run as in
    #      testfreeze2.py:172-195 with the streak gate disabled) -----------------
    from oracle import oracle as O  # area-weighted vertex normals, as on the GPU
    N0 = O.vertex_normals(m.V, m.F).astype(np.float64)
    P0 = m.V.astype(np.float64)
    F0 = m.F.astype(np.int64)
    treeP0 = cKDTree(P0)
    ntier = len(tf.TIERS)
    K = 20
    S_it = S.astype(np.float64)
    treeS0 = cKDTree(S_it)
    _, idx0 = treeS0.query(S_it, k=K + 1)
    idx0 = np.sort(idx0[:, 1:], axis=1)
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
    traj = []
    for it in range(5):
        S_it, fs, _ = tf.lloyd_iter_sites_only(S_it, P0, F0, N0, vf, treeP0, fs, k_neigh=K, k_proj=5)
        traj.append(S_it.copy())
    np.savez_compressed(os.path.join(HERE, "lloyd_py_fp64.npz"), S0=S, N0=N0.astype(np.float32),
                        traj=np.stack(traj), K=K)

    # ---- evaluation (evaluate.py:47-290) ------------------------------------------
    mc = mg.icosphere(2)
    Vc = (mc.V * np.float32(1.01)).astype(np.float32)
    Vc[::7] *= np.float32(0.98)
    Vr, Fr = mg.icosphere(3).V, mg.icosphere(3).F
    dH = ev.hausdorff_bvh(Vc.astype(np.float64), mc.F.astype(np.int64), Vr.astype(np.float64),
                          Fr.astype(np.int64), leaf_size=8)
    row = ev.evaluate_mesh("cand", Vc.astype(np.float64), mc.F.astype(np.int64), Vr.astype(np.float64),
                           Fr.astype(np.int64), 8)
    P = rng.normal(size=(400, 3))
    tri = rng.normal(size=(400, 3, 3))
    d2 = np.array([ev._point_triangle_d2(P[i], tri[i, 0], tri[i, 1], tri[i, 2]) for i in range(400)])
    np.savez_compressed(os.path.join(HERE, "evaluate.npz"), Vc=Vc, Fc=mc.F, Vr=Vr, Fr=Fr, dH=dH,
                        quality=np.array([row[k] for k in ["Qmin", "Qavg", "theta_min", "theta_min_avg",
                                                            "theta_lt_30_pct", "theta_gt_90_pct"]]),
                        P=P.astype(np.float32), tri=tri.astype(np.float32), d2=d2)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPU_CVT_REF")
    if not ref:
        sys.exit(f"usage: {sys.argv[0]} <reference checkout>  (or set GPU_CVT_REF)")
    main(ref)
