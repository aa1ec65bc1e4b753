"""gpu_cvt command line: the reference driver's contract (main.cu:371-1123).

    python -m gpu_cvt_b200.cli <mesh.obj> [mode=1] [iters=100] [options]

mode 0: freezing off ("gpucvt"), 1: five-tier freezing ("freeze"),
2: six-tier freezing ("freeze_tiered").  Like the reference, the sites start
as the mesh vertices (main.cu:493) unless --sites N asks for N area-uniform
samples.  Outputs, under experiments/output/<gpucvt|freeze|freeze_tiered>/<mesh>/
(main.cu:621-638, 911-990):

* eval_iters.csv  -- every DUMP_STRIDE=10 iterations: quality, one-sided
                     Hausdorff, per-stage milliseconds, freeze counts
                     (the reference's 28 columns, evaluate.cuh:468-550)
* iter_%03d.obj, iter_%03d_sites.xyz, iter_%03d_frozen.txt -- the
                     dual-triangle mesh, the sites ("x y z" lines,
                     buildmesh.cuh:203-207) and the frozen mask at those
                     iterations
and one row appended to experiments/runs.csv (main.cu:342-368).  The stdout
lines follow main.cu's.

Per-stage times come from CUDA events between the fused kernel groups:
knn_sites_ms = grid build + site KNN (the site->vertex search is fused into
it, so knn_site_to_mesh_ms is 0), centroids_ms = the per-site kernel (frame,
clip, centroid, centroid->vertex KNN, projection, freeze test; uv, centroid
KNN and projection columns are 0); freeze_ms is 0 as well, the freeze test
and the bookkeeping being part of the projection kernels counted there.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

EVAL_HEADER = ("mesh,mode,iter,Qmin,Qavg,theta_min,theta_min_avg,theta_lt_30_pct,theta_gt_90_pct,dH,"
               "iter_remesh_ms,total_remesh_ms,freeze_cell_num,n_vertices,freeze_pct,"
               "knn_sites_ms,knn_site_to_mesh_ms,uv_from_mesh_ms,centroids_ms,knn_centroid_to_mesh_ms,project_ms,"
               "freeze_ms,count_same,count_low_disp,count_both,count_newly_frozen,blocked_by_same,"
               "blocked_by_low_disp")
RUNS_HEADER = "meshname,mode,final_nv,final_nf,converge_rate,used_iterations,total_remeshing_time"
MODE_NAME = {0: "baseline", 1: "freezing_cvt", 2: "freezing_cvt_tiered"}
ROOT_DIR = {0: "gpucvt", 1: "freeze", 2: "freeze_tiered"}
DUMP_STRIDE = 10


def _g(x):
    """Shortest round-trip text of a float, like the reference's ostream <<."""
    x = float(x)
    if math.isnan(x):
        return "nan"
    return f"{x:.6g}"


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="gpu_cvt", description=__doc__.split("\n\n")[0])
    ap.add_argument("mesh")
    ap.add_argument("mode", nargs="?", type=int, default=1)
    ap.add_argument("iters", nargs="?", type=int, default=100)
    ap.add_argument("--k", type=int, default=32, help="neighbours per site (K_NEIGH, main.cu:398)")
    ap.add_argument("--sites", type=int, default=0, help="area-uniform sites instead of the vertices")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--profile", choices=["ref", "mixed", "fp64"], default="ref")
    ap.add_argument("--out-root", default=".", help="directory that holds experiments/")
    a = ap.parse_args(argv)
    if a.mode not in (0, 1, 2):
        print("mode must be 0, 1 or 2", file=sys.stderr)
        return 1

    import torch
    from . import engine as E
    from . import meshgen as mg

    print(f"mode {a.mode} ({MODE_NAME[a.mode]})")
    m = mg.load_obj(a.mesh)
    name = os.path.splitext(os.path.basename(a.mesh))[0]
    print(f"V {m.nV}")
    print(f"F {m.nF}")
    if m.nV == 0 or m.nF == 0:
        return 1
    mesh = E.Mesh(m.V, m.F)
    R = mesh.R
    freeze_disp = np.float32(np.float32(np.float32(0.01) * np.float32(R)) * np.float32(0.01)) * np.float32(R)
    print(f"freeze_disp {float(freeze_disp):.6g} (squared, linear=0.01*R R={R:.6g})")
    S0 = mg.sample_sites(m.V, m.F, a.sites, seed=a.seed) if a.sites > 0 else m.V.copy()
    n = S0.shape[0]
    cells = E.grid_cells(mesh, n, a.k)
    eng = E.Engine(E.params(k=a.k, mode=a.mode, profile=a.profile), 1, n, cells)
    seg = eng.add(mesh, S0)
    out_dir = os.path.join(a.out_root, "experiments", "output", ROOT_DIR[a.mode], name)
    os.makedirs(out_dir, exist_ok=True)
    eval_csv = os.path.join(out_dir, "eval_iters.csv")
    with open(eval_csv, "w") as fh:
        fh.write(EVAL_HEADER + "\n")
    total_ms = 0.0
    last_nf = 0
    frozen_ratio = 0.0
    used = 0
    for it in range(a.iters):
        print(f"\n=== iter {it} ===")
        ms = eng.profile(1)           # one iteration, CUDA events between kernel groups
        knn_ms = ms["grid"] + ms["knn"]
        cell_ms = ms["cell"]
        freeze_ms = ms["tail"]
        print(f"knn_sites_ms {knn_ms:.3f}")
        print("knn_site_to_mesh_ms 0.000")
        print(f"centroids_ms {cell_ms:.3f}")
        print(f"freeze_ms {freeze_ms:.3f}")
        iter_ms = knn_ms + cell_ms
        total_ms += iter_ms
        print(f"iter_remesh_ms {iter_ms:.3f} (total_remesh_ms {total_ms:.3f})")
        st = eng.stats(seg, it)
        print(f"same neighbors {st['same']}")
        print(f"low displacement {st['low']}")
        print(f"both {st['both']}")
        print(f"pass2 {st['newly_frozen']}")
        state = eng.state(seg)
        nfrozen = int(state["frozen"].sum())
        frozen_ratio = nfrozen / n
        print(f"total frozen so far {nfrozen} / {n} ({100.0 * frozen_ratio:.2f}%)")
        if it % DUMP_STRIDE == 0:
            F, ev = eng.faces(seg)
            S = eng.sites(seg)
            last_nf = F.shape[0]
            path = os.path.join(out_dir, f"iter_{it:03d}.obj")
            mg.save_obj(path, S, F)
            with open(os.path.join(out_dir, f"iter_{it:03d}_sites.xyz"), "w") as fh:   # write_pts_cpu
                fh.write("".join(f"{_g(x)} {_g(y)} {_g(z)}\n" for x, y, z in S))
            with open(os.path.join(out_dir, f"iter_{it:03d}_frozen.txt"), "w") as fh:
                fh.write("\n".join(str(int(x)) for x in state["frozen"]) + "\n")
            print(f"iter {it} V {n} faces {last_nf} wrote {path}")
            bs = max(st["low"] - st["both"], 0)
            bl = max(st["same"] - st["both"], 0)
            row = [name, ROOT_DIR[a.mode], it, _g(ev["Qmin"]), _g(ev["Qavg"]), _g(ev["theta_min"]),
                   _g(ev["theta_min_avg"]), _g(ev["theta_lt_30_pct"]), _g(ev["theta_gt_90_pct"]), _g(ev["dH"]),
                   _g(iter_ms), _g(total_ms), nfrozen, n, _g(100.0 * nfrozen / n), _g(knn_ms), 0, 0, _g(cell_ms), 0,
                   0, _g(freeze_ms), st["same"], st["low"], st["both"], st["newly_frozen"], bs, bl]
            with open(eval_csv, "a") as fh:
                fh.write(",".join(str(x) for x in row) + "\n")
        used = it + 1
    print(f"\nTotal remeshing time (mesh rebuilding excluded): {total_ms:.3f} ms")
    runs = os.path.join(a.out_root, "experiments", "runs.csv")
    new = not os.path.exists(runs)
    with open(runs, "a") as fh:
        if new:
            fh.write(RUNS_HEADER + "\n")
        fh.write(f"{name},{ROOT_DIR[a.mode]},{n},{last_nf},{_g(frozen_ratio)},{used},{_g(total_ms)}\n")
    eng.close()
    mesh.close()
    torch.cuda.synchronize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
