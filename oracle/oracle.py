"""numpy front end of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke``
and by the CPU-baseline leg of ``bench.py`` -- never by the product package.

Each function restates one stage of the reference (Harper-Yan/GPU_CVT); the
C++ source ``oracle/cvt_oracle.cpp`` cites the file:line of every stage.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

P_REF, P_MIXED, P_FP64 = 0, 1, 2
PROFILES = {"ref": P_REF, "mixed": P_MIXED, "fp64": P_FP64}


def build(force: bool = False) -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "cvt_oracle.cpp")
    if force or not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        _declare(_LIB)
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _declare(L):
    vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
    sigs = {
        "oracle_version": ([], i32),
        "oracle_set_threads": ([i32], None),
        "oracle_max_threads": ([], i32),
        "oracle_build_vf": ([i32, i32, vp, vp, vp], None),
        "oracle_vertex_normals": ([vp, i32, vp, i32, vp], None),
        "oracle_knn_points_bf": ([vp, i32, i32, vp, vp, vp], None),
        "oracle_knn_points_grid": ([vp, i32, i32, vp, vp, vp], None),
        "oracle_drop_self": ([vp, i32, i32, i32, vp, vp], None),
        "oracle_knn_vertices_bf": ([vp, i32, vp, i32, i32, i32, vp, vp], None),
        "oracle_frames": ([vp, vp, i32, vp, vp], None),
        "oracle_clip_centroids": ([vp, i32, vp, vp, vp, i32, f32, i32, vp, vp], None),
        "oracle_closest_point_tri": ([vp, vp, vp, vp, vp], None),
        "oracle_project": ([vp, i32, vp, i32, vp, i32, vp, vp, vp, i32, i32, vp, vp], None),
        "oracle_freeze": ([vp, vp, i32, vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, vp], None),
        "oracle_tiers": ([i32, i32, i32, vp, vp, vp, vp, vp], None),
        "oracle_lloyd_run": ([vp, i32, vp, i32, vp, vp, i32, i32, i32, i32, i32, i32, i32, f32,
                              vp, vp, vp, vp, vp, vp, vp, i32, i32], None),
        "oracle_lloyd_run_f64": ([vp, i32, vp, i32, vp, vp, i32, i32, i32, i32, i32, i32, f32,
                                  vp, vp, vp, vp, vp, vp, i32, i32], None),
        "oracle_pca_frames": ([vp, i32, vp, i32, vp, vp, vp, vp], None),
        "oracle_project_bvh": ([vp, i32, vp, i32, vp, i32, i32, vp, vp], None),
        "oracle_point_tri_d2": ([vp, vp, vp, vp], f32),
        "oracle_bvh_node_count": ([vp, vp, i32, i32], i32),
        "oracle_bvh_build": ([vp, vp, i32, i32, vp, vp], None),
        "oracle_hausdorff_one_sided": ([vp, i32, vp, i32, vp, i32, vp, i32, i32], f32),
        "oracle_quality": ([vp, vp, i32, vp], None),
        "oracle_extract_faces": ([vp, i32, vp, vp, vp, i32, f32, f32, f32, f32, vp], i32),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint8)


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def build_vf(nV, F):
    F = _i32(F)
    off = np.zeros(nV + 1, np.int32)
    fcs = np.zeros(3 * F.shape[0], np.int32)
    lib().oracle_build_vf(nV, F.shape[0], _p(F), _p(off), _p(fcs))
    return off, fcs


def vertex_normals(V, F):
    V, F = _f32(V), _i32(F)
    N = np.zeros_like(V)
    lib().oracle_vertex_normals(_p(V), V.shape[0], _p(F), F.shape[0], _p(N))
    return N


def knn_points(P, kk, frozen=None, method="grid", knn=None, dist=None):
    """Exact kk nearest points (self included), (d2, index) order."""
    P = _f32(P)
    n = P.shape[0]
    knn = np.full((n, kk), 0, np.uint32) if knn is None else knn
    dist = np.full((n, kk), np.inf, np.float32) if dist is None else dist
    fn = lib().oracle_knn_points_grid if method == "grid" else lib().oracle_knn_points_bf
    fn(_p(P), n, kk, _p(_u8(frozen)), _p(knn), _p(dist))
    return knn, dist


def drop_self(raw, kout, frozen=None, out=None):
    raw = _u32(raw)
    n, kin = raw.shape
    out = np.zeros((n, kout), np.uint32) if out is None else out
    lib().oracle_drop_self(_p(raw), n, kin, kout, _p(_u8(frozen)), _p(out))
    return out


def knn_vertices(V, Q, k, exclude_self=False, frozen=None, out=None):
    V, Q = _f32(V), _f32(Q)
    out = np.full((Q.shape[0], k), -1, np.int32) if out is None else out
    lib().oracle_knn_vertices_bf(_p(V), V.shape[0], _p(Q), Q.shape[0], k, int(exclude_self),
                                 _p(_u8(frozen)), _p(out))
    return out


def frames(N, nearest):
    N = _f32(N)
    nearest = _i32(nearest)
    n = nearest.shape[0]
    U = np.zeros((n, 3), np.float32)
    Vv = np.zeros((n, 3), np.float32)
    lib().oracle_frames(_p(N), _p(nearest), n, _p(U), _p(Vv))
    return U, Vv


def clip_centroids(S, U, Vv, knn, R, profile=P_REF, return_nverts=False):
    S, U, Vv, knn = _f32(S), _f32(U), _f32(Vv), _u32(knn)
    n, K = knn.shape
    cent = np.zeros((n, 3), np.float32)
    nv = np.zeros(n, np.int32)
    lib().oracle_clip_centroids(_p(S), n, _p(U), _p(Vv), _p(knn), K, float(R), profile, _p(cent), _p(nv))
    return (cent, nv) if return_nverts else cent


def closest_point_tri(P, A, B, Cc):
    out = np.zeros(3, np.float32)
    lib().oracle_closest_point_tri(_p(_f32(P)), _p(_f32(A)), _p(_f32(B)), _p(_f32(Cc)), _p(out))
    return out


def project(cent, V, F, knnv, profile=P_REF, Sold=None):
    cent, V, F, knnv = _f32(cent), _f32(V), _i32(F), _i32(knnv)
    off, fcs = build_vf(V.shape[0], F)
    n, kp = knnv.shape
    Sold = cent if Sold is None else _f32(Sold)
    Snew = np.zeros((n, 3), np.float32)
    lib().oracle_project(_p(cent), n, _p(V), V.shape[0], _p(F), F.shape[0], _p(off), _p(fcs), _p(knnv), kp,
                         profile, _p(Sold), _p(Snew))
    return Snew


def tiers(mode, site_normals, knn):
    site_normals, knn = _f32(site_normals), _u32(knn)
    n, K = knn.shape
    tier = np.zeros(n, np.uint8)
    nv = np.zeros(n, np.float64)
    L = np.zeros(n, np.float64)
    lib().oracle_tiers(mode, n, K, _p(site_normals), _p(knn), _p(tier), _p(nv), _p(L))
    return tier, nv, L


def freeze(S, Snew, knn, prev, has_prev, tier, thr2_tier, need_tier, streak, frozen):
    """One freeze-test + apply pass; streak/frozen updated in place."""
    S, Snew, knn, prev = _f32(S), _f32(Snew), _u32(knn), _u32(prev)
    n, K = knn.shape
    cand = np.zeros(n, np.uint8)
    counts = np.zeros(4, np.int32)
    lib().oracle_freeze(_p(S), _p(Snew), n, _p(knn), _p(prev), K, int(has_prev), _p(_u8(tier)),
                        _p(_f32(thr2_tier)), _p(_i32(need_tier)), _p(streak), _p(cand), _p(frozen), _p(counts))
    return cand, counts


PROJ = {"onering": 0, "bvh": 1}
FRAME = {"vertex": 0, "pca": 1}


def lloyd_run(V, F, S0, K, mode, iters, profile=P_REF, kproj=5, ex_quirk=True, R=None, N=None, proj="onering",
              frame="vertex"):
    """Full remesh run; returns dict(S, counts, maxdisp, frozen, tier, knn, knnv, cent).
    proj "bvh" / frame "pca" select the engine's projection and frame options."""
    pm = PROJ[proj] if isinstance(proj, str) else int(proj)
    fm = FRAME[frame] if isinstance(frame, str) else int(frame)
    V, F = _f32(V), _i32(F)
    nV, nF = V.shape[0], F.shape[0]
    if N is None:
        N = vertex_normals(V, F)
    if R is None:
        ext = V.max(0) - V.min(0)
        R = float(np.float32(max(ext[0], ext[1], ext[2])))
    n = S0.shape[0]
    counts = np.zeros((max(iters, 1), 4), np.int32)
    maxdisp = np.zeros(max(iters, 1), np.float64)
    frozen = np.zeros(n, np.uint8)
    tier = np.zeros(n, np.uint8)
    knn = np.zeros((n, K), np.uint32)
    knnv = np.zeros((n, kproj), np.int32)
    if profile == P_FP64:
        S = np.ascontiguousarray(S0, dtype=np.float64).copy()
        lib().oracle_lloyd_run_f64(_p(V), nV, _p(F), nF, _p(_f32(N)), _p(S), n, K, mode, iters, kproj,
                                   int(ex_quirk), float(R), _p(counts), _p(maxdisp), _p(frozen), _p(tier),
                                   _p(knn), _p(knnv), pm, fm)
        cent = None
    else:
        S = _f32(S0).copy()
        cent = np.zeros((n, 3), np.float32)
        lib().oracle_lloyd_run(_p(V), nV, _p(F), nF, _p(_f32(N)), _p(S), n, K, mode, profile, iters, kproj,
                               int(ex_quirk), float(R), _p(counts), _p(maxdisp), _p(frozen), _p(tier),
                               _p(knn), _p(knnv), _p(cent), pm, fm)
    return dict(S=S, counts=counts[:iters], maxdisp=maxdisp[:iters], frozen=frozen, tier=tier, knn=knn,
                knnv=knnv, cent=cent)


def pca_frames(S, knn, N, nearest):
    """Frames from the PCA normal of each site's neighbours (cvt_frames_pca)."""
    S, knn, N, nearest = _f32(S), _u32(knn), _f32(N), _i32(nearest)
    n, K = knn.shape
    U = np.zeros((n, 3), np.float32)
    Vv = np.zeros((n, 3), np.float32)
    lib().oracle_pca_frames(_p(S), n, _p(knn), K, _p(N), _p(nearest), _p(U), _p(Vv))
    return U, Vv


def project_bvh(cent, V, F, profile=P_REF, Sold=None):
    """Closest point on the mesh through its BVH (cvt_project_bvh)."""
    cent, V, F = _f32(cent), _f32(V), _i32(F)
    Snew = np.zeros_like(cent)
    lib().oracle_project_bvh(_p(cent), cent.shape[0], _p(V), V.shape[0], _p(F), F.shape[0], int(profile),
                             _p(None if Sold is None else _f32(Sold)), _p(Snew))
    return Snew


def point_tri_d2(P, A, B, Cc) -> float:
    return float(lib().oracle_point_tri_d2(_p(_f32(P)), _p(_f32(A)), _p(_f32(B)), _p(_f32(Cc))))


def bvh_build(V, F, leaf=8):
    """Reference BVH (median split, stable sort, leaf 8).  Returns
    (nodes structured array, tri index array)."""
    V, F = _f32(V), _i32(F)
    nn = lib().oracle_bvh_node_count(_p(V), _p(F), F.shape[0], leaf)
    dt = np.dtype([("bmin", np.float32, 3), ("bmax", np.float32, 3), ("left", np.int32),
                   ("right", np.int32), ("triStart", np.int32), ("triCount", np.int32)])
    nodes = np.zeros(nn, dt)
    tri = np.zeros(F.shape[0], np.int32)
    lib().oracle_bvh_build(_p(V), _p(F), F.shape[0], leaf, _p(nodes), _p(tri))
    return nodes, tri


def hausdorff_one_sided(V1, F1, V2, F2, use_bvh=True) -> float:
    V1, F1, V2, F2 = _f32(V1), _i32(F1), _f32(V2), _i32(F2)
    return float(lib().oracle_hausdorff_one_sided(_p(V1), V1.shape[0], _p(F1), F1.shape[0], _p(V2),
                                                  V2.shape[0], _p(F2), F2.shape[0], int(use_bvh)))


def hausdorff_symmetric(V1, F1, V2, F2) -> float:
    return max(hausdorff_one_sided(V1, F1, V2, F2), hausdorff_one_sided(V2, F2, V1, F1))


def quality(V, F):
    out = np.zeros(6, np.float32)
    V, F = _f32(V), _i32(F)
    lib().oracle_quality(_p(V), _p(F), F.shape[0], _p(out))
    keys = ["Qmin", "Qavg", "theta_min", "theta_min_avg", "theta_lt_30_pct", "theta_gt_90_pct"]
    return dict(zip(keys, [float(x) for x in out]))


def extract_faces(S, U, Vv, knn, R2, eps_clip=1e-8, tol_active=1e-7, degenerate_eps=1e-6):
    S, U, Vv, knn = _f32(S), _f32(U), _f32(Vv), _u32(knn)
    n, K = knn.shape
    Fo = np.zeros((n * 256, 3), np.int32)
    nf = lib().oracle_extract_faces(_p(S), n, _p(U), _p(Vv), _p(knn), K, float(R2), float(eps_clip),
                                    float(tol_active), float(degenerate_eps), _p(Fo))
    return Fo[:nf].copy()
