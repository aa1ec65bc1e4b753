"""The reference's stage functions, one by one, over torch CUDA tensors.

Same names and argument meaning as the reference's header-only CUDA stages
(Harper-Yan/GPU_CVT), so a driver written against them reads the same:

=============================================  ======================================
reference (file:line)                          here
=============================================  ======================================
run_knn_bitonic_hubs (site_knn.cuh:20)         run_knn_bitonic_hubs
run_knn_bitonic_query_to_mesh (site_knn.cuh:57) run_knn_bitonic_query_to_mesh
knn_drop_self_kernel (site_knn.cuh:79)         knn_drop_self
zero/accumulate/normalize_normals              vertex_normals
  (site_normals.cuh:14-41)
uv_from_nearest_vertex_normal (site_normals.cuh:69) uv_from_nearest_vertex_normal
centroids_tangent_voronoi (2dClip.cuh:82)      centroids_tangent_voronoi
knn_vertices_bruteforce_k (near_project.cuh:55) knn_vertices_bruteforce_k
restore_prev_knn_* (main.cu:302,               restore_prev_knn_for_frozen
  near_project.cuh:96)
project_centroids_to_mesh (near_project.cuh:150) project_centroids_to_mesh
freeze_test_kernel_streak(_tiered) +           freeze_test_streak
  freeze_apply_cand_kernel (freezetest.cuh)
count_frozen_kernel (freezetest.cuh:50)        count_frozen
tier1/tier2 host code (main.cu:18-150)         tier_ids
hausdorff_cand_to_ref_gpu (evaluate.cuh:360)   hausdorff_cand_to_ref
=============================================  ======================================

Every function runs the libgpucvt kernel on the current torch CUDA stream;
tensors must be contiguous CUDA tensors of the stated dtypes.  The timed
KNN wrappers return elapsed milliseconds like the reference's.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import call


def _p(t):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _timed(fn):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    fn()
    e1.record()
    e1.synchronize()
    return float(e0.elapsed_time(e1))


def run_knn_bitonic_hubs(N, K, frozen, pts, knn, dist) -> float:
    """Exact K nearest sites (self included) of every site; frozen rows are
    left untouched.  pts float32 (N,3); knn uint32/int32 (N,K); dist float32
    (N,K) or None.  Returns elapsed ms."""
    return _timed(lambda: call("cvt_knn_sites", _p(pts), int(N), int(K), _p(frozen), _p(knn), _p(dist), _stream()))


def run_knn_bitonic_query_to_mesh(nCand, candidates, query, nQ, K, frozen, knn, dist, name_for_timing="") -> float:
    """K nearest of the candidate points (mesh vertices) for each query point."""
    return _timed(lambda: call("cvt_knn_query_to_points", _p(candidates), int(nCand), _p(query), int(nQ), int(K),
                               _p(frozen), _p(knn), _p(dist), _stream()))


def knn_drop_self(knn_in, knn_out, n, kin, kout) -> None:
    call("cvt_knn_drop_self", _p(knn_in), int(n), int(kin), int(kout), _p(knn_out), _stream())


def restore_prev_knn_for_frozen(frozen, prev, cur, n, k) -> None:
    call("cvt_restore_frozen_rows", _p(frozen), _p(prev), _p(cur), int(n), int(k), _stream())


def vertex_normals(V, F, vf_off, vf_faces, N) -> None:
    call("cvt_vertex_normals", _p(V), V.shape[0], _p(F), F.shape[0], _p(vf_off), _p(vf_faces), _p(N), _stream())


def uv_from_nearest_vertex_normal(N0, knnV, U, V, kproj=5) -> None:
    call("cvt_frames", _p(N0), _p(knnV), int(kproj), knnV.shape[0], _p(U), _p(V), _stream())


def centroids_tangent_voronoi(S, U, V, knn, nV, K, R, cent, profile=0, nverts=None) -> None:
    call("cvt_clip_centroids", _p(S), _p(U), _p(V), _p(knn), int(nV), int(K), float(R), int(profile), _p(cent),
         _p(nverts), _stream())


def knn_vertices_bruteforce_k(Vpos, nV, Q, nQ, frozen, out_idx, kproj=5, exclude_self=False) -> None:
    call("cvt_knn_vertices", _p(Vpos), int(nV), _p(Q), int(nQ), int(kproj), int(bool(exclude_self)), _p(frozen),
         _p(out_idx), _stream())


def project_centroids_to_mesh(cent3d, Vpos, F, vf_off, vf_faces, knnV, nV, nF, nQ, Sold, out_Snew, kproj=5,
                              profile=0) -> None:
    call("cvt_project", _p(cent3d), _p(Vpos), _p(F), _p(vf_off), _p(vf_faces), _p(knnV), int(kproj), int(nV),
         int(nF), int(nQ), int(profile), _p(Sold), _p(out_Snew), _stream())


def freeze_test_streak(S, Snew, knn, prev_knn, K, has_prev, thr2_tier, need_tier, streak, cand, frozen, counts,
                       tier=None) -> None:
    """Streak freeze test + apply.  thr2_tier / need_tier: 6 host values each
    (a single value is broadcast, the untiered reference kernel)."""
    thr = (C.c_float * 6)(*([float(x) for x in thr2_tier] if hasattr(thr2_tier, "__len__") else [float(thr2_tier)] * 6))
    need = (C.c_int * 6)(*([int(x) for x in need_tier] if hasattr(need_tier, "__len__") else [int(need_tier)] * 6))
    call("cvt_freeze", _p(S), _p(Snew), _p(knn), _p(prev_knn), S.shape[0], int(K), int(has_prev), _p(tier), thr, need,
         _p(streak), _p(cand), _p(frozen), _p(counts), _stream())


def count_frozen(frozen, n, out_sum) -> None:
    call("cvt_count_frozen", _p(frozen), int(n), _p(out_sum), _stream())


def tier_ids(mode, site_normals, knn, tier) -> None:
    call("cvt_tiers", int(mode), knn.shape[0], knn.shape[1], _p(site_normals), _p(knn), _p(tier), _stream())


def hausdorff_cand_to_ref(ref_mesh, Vcand, Fcand) -> float:
    """One-sided Hausdorff (candidate probes -> reference surface)."""
    return ref_mesh.hausdorff_from(Vcand, Fcand, _stream())


def extract_faces(S, U, V, knn, R2, max_faces=None):
    """Dual triangles of the sites (cell_poly2d_kernel + emit_faces_from_labels_kernel
    + sort/unique/degenerate filter, main.cu:928-974).  Returns an int32
    CUDA tensor (nF, 3)."""
    n, K = knn.shape
    cap = int(max_faces or 4 * n + 64)
    out = torch.empty((cap, 3), dtype=torch.int32, device=S.device)
    nf = C.c_int()
    try:
        call("cvt_extract_faces", _p(S), _p(U), _p(V), _p(knn), int(n), int(K), float(R2), _p(out), cap,
             C.byref(nf), _stream())
    except _lib.CvtError as e:
        if e.status != 5:
            raise
        return extract_faces(S, U, V, knn, R2, max_faces=nf.value)
    return out[:nf.value]


def quality(V, F) -> dict:
    """Triangle quality metrics (eval_quality_angles_cpu, evaluate.cuh:388)."""
    out = (C.c_float * 6)()
    call("cvt_quality", _p(V), _p(F), F.shape[0], out, _stream())
    keys = ["Qmin", "Qavg", "theta_min", "theta_min_avg", "theta_lt_30_pct", "theta_gt_90_pct"]
    return dict(zip(keys, [float(x) for x in out]))


def launch_count() -> int:
    return _lib.launch_count()
