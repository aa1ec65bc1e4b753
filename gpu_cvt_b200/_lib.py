"""ctypes binding of libgpucvt.so (include/gpu_cvt.h).

The library is the only compute path: if it is missing or fails to load, every
call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpucvt.so")

vp, i32, f32, u64 = C.c_void_p, C.c_int, C.c_float, C.c_ulonglong


class CvtError(RuntimeError):
    """A libgpucvt call returned a non-zero cvt_status_t."""

    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed: status {status} ({msg})")
        self.status = status


class MeshInfo(C.Structure):
    _fields_ = [("nV", i32), ("nF", i32), ("R", f32), ("area", f32), ("bbox_lo", f32 * 3),
                ("bbox_hi", f32 * 3), ("diag", f32), ("device_bytes", C.c_size_t)]


class Params(C.Structure):
    _fields_ = [("k", i32), ("mode", i32), ("profile", i32), ("kproj", i32), ("ex_quirk", i32),
                ("cell_factor", f32), ("use_graph", i32), ("knn_block", i32), ("clip_block", i32),
                ("proj_block", i32), ("proj_mode", i32), ("frame_mode", i32), ("knn_reuse", i32)]


class EvalOut(C.Structure):
    _fields_ = [("dH", f32), ("Qmin", f32), ("Qavg", f32), ("theta_min", f32), ("theta_min_avg", f32),
                ("theta_lt_30_pct", f32), ("theta_gt_90_pct", f32), ("n_faces", i32), ("diag", f32)]


class IterStats(C.Structure):
    _fields_ = [("same", i32), ("low", i32), ("both", i32), ("newly_frozen", i32), ("max_motion", f32),
                ("iter", i32), ("knn_reused", i32), ("knn_searched", i32)]


# name -> argtypes (all return cvt_status_t unless listed in _RESTYPES)
_SIGS = {
    "cvt_status_string": [i32],
    "cvt_last_error": [],
    "cvt_version": [],
    "cvt_launch_count": [],
    "cvt_knn_sites": [vp, i32, i32, vp, vp, vp, vp],
    "cvt_knn_sites_noalloc": [vp, i32, i32, vp, vp, vp, vp],
    "cvt_knn_query_to_points": [vp, i32, vp, i32, i32, vp, vp, vp, vp],
    "cvt_knn_vertices": [vp, i32, vp, i32, i32, i32, vp, vp, vp],
    "cvt_knn_drop_self": [vp, i32, i32, i32, vp, vp],
    "cvt_restore_frozen_rows": [vp, vp, vp, i32, i32, vp],
    "cvt_vertex_normals": [vp, i32, vp, i32, vp, vp, vp, vp],
    "cvt_frames": [vp, vp, i32, i32, vp, vp, vp],
    "cvt_frames_pca": [vp, i32, vp, i32, vp, vp, i32, vp, vp, vp],
    "cvt_project_bvh": [vp, vp, i32, i32, vp, vp, vp],
    "cvt_clip_centroids": [vp, vp, vp, vp, i32, i32, f32, i32, vp, vp, vp],
    "cvt_project": [vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, vp, vp, vp],
    "cvt_freeze": [vp, vp, vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp],
    "cvt_count_frozen": [vp, i32, vp, vp],
    "cvt_tiers": [i32, i32, i32, vp, vp, vp, vp],
    "cvt_hausdorff_to_mesh": [vp, vp, i32, vp, i32, vp, vp],
    "cvt_hausdorff_meshes": [vp, vp, vp, vp, vp, vp],
    "cvt_mesh_get_bvh": [vp, vp, i32, vp, i32, vp],
    "cvt_release_cached_memory": [],
    "cvt_autotune": [vp, vp, i32, i32, vp, vp],
    "cvt_segment_cells": [vp, i32, vp, vp],
    "cvt_mesh_create": [vp, i32, vp, i32, vp],
    "cvt_set_vertex_cell_factor": [f32],
    "cvt_mesh_info": [vp, vp],
    "cvt_mesh_device_arrays": [vp, vp, vp, vp, vp, vp],
    "cvt_mesh_destroy": [vp],
    "cvt_params_default": [vp],
    "cvt_engine_create": [vp, i32, i32, i32, vp],
    "cvt_engine_destroy": [vp],
    "cvt_engine_add_segment": [vp, vp, vp, i32, i32, vp, vp],
    "cvt_engine_remove_segment": [vp, i32],
    "cvt_engine_run": [vp, i32, vp],
    "cvt_engine_get_sites": [vp, i32, vp, i32, vp],
    "cvt_engine_get_sites_f64": [vp, i32, vp, vp],
    "cvt_engine_get_state": [vp, i32, vp, vp, vp, vp, vp],
    "cvt_engine_get_stats": [vp, i32, i32, vp, vp],
    "cvt_engine_segment_iters": [vp, i32, vp],
    "cvt_engine_last_launches": [vp, vp],
    "cvt_engine_profile": [vp, i32, vp, vp],
    "cvt_engine_set_stop": [vp, i32, f32, i32],
    "cvt_engine_poll": [vp, vp, vp, i32, vp],
    "cvt_mesh_sample_sites": [vp, i32, u64, vp, vp],
    "cvt_engine_evaluate": [vp, i32, vp, vp],
    "cvt_engine_faces": [vp, i32, vp, i32, vp, vp, vp],
    "cvt_extract_faces": [vp, vp, vp, vp, i32, i32, f32, vp, i32, vp, vp],
    "cvt_quality": [vp, vp, i32, vp, vp],
    "cvt_remesh": [vp, i32, vp, i32, vp, i32, vp, i32, vp, vp],
    "cvt_remesh_batch": [i32, vp, vp, vp, vp, vp, vp, vp, i32, vp],
}
_RESTYPES = {"cvt_status_string": C.c_char_p, "cvt_last_error": C.c_char_p, "cvt_version": i32,
             "cvt_launch_count": u64, "cvt_set_vertex_cell_factor": None, "cvt_params_default": None}

_lib = None


def exported_symbols():
    return list(_SIGS)


def load(path: str | None = None):
    """Load (building first if the library is absent) and declare the ABI."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if path is None and not os.path.exists(p) and os.path.isdir(os.path.join(HERE, "csrc")):
        from . import build as _b
        _b.build()
    if not os.path.exists(p):
        raise OSError(f"libgpucvt.so not found at {p}; run `python -m gpu_cvt_b200.build`")
    L = C.CDLL(p)
    for name, args in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, i32)
    if path is None:
        _lib = L
    return L


def call(name: str, *args):
    L = load()
    st = getattr(L, name)(*args)
    if st != 0:
        msg = L.cvt_last_error()
        raise CvtError(name, st, msg.decode() if msg else "")
    return st


def last_error() -> str:
    m = load().cvt_last_error()
    return m.decode() if m else ""


def launch_count() -> int:
    return int(load().cvt_launch_count())
