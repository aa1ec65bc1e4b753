"""Resident meshes and the multi-segment Lloyd engine (host side, ctypes).

``Mesh``     -- a compacted, preprocessed mesh resident in HBM (vertex
               normals, vertex->face CSR, vertex grid, BVH); mirrors the
               set-up of main.cu:421-542.
``Engine``   -- up to ``max_segments`` (mesh, site set) segments iterated
               together: each Lloyd iteration of main.cu:669-881 is one pass
               of fused kernels over every active segment, replayed from a
               CUDA graph.
``remesh``   -- one call with host arrays (upload, iterate, download).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import EvalOut, IterStats, MeshInfo, Params, call

PROFILE = {"ref": 0, "mixed": 1, "fp64": 2}


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


PROJ = {"onering": 0, "bvh": 1}
FRAME = {"vertex": 0, "pca": 1}


def params(k=24, mode=0, profile="ref", kproj=5, ex_quirk=True, cell_factor=1.1, use_graph=True,
           knn_block=0, clip_block=0, proj_block=0, proj="onering", frame="vertex", knn_reuse=True) -> Params:
    """Engine parameters.  proj: "onering" (the reference's projection onto
    the one-rings of the 5 nearest vertices) or "bvh" (exact closest point
    through the mesh's BVH); frame: "vertex" (the nearest vertex normal, as
    the reference) or "pca" (PCA normal of the site's neighbours);
    knn_reuse: take the K-lists from each site's kept candidate list while
    the sites' motion proves it exact (same lists, less work)."""
    p = Params()
    _lib.load().cvt_params_default(C.byref(p))
    p.k = int(k)
    p.mode = int(mode)
    p.profile = PROFILE[profile] if isinstance(profile, str) else int(profile)
    p.kproj = int(kproj)
    p.ex_quirk = int(bool(ex_quirk))
    p.cell_factor = float(cell_factor)
    p.use_graph = int(bool(use_graph))
    p.knn_block, p.clip_block, p.proj_block = int(knn_block), int(clip_block), int(proj_block)
    p.proj_mode = PROJ[proj] if isinstance(proj, str) else int(proj)
    p.frame_mode = FRAME[frame] if isinstance(frame, str) else int(frame)
    p.knn_reuse = int(bool(knn_reuse))
    return p


class Mesh:
    """A mesh uploaded and preprocessed once (host float32 V, int32 F in)."""

    def __init__(self, V, F):
        self.V_host = np.ascontiguousarray(V, dtype=np.float32)
        self.F_host = np.ascontiguousarray(F, dtype=np.int32)
        h = C.c_void_p()
        call("cvt_mesh_create", _ptr(self.V_host), self.V_host.shape[0], _ptr(self.F_host),
             self.F_host.shape[0], C.byref(h))
        self.handle = h
        inf = MeshInfo()
        call("cvt_mesh_info", h, C.byref(inf))
        self.nV, self.nF = inf.nV, inf.nF
        self.R = float(inf.R)
        self.area = float(inf.area)
        self.bbox_lo = np.array(inf.bbox_lo[:], np.float32)
        self.bbox_hi = np.array(inf.bbox_hi[:], np.float32)
        self.diag = float(inf.diag)
        self.device_bytes = int(inf.device_bytes)

    def device_arrays(self):
        """Raw device pointers (V, F, N, vf_off, vf_faces) of the compacted mesh."""
        ptrs = [C.c_void_p() for _ in range(5)]
        call("cvt_mesh_device_arrays", self.handle, *[C.byref(p) for p in ptrs])
        return [p.value for p in ptrs]

    def hausdorff_from(self, Vc, Fc, stream=None) -> float:
        """One-sided Hausdorff distance from the probe set of the candidate
        mesh (device pointers or torch CUDA tensors) to this mesh."""
        out = C.c_float()
        call("cvt_hausdorff_to_mesh", self.handle, _dptr(Vc), int(_rows(Vc)), _dptr(Fc), int(_rows(Fc)),
             C.byref(out), stream)
        return float(out.value)

    def bvh(self):
        """(nodes structured array, face ids) of the evaluation BVH."""
        n = C.c_int()
        call("cvt_mesh_get_bvh", self.handle, None, 0, None, 0, C.byref(n))
        dt = np.dtype([("bmin", np.float32, 3), ("bmax", np.float32, 3), ("left", np.int32),
                       ("right", np.int32), ("triStart", np.int32), ("triCount", np.int32)])
        nodes = np.zeros(n.value, dt)
        tri = np.zeros(self.nF, np.int32)
        call("cvt_mesh_get_bvh", self.handle, nodes.ctypes.data_as(C.c_void_p), n.value,
             tri.ctypes.data_as(C.c_void_p), self.nF, C.byref(n))
        return nodes, tri

    def hausdorff(self, other: "Mesh", stream=None) -> dict:
        """Symmetric Hausdorff distance to another mesh (scripts/evaluate.py
        hausdorff_bvh): {"dH": max of both sides, "self_to_other", "other_to_self"}."""
        out, ab, ba = C.c_float(), C.c_float(), C.c_float()
        call("cvt_hausdorff_meshes", self.handle, other.handle, C.byref(out), C.byref(ab), C.byref(ba), stream)
        return {"dH": float(out.value), "self_to_other": float(ab.value), "other_to_self": float(ba.value)}

    def sample_sites(self, out_tensor, seed: int, stream=None) -> None:
        """Fill a (n,3) float32 CUDA tensor with area-uniform points (device
        sampler, counter hash of (seed, i))."""
        call("cvt_mesh_sample_sites", self.handle, int(out_tensor.shape[0]), C.c_ulonglong(seed & (2**64 - 1)),
             C.c_void_p(out_tensor.data_ptr()), stream)

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().cvt_mesh_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _dptr(t):
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return C.c_void_p(int(t))


def _rows(t):
    return t.shape[0]


class Engine:
    """Capacity-based multi-segment engine."""

    def __init__(self, p: Params, max_segments: int, max_sites: int, max_cells: int):
        self.p = p
        self.K = p.k
        h = C.c_void_p()
        call("cvt_engine_create", C.byref(p), int(max_segments), int(max_sites), int(max_cells), C.byref(h))
        self.handle = h
        self.meshes = {}
        self.sizes = {}

    def add(self, mesh: Mesh, sites, stream=None) -> int:
        """Add a segment; ``sites`` is a host (n,3) array or a CUDA tensor."""
        sid = C.c_int()
        if hasattr(sites, "data_ptr"):
            n = int(sites.shape[0])
            call("cvt_engine_add_segment", self.handle, mesh.handle, C.c_void_p(sites.data_ptr()), n, 1,
                 C.byref(sid), stream)
        else:
            s = np.ascontiguousarray(sites, dtype=np.float32)
            n = int(s.shape[0])
            call("cvt_engine_add_segment", self.handle, mesh.handle, _ptr(s), n, 0, C.byref(sid), stream)
        self.meshes[sid.value] = mesh
        self.sizes[sid.value] = n
        return sid.value

    def remove(self, seg: int) -> None:
        call("cvt_engine_remove_segment", self.handle, int(seg))
        self.meshes.pop(seg, None)
        self.sizes.pop(seg, None)

    def run(self, iters: int, stream=None) -> None:
        call("cvt_engine_run", self.handle, int(iters), stream)

    def sites(self, seg: int) -> np.ndarray:
        out = np.zeros((self.sizes[seg], 3), np.float32)
        call("cvt_engine_get_sites", self.handle, int(seg), _ptr(out), 0, None)
        return out

    def sites_to_device(self, seg: int, out_tensor, stream=None) -> None:
        call("cvt_engine_get_sites", self.handle, int(seg), C.c_void_p(out_tensor.data_ptr()), 1, stream)

    def sites_f64(self, seg: int) -> np.ndarray:
        out = np.zeros((self.sizes[seg], 3), np.float64)
        call("cvt_engine_get_sites_f64", self.handle, int(seg), _ptr(out), None)
        return out

    def state(self, seg: int):
        n = self.sizes[seg]
        knn = np.zeros((n, self.K), np.uint32)
        knnv = np.zeros((n, 5), np.int32)
        frozen = np.zeros(n, np.uint8)
        tier = np.zeros(n, np.uint8)
        call("cvt_engine_get_state", self.handle, int(seg), _ptr(knn), _ptr(knnv), _ptr(frozen), _ptr(tier), None)
        return dict(knn=knn, knnv=knnv, frozen=frozen, tier=tier)

    def stats(self, seg: int, it: int) -> dict:
        s = IterStats()
        call("cvt_engine_get_stats", self.handle, int(seg), int(it), C.byref(s), None)
        return dict(same=s.same, low=s.low, both=s.both, newly_frozen=s.newly_frozen, max_motion=s.max_motion,
                    iter=s.iter, knn_reused=s.knn_reused, knn_searched=s.knn_searched)

    def iters(self, seg: int) -> int:
        v = C.c_int()
        call("cvt_engine_segment_iters", self.handle, int(seg), C.byref(v))
        return v.value

    def profile(self, iters: int, stream=None):
        """Per-kernel-group ms per iteration: grid, knn, clip, proj (with the
        deferred sites and the bookkeeping), tail (0), and cell = clip + proj."""
        ms = (C.c_float * 5)()
        call("cvt_engine_profile", self.handle, int(iters), ms, stream)
        d = dict(zip(("grid", "knn", "clip", "proj", "tail"), [float(x) for x in ms]))
        d["cell"] = d["clip"] + d["proj"]
        return d

    def evaluate(self, seg: int, stream=None) -> dict:
        """Dual-triangle mesh of the current sites: quality and one-sided
        Hausdorff distance to the segment's mesh (dH_rel = dH / bbox diag)."""
        o = EvalOut()
        call("cvt_engine_evaluate", self.handle, int(seg), C.byref(o), stream)
        d = {f: getattr(o, f) for f, _ in EvalOut._fields_}
        d["dH_rel"] = d["dH"] / d["diag"] if d["diag"] > 0 else float("nan")
        return d

    def set_stop(self, seg: int, max_motion: float, max_iters: int) -> None:
        """Device-side stop rule: stop once no site moves more than max_motion
        in an iteration (< 0: never), or after max_iters iterations (0: never)."""
        call("cvt_engine_set_stop", self.handle, int(seg), float(max_motion), int(max_iters))

    def poll(self, cap: int, stream=None):
        """(iters, state) per segment slot; state 0 free, 1 iterating, 2 stopped."""
        it = (C.c_int * cap)()
        st = (C.c_int * cap)()
        call("cvt_engine_poll", self.handle, it, st, int(cap), stream)
        return list(it), list(st)

    def faces(self, seg: int, stream=None):
        """(faces int32 (nF,3), evaluation dict) of the current sites."""
        n = self.sizes[seg]
        cap = 4 * n + 64
        while True:
            F = np.zeros((cap, 3), np.int32)
            nf = C.c_int()
            o = EvalOut()
            st = _lib.load().cvt_engine_faces(self.handle, int(seg), _ptr(F), cap, C.byref(nf), C.byref(o), stream)
            if st == 5 and nf.value > cap:
                cap = nf.value
                continue
            if st != 0:
                raise _lib.CvtError("cvt_engine_faces", st, _lib.last_error())
            d = {f: getattr(o, f) for f, _ in EvalOut._fields_}
            d["dH_rel"] = d["dH"] / d["diag"] if d["diag"] > 0 else float("nan")
            return F[:nf.value].copy(), d

    def last_launches(self) -> int:
        v = C.c_longlong()
        call("cvt_engine_last_launches", self.handle, C.byref(v))
        return int(v.value)

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().cvt_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def grid_cells(mesh: Mesh, n_sites: int, k: int, cell_factor: float = 1.1) -> int:
    """Cells a segment of ``n_sites`` sites on ``mesh`` reserves (mirrors the
    library's surface-grid sizing; used to size engine capacity)."""
    lo = mesh.bbox_lo.astype(np.float64)
    hi = mesh.bbox_hi.astype(np.float64)
    ext = hi - lo
    emax = max(float(ext.max()), 1e-20)
    dens = max(n_sites, 1) / max(mesh.area, 1e-30)
    h = cell_factor * np.sqrt((k + 1) / (np.pi * dens))
    h = max(h, emax / 2048.0)
    pad = 1e-4 * emax
    cap = 4 * n_sites + 64
    for _ in range(200):
        dims = [max(1, int(np.ceil((e + 2 * pad) / h))) for e in ext]
        prod = dims[0] * dims[1] * dims[2]
        if prod <= cap:
            break
        h *= 1.05
    return int(prod) + 1


def autotune(mesh: Mesh, sites, prm: Params, iters: int = 4):
    """Launch-shape autotuner (``cvt_autotune``): returns (tuned copy of the
    params, per-iteration ms of the chosen KNN, clip and projection shapes)."""
    S = np.ascontiguousarray(sites, np.float32)
    q = Params()
    C.memmove(C.byref(q), C.byref(prm), C.sizeof(Params))
    ms = (C.c_float * 3)()
    call("cvt_autotune", mesh.handle, _ptr(S), S.shape[0], int(iters), C.byref(q), ms)
    return q, {"knn": float(ms[0]), "clip": float(ms[1]), "proj": float(ms[2])}


def tiles(prm: Params) -> dict:
    return {"knn_block": prm.knn_block, "clip_block": prm.clip_block, "proj_block": prm.proj_block}


def remesh(V, F, sites, k=24, mode=0, profile="ref", iters=50, ex_quirk=True, cell_factor=1.1, with_counts=False,
           prm: Params | None = None):
    """One-call remesh through ``cvt_remesh`` (host arrays in and out); prm,
    when given, replaces the parameters built from the keywords."""
    V = np.ascontiguousarray(V, np.float32)
    F = np.ascontiguousarray(F, np.int32)
    S = np.ascontiguousarray(sites, np.float32)
    out = np.zeros_like(S)
    counts = np.zeros((max(iters, 1), 4), np.int32)
    p = prm if prm is not None else params(k=k, mode=mode, profile=profile, ex_quirk=ex_quirk, cell_factor=cell_factor)
    call("cvt_remesh", _ptr(V), V.shape[0], _ptr(F), F.shape[0], _ptr(S), S.shape[0], C.byref(p), int(iters),
         _ptr(out), _ptr(counts))
    return (out, counts[:iters]) if with_counts else out


def _host_ptr(a):
    """Address of a host array: a C-contiguous numpy array, or a CPU torch
    tensor (e.g. pinned with .pin_memory())."""
    if hasattr(a, "data_ptr"):
        if a.is_cuda or not a.is_contiguous():
            raise ValueError("remesh_batch takes contiguous host arrays")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("remesh_batch takes contiguous host arrays")
    return a.ctypes.data


def remesh_batch(Vs, Fs, sites, prm: Params, iters: int, outs=None):
    """Many meshes in one call through ``cvt_remesh_batch`` (host arrays in
    and out; float32 V/sites, int32 F, numpy or CPU torch tensors).  Returns
    the list of output site arrays (``outs`` when given, else new float32
    numpy arrays)."""
    n = len(Vs)
    if not (len(Fs) == n == len(sites)) or n == 0:
        raise ValueError("remesh_batch: one V, F and site array per mesh")
    if outs is None:
        outs = [np.zeros((int(S.shape[0]), 3), np.float32) for S in sites]
    P = C.c_void_p * n
    I = C.c_int * n
    vp_, fp_, sp_, op_ = P(*[_host_ptr(v) for v in Vs]), P(*[_host_ptr(f) for f in Fs]), \
        P(*[_host_ptr(s) for s in sites]), P(*[_host_ptr(o) for o in outs])
    nv, nf, ns = I(*[int(v.shape[0]) for v in Vs]), I(*[int(f.shape[0]) for f in Fs]), I(*[int(s.shape[0]) for s in sites])
    call("cvt_remesh_batch", n, vp_, nv, fp_, nf, sp_, ns, C.byref(prm), int(iters), op_)
    return outs
