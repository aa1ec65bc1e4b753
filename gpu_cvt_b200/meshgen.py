"""Seeded procedural meshes, the area-uniform site sampler and OBJ I/O.

The reference ships no meshes and initialises its sites as the mesh vertices
(main.cu:493, ``dS <- dV``).  The remesh workloads used here need site sets
that are independent of the vertex set, so this module provides:

* ``icosphere(level)``        -- unit icosphere (level 5: 10,242 V / 20,480 F)
* ``torus(...)``              -- (R, r) torus on an (nu x nv) grid with optional
                                 Gaussian noise along the analytic normals
* ``superellipsoid(...)``     -- |x|^p+|y|^p+|z|^p=1 via a cube-sphere lattice,
                                 optional jitter of a fraction of the triangles
* ``procedural_family(...)``  -- random spheres / tori / superquadrics
* ``sample_sites(V, F, n, seed)`` -- area-uniform points on the surface
* ``load_obj`` / ``save_obj`` -- OBJ parsing with the reference's rules
                                 (fan triangulation, negative indices,
                                 main.cu:162-228) and unused-vertex compaction
                                 (main.cu:230-257)

Everything is deterministic for a given seed (numpy ``default_rng``).
Positions are float32, faces int32, matching the reference's float3 / int3
device layout.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = [
    "Mesh", "icosphere", "torus", "superellipsoid", "superquadric",
    "procedural_family", "sample_sites", "load_obj", "save_obj",
    "compact_mesh", "mesh_area", "bbox_max_edge", "bbox_diag",
    "workload_mesh",
]


@dataclass
class Mesh:
    V: np.ndarray  # float32 [nV, 3]
    F: np.ndarray  # int32 [nF, 3]
    name: str = "mesh"

    @property
    def nV(self) -> int:
        return int(self.V.shape[0])

    @property
    def nF(self) -> int:
        return int(self.F.shape[0])


def _as_mesh(V, F, name) -> Mesh:
    return Mesh(np.ascontiguousarray(V, dtype=np.float32),
                np.ascontiguousarray(F, dtype=np.int32), name)


# --------------------------------------------------------------------------
# icosphere
# --------------------------------------------------------------------------
def icosphere(level: int = 5, radius: float = 1.0) -> Mesh:
    """Unit icosphere by repeated 4-to-1 midpoint subdivision.

    Level L has 10*4^L + 2 vertices and 20*4^L faces (level 5: 10,242 / 20,480).
    """
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
             (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    V = np.array(verts, dtype=np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]],
                 dtype=np.int64)
    for _ in range(level):
        nV = V.shape[0]
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0)
        e = np.sort(e, axis=1)
        key = e[:, 0] * (nV + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (nV + 1)
        b = uniq % (nV + 1)
        mid = V[a] + V[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        V = np.concatenate([V, mid], axis=0)
        nf = F.shape[0]
        m01 = nV + inv[:nf]
        m12 = nV + inv[nf:2 * nf]
        m20 = nV + inv[2 * nf:]
        F = np.concatenate([
            np.stack([F[:, 0], m01, m20], 1),
            np.stack([F[:, 1], m12, m01], 1),
            np.stack([F[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1)], axis=0)
    return _as_mesh(V * radius, F, f"icosphere{level}")


# --------------------------------------------------------------------------
# torus
# --------------------------------------------------------------------------
def torus(R: float = 1.0, r: float = 0.3, nu: int = 200, nv: int = 100,
          noise_sigma: float = 0.0, seed: int | None = None,
          center=(0.0, 0.0, 0.0)) -> Mesh:
    """(R, r) torus on an nu x nv grid (2*nu*nv triangles), optional
    N(0, noise_sigma) displacement of every vertex along its analytic normal."""
    i = np.arange(nu, dtype=np.float64)
    j = np.arange(nv, dtype=np.float64)
    u = 2.0 * np.pi * i / nu
    v = 2.0 * np.pi * j / nv
    uu, vv = np.meshgrid(u, v, indexing="ij")
    nx = np.cos(vv) * np.cos(uu)
    ny = np.cos(vv) * np.sin(uu)
    nz = np.sin(vv)
    x = (R + r * np.cos(vv)) * np.cos(uu)
    y = (R + r * np.cos(vv)) * np.sin(uu)
    z = r * np.sin(vv)
    P = np.stack([x, y, z], -1).reshape(-1, 3)
    N = np.stack([nx, ny, nz], -1).reshape(-1, 3)
    if noise_sigma > 0.0:
        rng = np.random.default_rng(seed)
        P = P + N * rng.normal(0.0, noise_sigma, size=(P.shape[0], 1))
    P = P + np.asarray(center, dtype=np.float64)
    ii, jj = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    a = ii * nv + jj
    b = ((ii + 1) % nu) * nv + jj
    c = ((ii + 1) % nu) * nv + (jj + 1) % nv
    d = ii * nv + (jj + 1) % nv
    F = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3),
                        np.stack([a, c, d], -1).reshape(-1, 3)], axis=0)
    return _as_mesh(P, F, f"torus{nu}x{nv}")


# --------------------------------------------------------------------------
# cube-sphere lattice: superellipsoids / superquadrics / spheres
# --------------------------------------------------------------------------
def _cube_lattice(m: int):
    """Shared-vertex triangulation of the cube [-1,1]^3 surface with an m x m
    grid per face.  Returns (P float64 [nV,3] on the cube, F int64 [12 m^2, 3])."""
    g = np.arange(m + 1)
    A, B = np.meshgrid(g, g, indexing="ij")
    A = A.ravel()
    B = B.ravel()
    zeros = np.zeros_like(A)
    full = np.full_like(A, m)
    # (axis-permuted integer coordinates, outward orientation flag)
    faces = [
        (np.stack([full, A, B], 1), False),
        (np.stack([zeros, A, B], 1), True),
        (np.stack([A, full, B], 1), True),
        (np.stack([A, zeros, B], 1), False),
        (np.stack([A, B, full], 1), False),
        (np.stack([A, B, zeros], 1), True),
    ]
    keys = []
    tris = []
    base = 0
    ii, jj = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    ii = ii.ravel()
    jj = jj.ravel()
    for coords, flip in faces:
        keys.append((coords[:, 0] * (m + 1) + coords[:, 1]) * (m + 1) + coords[:, 2])
        a = base + ii * (m + 1) + jj
        b = base + (ii + 1) * (m + 1) + jj
        c = base + (ii + 1) * (m + 1) + jj + 1
        d = base + ii * (m + 1) + jj + 1
        t1 = np.stack([a, b, c], 1)
        t2 = np.stack([a, c, d], 1)
        if flip:
            t1 = t1[:, [0, 2, 1]]
            t2 = t2[:, [0, 2, 1]]
        tris.append(np.concatenate([t1, t2], 0))
        base += coords.shape[0]
    keys = np.concatenate(keys)
    uniq, first, inv = np.unique(keys, return_index=True, return_inverse=True)
    # vertex order: first appearance order (stable across numpy versions)
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    F = rank[inv][np.concatenate(tris, 0)]
    k = uniq[order]
    cz = k % (m + 1)
    cy = (k // (m + 1)) % (m + 1)
    cx = k // ((m + 1) * (m + 1))
    P = np.stack([cx, cy, cz], 1).astype(np.float64) * (2.0 / m) - 1.0
    return P, F


def superquadric(exponent: float = 8.0, tris: int = 2_000_000,
                 axes=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0),
                 jitter_frac: float = 0.0, jitter: float = 0.0,
                 seed: int | None = None, name: str | None = None) -> Mesh:
    """Surface |x/a|^p + |y/b|^p + |z/c|^p = 1 (p = exponent) triangulated by
    radially projecting a cube lattice (12 m^2 triangles, m = round(sqrt(tris/12))).

    ``jitter_frac`` of the triangles (chosen with ``seed``) get their vertices
    displaced by N(0, jitter) in each coordinate."""
    m = max(2, int(round(math.sqrt(tris / 12.0))))
    P, F = _cube_lattice(m)
    s = np.sum(np.abs(P) ** exponent, axis=1) ** (1.0 / exponent)
    P = P / s[:, None]
    P = P * np.asarray(axes, dtype=np.float64) + np.asarray(center, dtype=np.float64)
    if jitter_frac > 0.0 and jitter > 0.0:
        rng = np.random.default_rng(seed)
        nsel = max(1, int(round(jitter_frac * F.shape[0])))
        sel = rng.choice(F.shape[0], size=nsel, replace=False)
        vids = np.unique(F[sel].ravel())
        P[vids] += rng.normal(0.0, jitter, size=(vids.size, 3))
    return _as_mesh(P, F, name or f"superquadric_p{exponent:g}_{F.shape[0]}")


def superellipsoid(exponent: float = 8.0, tris: int = 2_000_000,
                   jitter_frac: float = 0.01, jitter: float = 1e-3,
                   seed: int = 2) -> Mesh:
    """Rounded box |x|^8+|y|^8+|z|^8=1 with ~2M triangles, 1% of the triangles
    jittered by 1e-3 (seeded)."""
    return superquadric(exponent, tris, jitter_frac=jitter_frac, jitter=jitter,
                        seed=seed, name=f"superellipsoid_p{exponent:g}")


def procedural_family(rng: np.random.Generator, tri_lo: int = 5_000,
                      tri_hi: int = 200_000) -> Mesh:
    """One random mesh of the sphere / torus / superquadric families with a
    triangle count drawn log-uniform in [tri_lo, tri_hi]."""
    kind = int(rng.integers(0, 3))
    ntri = int(round(math.exp(rng.uniform(math.log(tri_lo), math.log(tri_hi)))))
    center = rng.uniform(-2.0, 2.0, size=3)
    if kind == 0:
        rad = float(rng.uniform(0.5, 2.0))
        return superquadric(2.0, ntri, axes=(rad, rad, rad), center=center,
                            name=f"sphere_{ntri}")
    if kind == 1:
        R = float(rng.uniform(0.8, 2.0))
        r = float(rng.uniform(0.15, 0.45)) * R
        ratio = R / r
        nv = max(8, int(round(math.sqrt(ntri / (2.0 * ratio)))))
        nu = max(8, int(round(ntri / (2.0 * nv))))
        return torus(R, r, nu, nv, center=center)
    p = float(rng.uniform(2.5, 10.0))
    axes = rng.uniform(0.5, 2.0, size=3)
    return superquadric(p, ntri, axes=tuple(axes), center=center,
                        name=f"superquadric_p{p:.2f}_{ntri}")


# --------------------------------------------------------------------------
# sites
# --------------------------------------------------------------------------
def mesh_area(V, F) -> float:
    V = np.asarray(V, dtype=np.float64)
    F = np.asarray(F, dtype=np.int64)
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    return float(0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum())


def sample_sites(V, F, n: int, seed: int = 0) -> np.ndarray:
    """``n`` points uniformly distributed by area on the triangle mesh.

    A triangle is drawn from the area CDF, then a point uniformly inside it
    with the square-root barycentric map.  float64 arithmetic, float32 out."""
    V = np.asarray(V, dtype=np.float64)
    F = np.asarray(F, dtype=np.int64)
    rng = np.random.default_rng(seed)
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    area = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)
    cdf = np.cumsum(area)
    cdf /= cdf[-1]
    fi = np.searchsorted(cdf, rng.random(n), side="right")
    fi = np.minimum(fi, F.shape[0] - 1)
    r1 = np.sqrt(rng.random(n))[:, None]
    r2 = rng.random(n)[:, None]
    P = (1.0 - r1) * a[fi] + r1 * (1.0 - r2) * b[fi] + r1 * r2 * c[fi]
    return np.ascontiguousarray(P, dtype=np.float32)


# --------------------------------------------------------------------------
# bbox helpers
# --------------------------------------------------------------------------
def bbox_max_edge(V) -> float:
    """R of the reference: the longest bbox edge, float32 (main.cu:223-227)."""
    V = np.asarray(V, dtype=np.float32)
    ext = V.max(axis=0) - V.min(axis=0)
    return float(np.float32(max(ext[0], ext[1], ext[2])))


def bbox_diag(V) -> float:
    V = np.asarray(V, dtype=np.float64)
    return float(np.linalg.norm(V.max(axis=0) - V.min(axis=0)))


# --------------------------------------------------------------------------
# OBJ
# --------------------------------------------------------------------------
def load_obj(path: str) -> Mesh:
    """OBJ loader with the reference's rules: ``v x y z`` lines, ``f`` lines
    with 1-based (or negative, relative) indices and optional ``/vt/vn``
    suffixes, polygons fan-triangulated around their first corner
    (main.cu:162-228).  Unused vertices are then removed (main.cu:230-257)."""
    V = []
    F = []
    with open(path, "r") as fh:
        for line in fh:
            if len(line) < 2:
                continue
            if line[0] == "v" and line[1] in " \t":
                parts = line[2:].split()
                V.append((float(parts[0]), float(parts[1]), float(parts[2])))
            elif line[0] == "f" and line[1] in " \t":
                idx = []
                for tok in line[2:].split():
                    head = tok.split("/")[0]
                    try:
                        vi = int(head)
                    except ValueError:
                        break
                    if vi < 0:
                        vi = len(V) + vi + 1
                    idx.append(vi - 1)
                for k in range(1, len(idx) - 1):
                    F.append((idx[0], idx[k], idx[k + 1]))
    import os
    name = os.path.splitext(os.path.basename(path))[0]
    Vn = np.asarray(V, dtype=np.float32).reshape(-1, 3)
    Fn = np.asarray(F, dtype=np.int64).reshape(-1, 3)
    Vc, Fc = compact_mesh(Vn, Fn)
    return _as_mesh(Vc, Fc, name)


def compact_mesh(V, F):
    """Drop vertices no face references and renumber (main.cu:230-257)."""
    V = np.asarray(V)
    F = np.asarray(F, dtype=np.int64)
    nV = V.shape[0]
    used = np.zeros(nV, dtype=bool)
    ok = (F >= 0) & (F < nV)
    used[F[ok]] = True
    remap = np.full(nV, -1, dtype=np.int64)
    remap[used] = np.arange(int(used.sum()))
    Fr = np.where(ok, remap[np.clip(F, 0, max(nV - 1, 0))], -1)
    return V[used], Fr


def save_obj(path: str, V, F=None) -> None:
    V = np.asarray(V, dtype=np.float32)
    with open(path, "w") as fh:
        for p in V:
            fh.write(f"v {p[0]:.9g} {p[1]:.9g} {p[2]:.9g}\n")
        if F is not None:
            for t in np.asarray(F, dtype=np.int64):
                fh.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")


# --------------------------------------------------------------------------
# named workloads
# --------------------------------------------------------------------------
def workload_mesh(name: str) -> tuple[Mesh, np.ndarray, dict]:
    """The named remesh workloads: (mesh, initial sites, run parameters).

    * ``icosphere_2k``: icosphere level 5, 2,000 sites (seed 0), K=20,
      50 iterations, mode 0 (freezing off).
    * ``torus_100k``: torus R=1 r=0.3 200x100 with N(0,0.002) normal noise
      (seed 1), 100,000 sites, K=24, 100 iterations, mode 1 (freezing on).
    * ``superellipsoid_1m``: p=8 superellipsoid, ~2M triangles, 1% jittered by
      1e-3 (seed 2), 1,000,000 sites, K=32, 200 iterations.
    """
    if name == "icosphere_2k":
        m = icosphere(5)
        return m, sample_sites(m.V, m.F, 2000, seed=0), dict(k=20, iters=50, mode=0)
    if name == "torus_100k":
        m = torus(1.0, 0.3, 200, 100, noise_sigma=0.002, seed=1)
        return m, sample_sites(m.V, m.F, 100_000, seed=1), dict(k=24, iters=100, mode=1)
    if name == "superellipsoid_1m":
        m = superellipsoid(8.0, 2_000_000, 0.01, 1e-3, seed=2)
        return m, sample_sites(m.V, m.F, 1_000_000, seed=2), dict(k=32, iters=200, mode=1)
    raise KeyError(name)
