"""Internal consistency of the oracle: fast paths equal brute force, the
reference's quirks are reproduced, edge cases behave as the reference does."""
import numpy as np
import pytest

from gpu_cvt_b200 import meshgen as mg


@pytest.fixture(scope="module")
def ico():
    m = mg.icosphere(4)
    S = mg.sample_sites(m.V, m.F, 1500, seed=3)
    return m, S


def test_grid_knn_equals_bruteforce(oracle, ico):
    _, S = ico
    for kk in (1, 5, 21, 33):
        a = oracle.knn_points(S, kk, method="bf")
        b = oracle.knn_points(S, kk, method="grid")
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_knn_ties_broken_by_index(oracle):
    # a square lattice has many exact distance ties
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), [0.0], indexing="ij"), -1).reshape(-1, 3)
    knn, d = oracle.knn_points(g.astype(np.float32), 9, method="bf")
    for i in range(len(g)):
        row_d, row_i = d[i], knn[i]
        for t in range(8):
            assert row_d[t] < row_d[t + 1] or (row_d[t] == row_d[t + 1] and row_i[t] < row_i[t + 1])


def test_knn_small_n_pads_with_sentinel(oracle):
    P = np.random.default_rng(0).random((3, 3)).astype(np.float32)
    knn, d = oracle.knn_points(P, 5, method="bf")
    assert (knn[:, 3:] == 0xFFFFFFFF).all() and np.isinf(d[:, 3:]).all()


def test_knn_frozen_rows_untouched(oracle, ico):
    _, S = ico
    frozen = np.zeros(len(S), np.uint8)
    frozen[::3] = 1
    knn = np.full((len(S), 5), 7, np.uint32)
    oracle.knn_points(S, 5, frozen=frozen, method="bf", knn=knn)
    assert (knn[::3] == 7).all() and not (knn[1::3] == 7).all()


def test_drop_self_semantics(oracle):
    raw = np.array([[0, 5, 6, 7], [3, 1, 3, 4], [9, 8, 7, 6], [3, 3, 3, 3]], np.uint32)
    out = oracle.drop_self(raw, 3)
    assert out[0].tolist() == [5, 6, 7]          # self first
    assert out[1].tolist() == [3, 3, 4]          # self in the middle
    assert out[2].tolist() == [9, 8, 7]          # self absent: first K
    assert out[3].tolist() == [3, 3, 3]          # only self -> all i (i == 3)


def test_vertex_knn_exclude_self_quirk(oracle, ico):
    m, _ = ico
    Q = m.V[:50].copy()
    a = oracle.knn_vertices(m.V, Q, 5, exclude_self=False)
    b = oracle.knn_vertices(m.V, Q, 5, exclude_self=True)
    assert (a[:, 0] == np.arange(50)).all()      # a vertex is its own nearest
    assert not (b == np.arange(50)[:, None]).any()


def test_freeze_streak_logic(oracle):
    n, K = 6, 4
    S = np.zeros((n, 3), np.float32)
    Snew = S.copy()
    Snew[1, 0] = 1.0                              # large displacement
    knn = np.tile(np.arange(K, dtype=np.uint32), (n, 1))
    prev = knn.copy()
    prev[2, 0] = 99                               # neighbour list changed
    streak = np.array([0, 3, 3, 3, 254, 255], np.uint8)
    frozen = np.zeros(n, np.uint8)
    frozen[5] = 1
    cand, counts = oracle.freeze(S, Snew, knn, prev, True, None, [0.01] * 6, [4] * 6, streak, frozen)
    assert streak.tolist() == [1, 0, 0, 4, 255, 255]
    assert cand.tolist() == [0, 0, 0, 1, 1, 1]
    assert frozen.tolist() == [0, 0, 0, 1, 1, 1]
    assert counts.tolist() == [5, 5, 4, 2]
    # first iteration: no previous list -> streak and candidates cleared, no counts
    streak2 = streak.copy()
    cand, counts = oracle.freeze(S, Snew, knn, prev, False, None, [0.01] * 6, [4] * 6, streak2, frozen)
    assert (streak2 == 0).all() and (cand == 0).all() and (counts == 0).all()


def test_tiers(oracle):
    rng = np.random.default_rng(5)
    n, K = 200, 8
    N = rng.normal(size=(n, 3)).astype(np.float32)
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    N[:100] = np.array([0, 0, 1], np.float32)     # flat half
    knn = np.zeros((n, K), np.uint32)
    knn[:100] = rng.integers(0, 100, size=(100, K))
    knn[100:] = rng.integers(100, n, size=(100, K))
    t1, nv, _ = oracle.tiers(1, N, knn)
    t2, _, L = oracle.tiers(2, N, knn)
    assert (t1[:100] == 0).all() and (nv[:100] == 0).all()
    assert t1[100:].max() == 4                    # random normals -> highest variation
    assert set(np.unique(t2)).issubset({0, 1, 2, 3, 4, 5})
    assert ((t2 == 5) == ((t1 == 4) & (L > 0.8))).all()


def test_lloyd_profiles_agree(oracle):
    m, S0, p = mg.workload_mesh("icosphere_2k")
    r0 = oracle.lloyd_run(m.V, m.F, S0, 20, 0, 10, profile=oracle.P_REF)
    r1 = oracle.lloyd_run(m.V, m.F, S0, 20, 0, 10, profile=oracle.P_MIXED)
    r2 = oracle.lloyd_run(m.V, m.F, S0, 20, 0, 10, profile=oracle.P_FP64)
    diag = mg.bbox_diag(m.V)
    assert np.abs(r0["S"] - r2["S"]).max() / diag < 1e-4
    assert np.abs(r1["S"] - r2["S"]).max() / diag < 1e-4
    # sites stay on the unit sphere's surface mesh
    rad = np.linalg.norm(r0["S"], axis=1)
    assert rad.min() > 0.99 and rad.max() <= 1.0 + 1e-6


def test_mode1_freezes(oracle):
    m = mg.torus(1.0, 0.3, 60, 30, noise_sigma=0.002, seed=1)
    S0 = mg.sample_sites(m.V, m.F, 3000, seed=1)
    r = oracle.lloyd_run(m.V, m.F, S0, 24, 1, 40)
    assert r["counts"][0].tolist() == [0, 0, 0, 0]
    assert r["frozen"].sum() > 0 and r["counts"][:, 3].sum() == r["frozen"].sum()
    r2 = oracle.lloyd_run(m.V, m.F, S0, 24, 2, 40)
    assert set(np.unique(r2["tier"])).issubset(set(range(6)))


def test_bvh_and_hausdorff(oracle):
    m = mg.icosphere(3)
    nodes, tri = oracle.bvh_build(m.V, m.F)
    assert sorted(tri.tolist()) == list(range(m.nF))
    leaves = nodes[nodes["triCount"] > 0]
    assert leaves["triCount"].max() <= 8 and leaves["triCount"].sum() == m.nF
    c = mg.icosphere(2)
    Vc = c.V * np.float32(1.02)
    a = oracle.hausdorff_one_sided(Vc, c.F, m.V, m.F, use_bvh=True)
    b = oracle.hausdorff_one_sided(Vc, c.F, m.V, m.F, use_bvh=False)
    assert a == b and 0.015 < a < 0.03


def test_extract_faces_dual_mesh(oracle):
    m = mg.icosphere(4)
    S = mg.sample_sites(m.V, m.F, 800, seed=2)
    N = S / np.linalg.norm(S, axis=1, keepdims=True)
    U, V = oracle.frames(N, np.arange(len(S)))
    raw, _ = oracle.knn_points(S, 21)
    knn = oracle.drop_self(raw, 20)
    F = oracle.extract_faces(S, U, V, knn, float(mg.bbox_max_edge(S)))
    assert F.shape[0] > len(S)                    # roughly 2 triangles per site
    assert (F[:, 0] < F[:, 1]).all() and (F[:, 1] < F[:, 2]).all()
    assert len(np.unique(F, axis=0)) == len(F)


def _ru32(x):
    """float64 -> float32 rounded toward +inf."""
    r = np.float32(x)
    return np.where(r.astype(np.float64) < x, np.nextafter(r, np.float32(np.inf)), r).astype(np.float32)


def test_face_skip_bound_is_sound(oracle):
    """The projection kernel skips a face when lb > 0 and lb^2 > 1.001 best,
    lb being its lower bound on the distance from the query to whatever the
    closest-point code returns for the face (bounding sphere about the FP32
    centroid, radius rounded up; margins 0.05 (dc + radius) + 1e-4
    max|coordinate| + 1e-4 dc^2 / radius; faces with a corner angle under
    ~5.7 degrees are never skipped).  The same bound, restated here, stays
    below the distance of the oracle's FP32 closest point (the arithmetic of
    the FP32 profile, the one with the largest rounding) on thin triangles,
    small and large scales, coordinates up to 1e4 and queries on, near and
    far from the face."""
    rng = np.random.default_rng(11)
    n = 6000
    scale = 10.0 ** rng.uniform(-3, 0, n)
    base = rng.normal(size=(n, 3)) * (10.0 ** rng.uniform(-1, 4, n))[:, None]
    # corners: half random shapes, half thin ones near the angle limit
    a = np.zeros((n, 3))
    b = np.stack([np.ones(n), np.zeros(n), np.zeros(n)], 1)
    ang = np.where(rng.random(n) < 0.5, rng.uniform(0.3, 2.5, n), rng.uniform(0.101, 0.2, n))
    ln = rng.uniform(0.3, 1.0, n)
    c = np.stack([ln * np.cos(ang), ln * np.sin(ang), np.zeros(n)], 1)
    q, _ = np.linalg.qr(rng.normal(size=(n, 3, 3)))
    rot = lambda x: np.einsum("nij,nj->ni", q, x) * scale[:, None] + base
    A, B, C = (rot(x).astype(np.float32) for x in (a, b, c))
    A64, B64, C64 = (x.astype(np.float64) for x in (A, B, C))
    m = ((A64 + B64 + C64) / 3.0).astype(np.float32)
    r2 = np.max([((X - m.astype(np.float64)) ** 2).sum(1) for X in (A64, B64, C64)], axis=0)
    rad = _ru32(np.sqrt(r2) * (1.0 + 1e-9))
    P = [A64, B64, C64]
    flag = np.ones(n, bool)
    for j in range(3):
        u, v = P[(j + 1) % 3] - P[j], P[(j + 2) % 3] - P[j]
        cr = np.cross(u, v)
        flag &= (cr * cr).sum(1) >= 0.01 * (u * u).sum(1) * (v * v).sum(1)
    # triangles that FP32 collapses (tiny faces at coordinates of ~1e4) have
    # no normal; the angle flag already excludes them
    nrm = np.cross(B64 - A64, C64 - A64)
    with np.errstate(invalid="ignore", divide="ignore"):
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    checked = 0
    worst = np.inf
    for trial in range(3):
        w = rng.uniform(-0.5, 1.5, (n, 3))
        w /= w.sum(1, keepdims=True)
        on = w[:, :1] * A64 + w[:, 1:2] * B64 + w[:, 2:] * C64
        h = scale * 10.0 ** rng.uniform(-5, 2, n) * rng.choice([-1.0, 1.0], n)
        Q = (on + h[:, None] * nrm).astype(np.float32)
        d = Q - m
        dc = np.sqrt((d * d).sum(1, dtype=np.float32)).astype(np.float32)
        mc = np.maximum(np.abs(Q).max(1), np.abs(m).max(1))
        lb = (dc - rad - np.float32(0.05) * (dc + rad) - np.float32(1e-4) * mc
              - np.float32(1e-4) * (dc * dc / rad)).astype(np.float32)
        for i in np.nonzero(flag & (lb > 0))[0]:
            p = oracle.closest_point_tri(Q[i], A[i], B[i], C[i]).astype(np.float64)
            d2 = float(((p - Q[i].astype(np.float64)) ** 2).sum())
            ratio = d2 / (float(lb[i]) ** 2)
            worst = min(worst, ratio)
            checked += 1
    assert checked > 5000
    assert worst >= 1.0, f"bound above the computed distance: d2 / lb^2 = {worst}"


def test_bvh_projection_is_the_closest_point(oracle):
    """The oracle's BVH projection finds the closest point on the whole mesh:
    its distance equals a scan of every face."""
    from gpu_cvt_b200 import meshgen as mg
    m = mg.superellipsoid(8.0, 4_000, 0.01, 1e-3, seed=2)
    rng = np.random.default_rng(1)
    P = (m.V[rng.integers(0, m.nV, 150)] + rng.normal(0, 0.05, (150, 3))).astype(np.float32)
    for prof in (oracle.P_REF, oracle.P_MIXED):
        Q = oracle.project_bvh(P, m.V, m.F, profile=prof)
        d = np.linalg.norm(Q.astype(np.float64) - P, axis=1)
        A, B, Cc = m.V[m.F[:, 0]], m.V[m.F[:, 1]], m.V[m.F[:, 2]]
        for i in range(0, 150, 5):
            dmin = np.sqrt(min(oracle.point_tri_d2(P[i], A[f], B[f], Cc[f]) for f in range(m.nF)))
            assert abs(d[i] - dmin) <= 1e-6 * (1 + dmin)


def test_pca_frames_recover_plane_and_sphere_normals(oracle):
    """On a plane the PCA normal is the plane's normal whatever the start
    vertex normal; on a finely sampled sphere it is close to radial."""
    from gpu_cvt_b200 import meshgen as mg
    rng = np.random.default_rng(2)
    P = np.c_[rng.random((500, 2)), np.zeros(500)].astype(np.float32)
    tilt = np.array([[1, 0, 0], [0, 0.8, -0.6], [0, 0.6, 0.8]], np.float32)
    P = P @ tilt.T
    knn, _ = oracle.knn_points(P, 13, method="bf")
    knn = oracle.drop_self(knn, 12)
    N = np.tile(np.array([[0.3, 0.1, 0.95]], np.float32), (1, 1))
    U, V = oracle.pca_frames(P, knn, N / np.linalg.norm(N), np.zeros(500, np.int32))
    nrm = np.cross(U, V)
    assert np.abs(np.abs(nrm @ tilt[:, 2]) - 1).max() < 1e-5
    m = mg.icosphere(5)
    S = mg.sample_sites(m.V, m.F, 4000, seed=3)
    knn, _ = oracle.knn_points(S, 21, method="grid")
    knn = oracle.drop_self(knn, 20)
    N = oracle.vertex_normals(m.V, m.F)
    near = oracle.knn_vertices(m.V, S, 1)[:, 0]
    U, V = oracle.pca_frames(S, knn, N, near)
    nrm = np.cross(U, V)
    radial = S / np.linalg.norm(S, axis=1, keepdims=True)
    assert np.median(np.abs((nrm * radial).sum(1))) > 0.9999
