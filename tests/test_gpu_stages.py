"""Stage-by-stage parity of the libgpucvt kernels with the CPU oracle.

Integer outputs (neighbour lists, masks, counts) must be identical; FP32
outputs too, because kernels and oracle follow the same pinned operation
order (explicit FMAs, IEEE division and square root).
"""
import numpy as np
import pytest

from gpu_cvt_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def st():
    from gpu_cvt_b200 import stages
    assert torch.cuda.is_available()
    return stages


@pytest.fixture(scope="module")
def c1():
    m, S, p = mg.workload_mesh("icosphere_2k")
    return m, S


@pytest.mark.parametrize("kk", [1, 5, 21, 25, 33])
def test_knn_sites_bitexact(st, oracle, c1, kk):
    _, S = c1
    n = len(S)
    knn = torch.zeros((n, kk), dtype=torch.int32, device="cuda")
    dist = torch.zeros((n, kk), dtype=torch.float32, device="cuda")
    st.run_knn_bitonic_hubs(n, kk, None, dev(S), knn, dist)
    ok, od = oracle.knn_points(S, kk, method="bf")
    assert np.array_equal(host(knn).view(np.uint32), ok)
    assert np.array_equal(host(dist), od)


def test_knn_sites_frozen_rows_untouched(st, oracle, c1):
    _, S = c1
    n = len(S)
    frozen = np.zeros(n, np.uint8)
    frozen[::2] = 1
    knn = torch.full((n, 21), 7, dtype=torch.int32, device="cuda")
    st.run_knn_bitonic_hubs(n, 21, dev(frozen), dev(S), knn, None)
    k = host(knn)
    assert (k[::2] == 7).all()
    ok, _ = oracle.knn_points(S, 21, method="bf")
    assert np.array_equal(k[1::2].view(np.uint32), ok[1::2])


def test_knn_small_and_degenerate_inputs(st, oracle):
    rng = np.random.default_rng(0)
    for n in (1, 3, 40):
        P = rng.random((n, 3)).astype(np.float32)
        knn = torch.zeros((n, 9), dtype=torch.int32, device="cuda")
        dist = torch.zeros((n, 9), dtype=torch.float32, device="cuda")
        st.run_knn_bitonic_hubs(n, 9, None, dev(P), knn, dist)
        ok, od = oracle.knn_points(P, 9, method="bf")
        assert np.array_equal(host(knn).view(np.uint32), ok) and np.array_equal(host(dist), od)
    # duplicates and a lattice full of exact ties; a planar set (zero z extent)
    g = np.stack(np.meshgrid(np.arange(20), np.arange(20), [0.0], indexing="ij"), -1).reshape(-1, 3)
    P = np.concatenate([g, g[:50]]).astype(np.float32)
    knn = torch.zeros((len(P), 13), dtype=torch.int32, device="cuda")
    st.run_knn_bitonic_hubs(len(P), 13, None, dev(P), knn, None)
    ok, _ = oracle.knn_points(P, 13, method="bf")
    assert np.array_equal(host(knn).view(np.uint32), ok)


@pytest.mark.parametrize("ex", [False, True])
def test_knn_vertices_bitexact(st, oracle, c1, ex):
    m, S = c1
    out = torch.zeros((len(S), 5), dtype=torch.int32, device="cuda")
    st.knn_vertices_bruteforce_k(dev(m.V), m.nV, dev(S), len(S), None, out, 5, exclude_self=ex)
    assert np.array_equal(host(out), oracle.knn_vertices(m.V, S, 5, exclude_self=ex))


def test_knn_query_to_mesh(st, oracle, c1):
    m, S = c1
    knn = torch.zeros((len(S), 5), dtype=torch.int32, device="cuda")
    st.run_knn_bitonic_query_to_mesh(m.nV, dev(m.V), dev(S), len(S), 5, None, knn, None)
    assert np.array_equal(host(knn), oracle.knn_vertices(m.V, S, 5))


def test_drop_self_and_restore(st, oracle, c1):
    _, S = c1
    raw, _ = oracle.knn_points(S, 21, method="bf")
    raw[5] = raw[5][::-1]                       # self last
    raw[7, :] = 7                               # only self
    out = torch.zeros((len(S), 20), dtype=torch.int32, device="cuda")
    st.knn_drop_self(dev(raw.view(np.int32)), out, len(S), 21, 20)
    assert np.array_equal(host(out).view(np.uint32), oracle.drop_self(raw, 20))
    frozen = (np.arange(len(S)) % 3 == 0).astype(np.uint8)
    prev = torch.full((len(S), 20), -5, dtype=torch.int32, device="cuda")
    st.restore_prev_knn_for_frozen(dev(frozen), prev, out, len(S), 20)
    h = host(out)
    assert (h[::3] == -5).all() and not (h[1::3] == -5).any()


def test_normals_and_frames_bitexact(st, oracle, c1):
    m, S = c1
    off, fcs = oracle.build_vf(m.nV, m.F)
    N = torch.zeros((m.nV, 3), dtype=torch.float32, device="cuda")
    st.vertex_normals(dev(m.V), dev(m.F), dev(off), dev(fcs), N)
    No = oracle.vertex_normals(m.V, m.F)
    assert np.array_equal(host(N), No)
    knnv = oracle.knn_vertices(m.V, S, 5)
    knnv[3, 0] = -1
    U = torch.zeros((len(S), 3), dtype=torch.float32, device="cuda")
    V = torch.zeros_like(U)
    st.uv_from_nearest_vertex_normal(N, dev(knnv), U, V)
    Uo, Vo = oracle.frames(No, knnv[:, 0])
    assert np.array_equal(host(U), Uo) and np.array_equal(host(V), Vo)


@pytest.mark.parametrize("profile", [0, 1])
def test_clip_centroids_bitexact(st, oracle, c1, profile):
    m, S = c1
    No = oracle.vertex_normals(m.V, m.F)
    knnv = oracle.knn_vertices(m.V, S, 5)
    Uo, Vo = oracle.frames(No, knnv[:, 0])
    raw, _ = oracle.knn_points(S, 21, method="bf")
    knn = oracle.drop_self(raw, 20)
    R = mg.bbox_max_edge(m.V)
    cent = torch.zeros((len(S), 3), dtype=torch.float32, device="cuda")
    nv = torch.zeros(len(S), dtype=torch.int32, device="cuda")
    st.centroids_tangent_voronoi(dev(S), dev(Uo), dev(Vo), dev(knn.view(np.int32)), len(S), 20, R, cent, profile, nv)
    co, nvo = oracle.clip_centroids(S, Uo, Vo, knn, R, profile=profile, return_nverts=True)
    assert np.array_equal(host(nv), nvo)
    assert np.array_equal(host(cent), co)


def test_clip_overflow_fallback_exact(st, oracle):
    # a site with many neighbours on a circle: its cell has >32 vertices, so
    # the shared-memory path hands it to the 64-vertex fallback
    k = 40
    ang = np.linspace(0, 2 * np.pi, k, endpoint=False)
    P = np.concatenate([[[0, 0, 0]], np.stack([np.cos(ang), np.sin(ang), np.zeros(k)], 1) * 0.1]).astype(np.float32)
    n = len(P)
    knn = np.zeros((n, 40), np.uint32)
    for i in range(n):
        knn[i] = [j for j in range(n) if j != i][:40]
    U = np.tile(np.array([1, 0, 0], np.float32), (n, 1))
    V = np.tile(np.array([0, 1, 0], np.float32), (n, 1))
    cent = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    nv = torch.zeros(n, dtype=torch.int32, device="cuda")
    st.centroids_tangent_voronoi(dev(P), dev(U), dev(V), dev(knn.view(np.int32)), n, 40, 1.0, cent, 0, nv)
    co, nvo = oracle.clip_centroids(P, U, V, knn, 1.0, return_nverts=True)
    assert nvo[0] == 40
    assert np.array_equal(host(nv), nvo) and np.array_equal(host(cent), co)


@pytest.mark.parametrize("profile", [0, 1])
def test_project_bitexact(st, oracle, c1, profile):
    m, S = c1
    rng = np.random.default_rng(1)
    cent = (S * 1.01 + rng.normal(scale=0.01, size=S.shape)).astype(np.float32)
    cent[11] = np.nan
    knnv = oracle.knn_vertices(m.V, cent, 5)
    off, fcs = oracle.build_vf(m.nV, m.F)
    out = torch.zeros_like(dev(cent))
    st.project_centroids_to_mesh(dev(cent), dev(m.V), dev(m.F), dev(off), dev(fcs), dev(knnv), m.nV, m.nF, len(S),
                                 dev(S), out, 5, profile)
    exp = oracle.project(cent, m.V, m.F, knnv, profile=profile, Sold=S)
    assert np.array_equal(host(out), exp, equal_nan=True)


@pytest.mark.parametrize("tiered", [False, True])
def test_freeze_bitexact(st, oracle, c1, tiered):
    _, S = c1
    n = len(S)
    rng = np.random.default_rng(2)
    Snew = (S + rng.normal(scale=0.01, size=S.shape)).astype(np.float32)
    raw, _ = oracle.knn_points(S, 21, method="bf")
    knn = oracle.drop_self(raw, 20)
    prev = knn.copy()
    prev[rng.random(n) < 0.2, 3] = 0
    tier = rng.integers(0, 6, n).astype(np.uint8) if tiered else None
    thr = [1e-4, 1e-4, 2e-4, 2e-4, 1e-4, 3e-4]
    need = [4, 9, 14, 19, 24, 9] if tiered else [4] * 6
    streak = rng.integers(0, 30, n).astype(np.uint8)
    frozen = (rng.random(n) < 0.1).astype(np.uint8)
    d_streak, d_frozen = dev(streak), dev(frozen)
    d_cand = torch.zeros(n, dtype=torch.uint8, device="cuda")
    counts = torch.zeros(4, dtype=torch.int32, device="cuda")
    st.freeze_test_streak(dev(S), dev(Snew), dev(knn.view(np.int32)), dev(prev.view(np.int32)), 20, 1, thr, need,
                          d_streak, d_cand, d_frozen, counts, tier=dev(tier) if tiered else None)
    s2, f2 = streak.copy(), frozen.copy()
    cand, cnt = oracle.freeze(S, Snew, knn, prev, True, tier, thr, need, s2, f2)
    assert np.array_equal(host(d_streak), s2) and np.array_equal(host(d_frozen), f2)
    assert np.array_equal(host(d_cand), cand) and np.array_equal(host(counts), cnt)
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    st.count_frozen(d_frozen, n, total)
    assert int(host(total)[0]) == int(f2.sum())


@pytest.mark.parametrize("mode", [1, 2])
def test_tiers_bitexact(st, oracle, c1, mode):
    m, S = c1
    No = oracle.vertex_normals(m.V, m.F)
    nn = oracle.knn_vertices(m.V, S, 1)[:, 0]
    sn = No[nn]
    raw, _ = oracle.knn_points(S, 21, method="bf")
    knn = oracle.drop_self(raw, 20)
    tier = torch.zeros(len(S), dtype=torch.uint8, device="cuda")
    st.tier_ids(mode, dev(sn), dev(knn.view(np.int32)), tier)
    exp, _, _ = oracle.tiers(mode, sn, knn)
    assert np.array_equal(host(tier), exp)


def test_hausdorff(oracle):
    from gpu_cvt_b200.engine import Mesh
    ref = mg.icosphere(5)
    mesh = Mesh(ref.V, ref.F)
    c = mg.icosphere(3)
    Vc = (c.V * np.float32(1.01)).astype(np.float32)
    Vc[::5] *= np.float32(0.985)
    got = mesh.hausdorff_from(dev(Vc), dev(c.F))
    exp = oracle.hausdorff_one_sided(Vc, c.F, ref.V, ref.F)
    # same minima; a near-first traversal may prune a box whose bound ties the
    # best distance to the last ulp, hence a relative 1e-6 tolerance
    assert abs(got - exp) <= 1e-6 * exp
    mesh.close()


def test_hausdorff_symmetric(oracle):
    """Both sides of scripts/evaluate.py's hausdorff_bvh, including probes at
    input vertices that no face uses."""
    from gpu_cvt_b200.engine import Mesh
    ref = mg.icosphere(4)
    c = mg.icosphere(3)
    Vc = (c.V * np.float32(1.02)).astype(np.float32)
    Vc[::7] *= np.float32(0.97)
    Vc = np.vstack([Vc, np.array([[0.0, 0.0, 1.6]], np.float32)])   # unreferenced vertex
    A, B = Mesh(Vc, c.F), Mesh(ref.V, ref.F)
    got = A.hausdorff(B)
    ab = oracle.hausdorff_one_sided(Vc, c.F, ref.V, ref.F)
    ba = oracle.hausdorff_one_sided(ref.V, ref.F, Vc, c.F)
    assert abs(got["self_to_other"] - ab) <= 1e-6 * ab
    assert abs(got["other_to_self"] - ba) <= 1e-6 * ba
    assert got["dH"] == max(got["self_to_other"], got["other_to_self"])
    assert abs(got["self_to_other"] - 0.6) < 1e-5       # the lone vertex sets this side
    A.close(); B.close()


def test_extract_faces_and_quality(st, oracle):
    m = mg.icosphere(4)
    S = mg.sample_sites(m.V, m.F, 1500, seed=2)
    N = (S / np.linalg.norm(S, axis=1, keepdims=True)).astype(np.float32)
    U, V = oracle.frames(N, np.arange(len(S)))
    raw, _ = oracle.knn_points(S, 21, method="bf")
    knn = oracle.drop_self(raw, 20)
    R2 = float(mg.bbox_max_edge(S))
    F = st.extract_faces(dev(S), dev(U), dev(V), dev(knn.view(np.int32)), R2)
    Fo = oracle.extract_faces(S, U, V, knn, R2)
    assert np.array_equal(host(F), Fo)
    q = st.quality(dev(S), F)
    qo = oracle.quality(S, Fo)
    for k in qo:
        assert abs(q[k] - qo[k]) <= 1e-4 * max(1.0, abs(qo[k])), k


def _d2h(ptr, n, dtype):
    from cuda.bindings import runtime as rt
    out = np.empty(n, dtype)
    err, = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0
    return out


def test_mesh_ingest_on_device(oracle):
    """cvt_mesh_create does compaction, the face CSR and the bounds on the
    device: the same arrays as the host restatement (main.cu:230-285)."""
    from gpu_cvt_b200.engine import Mesh
    from gpu_cvt_b200._lib import CvtError
    rng = np.random.default_rng(5)
    m = mg.icosphere(3)
    # unreferenced vertices interleaved, faces shuffled
    extra = rng.normal(size=(7, 3)).astype(np.float32) * 3
    perm = rng.permutation(m.nV + 7)
    Vall = np.vstack([m.V, extra])[perm]
    inv = np.argsort(perm)
    F = inv[m.F][rng.permutation(m.nF)].astype(np.int32)
    M = Mesh(Vall, F)
    Vc, Fc = mg.compact_mesh(Vall, F)
    assert (M.nV, M.nF) == (Vc.shape[0], F.shape[0])
    pV, pF, pN, poff, pfcs = M.device_arrays()
    assert np.array_equal(_d2h(pV, Vc.size, np.float32).reshape(-1, 3), Vc)
    assert np.array_equal(_d2h(pF, F.size, np.int32).reshape(-1, 3), Fc)
    off, fcs = oracle.build_vf(M.nV, Fc)
    assert np.array_equal(_d2h(poff, M.nV + 1, np.int32), off)
    assert np.array_equal(_d2h(pfcs, 3 * M.nF, np.int32), fcs)
    assert np.array_equal(_d2h(pN, Vc.size, np.float32).reshape(-1, 3), oracle.vertex_normals(Vc, Fc))
    R = float(np.max(Vall.max(0) - Vall.min(0)))
    assert M.R == np.float32(R)
    a = Vc[Fc[:, 1]].astype(np.float64) - Vc[Fc[:, 0]]
    b = Vc[Fc[:, 2]].astype(np.float64) - Vc[Fc[:, 0]]
    area = 0.5 * np.linalg.norm(np.cross(a, b), axis=1).sum()
    assert abs(M.area - area) <= 1e-6 * area
    M.close()
    bad = F.copy()
    bad[3, 1] = Vall.shape[0]
    with pytest.raises(CvtError):
        Mesh(Vall, bad)
    Vn = Vall.copy()
    Vn[F[0, 0], 2] = np.nan
    with pytest.raises(CvtError):
        Mesh(Vn, F)
    unused = int(np.setdiff1d(np.arange(Vall.shape[0]), F.ravel())[0])
    Vn = Vall.copy()
    Vn[unused] = np.nan          # no face uses it: accepted
    Mesh(Vn, F).close()


@pytest.mark.parametrize("name", ["icosphere", "torus", "superquadric"])
def test_bvh_matches_recursive_build(oracle, name):
    """The device's level-by-level build gives the reference's recursive
    median-split tree node for node (evaluate.cuh:114-201)."""
    from gpu_cvt_b200.engine import Mesh
    if name == "icosphere":
        m = mg.icosphere(4)
    elif name == "torus":
        m = mg.torus(1.0, 0.3, 120, 60, noise_sigma=0.002, seed=1)
    else:
        m = mg.superquadric(8.0, 30_000, jitter_frac=0.01, jitter=1e-3, seed=2)
    M = Mesh(m.V, m.F)
    nodes, tri = M.bvh()
    en, et = oracle.bvh_build(m.V, m.F)
    assert nodes.shape == en.shape and np.array_equal(tri, et)
    for f in en.dtype.names:
        assert np.array_equal(nodes[f], en[f]), f
    M.close()


def test_memory_pool_reuse_and_release():
    """Meshes and engines freed go back to the library's pool and are reused;
    cvt_release_cached_memory hands the unused part back; work continues."""
    from gpu_cvt_b200 import engine as E
    from gpu_cvt_b200._lib import call
    m = mg.icosphere(3)
    S0 = mg.sample_sites(m.V, m.F, 500, seed=2)
    out = []
    for rep in range(3):
        out.append(E.remesh(m.V, m.F, S0, k=20, mode=0, iters=5))
        if rep == 1:
            call("cvt_release_cached_memory")
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[1], out[2])
