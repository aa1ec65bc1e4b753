"""The two options beyond the reference's algorithm, on the GPU against the
CPU oracle's restatement of the same arithmetic (bit for bit):

* projection through the mesh's BVH -- the exact closest point on the whole
  mesh instead of the one-rings of the 5 nearest vertices
  (near_project.cuh:149-189);
* frames from the PCA normal of each site's K neighbours instead of the
  nearest vertex normal (site_normals.cuh:69-110).

Both in the engine (every profile, freezing on) and as stage calls."""
import ctypes as C

import numpy as np
import pytest

from gpu_cvt_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def eng():
    from gpu_cvt_b200 import engine
    assert torch.cuda.is_available()
    return engine


def run_engine(eng, m_np, S0, k, mode, iters, profile, proj, frame):
    m = eng.Mesh(m_np.V, m_np.F)
    cells = eng.grid_cells(m, len(S0), k)
    e = eng.Engine(eng.params(k=k, mode=mode, profile=profile, proj=proj, frame=frame), 1, len(S0), cells)
    seg = e.add(m, S0)
    e.run(iters)
    S = e.sites_f64(seg) if profile == "fp64" else e.sites(seg)
    st = e.state(seg)
    counts = np.array([[e.stats(seg, i)[f] for f in ("same", "low", "both", "newly_frozen")] for i in range(iters)])
    e.close()
    m.close()
    return S, st, counts


@pytest.fixture(scope="module")
def torus():
    m = mg.torus(1.0, 0.3, 80, 40, noise_sigma=0.002, seed=1)
    return m, mg.sample_sites(m.V, m.F, 4000, seed=1)


@pytest.fixture(scope="module")
def rounded_box():
    """A small version of the 1M-site workload's mesh: superellipsoid with
    1% of the triangles jittered, whose thin faces make the one-ring and the
    whole-mesh closest points differ."""
    m = mg.superellipsoid(8.0, 20_000, 0.01, 1e-3, seed=2)
    return m, mg.sample_sites(m.V, m.F, 5000, seed=2)


@pytest.mark.parametrize("profile", ["ref", "mixed", "fp64"])
@pytest.mark.parametrize("proj,frame", [("bvh", "vertex"), ("onering", "pca"), ("bvh", "pca")])
def test_engine_options_bitexact(eng, oracle, torus, profile, proj, frame):
    m, S0 = torus
    S, st, counts = run_engine(eng, m, S0, 24, 1, 12, profile, proj, frame)
    r = oracle.lloyd_run(m.V, m.F, S0, 24, 1, 12, profile=oracle.PROFILES[profile], proj=proj, frame=frame)
    assert np.array_equal(counts, r["counts"])
    assert np.array_equal(st["frozen"], r["frozen"])
    assert np.array_equal(st["knn"], r["knn"])
    assert np.array_equal(st["knnv"], r["knnv"])
    assert np.array_equal(S, r["S"])


@pytest.mark.parametrize("mode", [0, 2])
def test_engine_bvh_projection_on_thin_faces(eng, oracle, rounded_box, mode):
    m, S0 = rounded_box
    S, st, counts = run_engine(eng, m, S0, 32, mode, 8, "mixed", "bvh", "vertex")
    r = oracle.lloyd_run(m.V, m.F, S0, 32, mode, 8, profile=oracle.P_MIXED, proj="bvh")
    assert np.array_equal(counts, r["counts"]) and np.array_equal(S, r["S"])
    assert np.isfinite(S).all()


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("profile", [0, 1])
def test_stage_project_bvh_bitexact_and_closest(oracle, rounded_box, profile):
    from gpu_cvt_b200 import _lib, engine as E
    m, S0 = rounded_box
    rng = np.random.default_rng(4)
    cent = (S0 + rng.normal(0, 0.02, S0.shape)).astype(np.float32)
    cent[::97] = np.nan
    M = E.Mesh(m.V, m.F)
    out = torch.zeros((len(cent), 3), dtype=torch.float32, device="cuda")
    cent_d, S0_d = _dev(cent), _dev(S0)      # held until the call has finished
    _lib.call("cvt_project_bvh", M.handle, C.c_void_p(cent_d.data_ptr()), len(cent), profile,
              C.c_void_p(S0_d.data_ptr()), C.c_void_p(out.data_ptr()), None)
    got = out.cpu().numpy()
    M.close()
    want = oracle.project_bvh(cent, m.V, m.F, profile=profile, Sold=S0)
    assert np.array_equal(got, want, equal_nan=True)
    # the exact closest point: against a scan of every face (200 sites)
    ok = np.isfinite(cent).all(1)
    idx = np.flatnonzero(ok)[:200]
    d_bvh = np.linalg.norm(got[idx].astype(np.float64) - cent[idx], axis=1)
    for i, d in zip(idx, d_bvh):
        A, B, Cc = m.V[m.F[:, 0]], m.V[m.F[:, 1]], m.V[m.F[:, 2]]
        d_all = np.sqrt(min(oracle.point_tri_d2(cent[i], A[f], B[f], Cc[f]) for f in
                            np.argsort(np.linalg.norm((A + B + Cc) / 3 - cent[i], axis=1))[:64]))
        assert abs(d - d_all) <= 1e-6 * (1 + d_all)


def test_stage_frames_pca_bitexact(oracle, torus):
    from gpu_cvt_b200 import _lib
    m, S0 = torus
    knn, _ = oracle.knn_points(S0, 25, method="grid")
    knn = oracle.drop_self(knn, 24)
    N = oracle.vertex_normals(m.V, m.F)
    near = oracle.knn_vertices(m.V, S0, 1)
    n = len(S0)
    U = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    Vv = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    S_d, knn_d, N_d, near_d = _dev(S0), _dev(knn.view(np.int32)), _dev(N), _dev(near)  # held until synchronised
    _lib.call("cvt_frames_pca", C.c_void_p(S_d.data_ptr()), n, C.c_void_p(knn_d.data_ptr()), 24,
              C.c_void_p(N_d.data_ptr()), C.c_void_p(near_d.data_ptr()), 1, C.c_void_p(U.data_ptr()),
              C.c_void_p(Vv.data_ptr()), None)
    torch.cuda.synchronize()
    u_o, v_o = oracle.pca_frames(S0, knn, N, near[:, 0])
    assert np.array_equal(U.cpu().numpy(), u_o) and np.array_equal(Vv.cpu().numpy(), v_o)
