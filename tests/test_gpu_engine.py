"""Whole-run parity of the fused engine with the CPU oracle's Lloyd loop
(main.cu:669-881), for every mode and profile, plus batching and
segment admission mid-run ("same result alone and in the mix")."""
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


def run_engine(eng, mesh_np, S0, k, mode, iters, profile="ref", ex_quirk=True):
    m = eng.Mesh(mesh_np.V, mesh_np.F)
    cells = eng.grid_cells(m, len(S0), k)
    e = eng.Engine(eng.params(k=k, mode=mode, profile=profile, ex_quirk=ex_quirk), 1, len(S0), cells)
    seg = e.add(m, S0)
    e.run(iters)
    S = e.sites_f64(seg) if profile == "fp64" else e.sites(seg)
    st = e.state(seg)
    counts = np.array([[e.stats(seg, i)[f] for f in ("same", "low", "both", "newly_frozen")] for i in range(iters)])
    e.close()
    m.close()
    return S, st, counts


@pytest.fixture(scope="module")
def c1():
    m, S, p = mg.workload_mesh("icosphere_2k")
    return m, S


@pytest.fixture(scope="module")
def small_torus():
    m = mg.torus(1.0, 0.3, 80, 40, noise_sigma=0.002, seed=1)
    return m, mg.sample_sites(m.V, m.F, 4000, seed=1)


@pytest.mark.parametrize("iters", [1, 2, 5])
def test_mode0_ref_bitexact_early(eng, oracle, c1, iters):
    m, S0 = c1
    S, st, counts = run_engine(eng, m, S0, 20, 0, iters)
    r = oracle.lloyd_run(m.V, m.F, S0, 20, 0, iters)
    assert np.array_equal(S, r["S"])
    assert np.array_equal(st["knn"], r["knn"])
    assert np.array_equal(st["knnv"], r["knnv"])
    assert np.array_equal(counts, r["counts"])


def test_mode0_ref_icosphere_2k_full_run(eng, oracle, c1):
    """The 2k-site icosphere workload: K=20, 50 iterations, freezing off."""
    m, S0 = c1
    S, st, counts = run_engine(eng, m, S0, 20, 0, 50)
    r = oracle.lloyd_run(m.V, m.F, S0, 20, 0, 50)
    diag = mg.bbox_diag(m.V)
    err = np.abs(S.astype(np.float64) - r["S"]).max() / diag
    assert err == 0.0, f"max deviation {err:.3e} of the bbox diagonal"
    assert np.array_equal(counts, r["counts"])


@pytest.mark.parametrize("mode", [1, 2])
def test_freezing_modes_bitexact(eng, oracle, small_torus, mode):
    m, S0 = small_torus
    S, st, counts = run_engine(eng, m, S0, 24, mode, 30)
    r = oracle.lloyd_run(m.V, m.F, S0, 24, mode, 30)
    assert np.array_equal(st["tier"], r["tier"])
    assert np.array_equal(counts, r["counts"])
    assert np.array_equal(st["frozen"], r["frozen"]) and st["frozen"].sum() > 0
    assert np.array_equal(S, r["S"])


def test_mixed_profile_bitexact(eng, oracle, small_torus):
    m, S0 = small_torus
    S, st, counts = run_engine(eng, m, S0, 24, 1, 10, profile="mixed")
    r = oracle.lloyd_run(m.V, m.F, S0, 24, 1, 10, profile=oracle.P_MIXED)
    assert np.array_equal(S, r["S"]) and np.array_equal(counts, r["counts"])


@pytest.mark.parametrize("k", [8, 32])
def test_list_sizes_bitexact(eng, oracle, small_torus, k):
    """The smallest and the largest supported K (K=32 is the 1M-site
    workload's): lists, masks and positions equal the oracle's run."""
    m, S0 = small_torus
    S, st, counts = run_engine(eng, m, S0, k, 1, 15, profile="mixed")
    r = oracle.lloyd_run(m.V, m.F, S0, k, 1, 15, profile=oracle.P_MIXED)
    assert np.array_equal(st["knn"], r["knn"])
    assert np.array_equal(counts, r["counts"])
    assert np.array_equal(st["frozen"], r["frozen"])
    assert np.array_equal(S, r["S"])


@pytest.mark.parametrize("mode,profile", [(0, "ref"), (1, "mixed")])
def test_far_centroids_bitexact(eng, oracle, mode, profile):
    """Sites cut off from the rest (a cap of 300 plus three lone sites) get
    cells that reach the clip square, so their centroids lie far off the
    sphere; the per-thread vertex search gives up on them and the deferred
    brute-force path finishes them, with the oracle's result."""
    m = mg.icosphere(5)
    S = mg.sample_sites(m.V, m.F, 3000, seed=3)
    lone = np.array([[1, 0, 0], [0, -1, 0], [-0.6, 0.6, -0.52915]], np.float32)
    lone /= np.linalg.norm(lone, axis=1, keepdims=True)
    S0 = np.vstack([S[S[:, 2] > 0.6][:300], lone]).astype(np.float32)
    r1 = oracle.lloyd_run(m.V, m.F, S0, 20, mode, 1, profile=oracle.PROFILES[profile])
    c = r1["cent"][-3:].astype(np.float64)
    far = np.sqrt(((c[:, None, :] - m.V[None, :, :].astype(np.float64)) ** 2).sum(-1)).min(1)
    assert far.min() > 0.25          # several vertex-grid cells (about 0.06) away
    S, st, counts = run_engine(eng, m, S0, 20, mode, 6, profile=profile)
    r = oracle.lloyd_run(m.V, m.F, S0, 20, mode, 6, profile=oracle.PROFILES[profile])
    assert np.array_equal(S, r["S"])
    assert np.array_equal(st["knnv"], r["knnv"])
    assert np.array_equal(counts, r["counts"])


def _unflagged_fraction(m):
    """Share of faces with a corner angle below ~5.7 degrees (sin^2 < 0.01),
    which the projection never skips."""
    V = m.V.astype(np.float64)
    P = [V[m.F[:, j]] for j in range(3)]
    ok = np.ones(len(m.F), bool)
    for j in range(3):
        u, v = P[(j + 1) % 3] - P[j], P[(j + 2) % 3] - P[j]
        cr = np.cross(u, v)
        ok &= (cr * cr).sum(1) >= 0.01 * (u * u).sum(1) * (v * v).sum(1)
    return 1.0 - ok.mean()


@pytest.mark.parametrize("case", ["thin_faces", "far_from_origin"])
@pytest.mark.parametrize("profile", ["ref", "mixed", "fp64"])
def test_face_skip_guards_bitexact(eng, oracle, case, profile):
    """The projection skips a face when its bounding sphere is provably
    farther than the best face so far.  Meshes that stress the rule's
    guards: long thin triangles, 40 % of them below the corner-angle limit
    under which a face is never skipped, and a torus centred ~370 units from
    the origin, where the FP32 distance to a sphere centre keeps few digits.
    Positions, vertex lists and counts equal the oracle's run."""
    if case == "thin_faces":
        m = mg.torus(1.0, 0.3, 400, 12, noise_sigma=0.002, seed=4)
        assert 0.3 < _unflagged_fraction(m) < 0.6
    else:
        m = mg.torus(1.0, 0.3, 80, 40, noise_sigma=0.002, seed=5, center=(300.0, -200.0, 100.0))
        assert np.abs(m.V).max() > 250
    S0 = mg.sample_sites(m.V, m.F, 3000, seed=6)
    S, st, counts = run_engine(eng, m, S0, 24, 1, 12, profile=profile)
    r = oracle.lloyd_run(m.V, m.F, S0, 24, 1, 12, profile=oracle.PROFILES[profile])
    assert np.array_equal(S, r["S"])
    assert np.array_equal(st["knnv"], r["knnv"])
    assert np.array_equal(counts, r["counts"])


@pytest.mark.parametrize("profile", ["ref", "mixed", "fp64"])
def test_launch_shapes_same_results_and_autotune(eng, small_torus, profile):
    """Every launch shape of the KNN, clip and projection kernels gives the
    same run bit for bit; the autotuner picks supported shapes."""
    m, S0 = small_torus
    M = eng.Mesh(m.V, m.F)
    clip = (32, 64) if profile == "fp64" else (64, 128)
    outs = []
    for kb, cb, pb in ((64, clip[0], 64), (128, clip[1], 128), (256, clip[1], 256)):
        e = eng.Engine(eng.params(k=24, mode=1, profile=profile, knn_block=kb, clip_block=cb, proj_block=pb), 1,
                       len(S0), eng.grid_cells(M, len(S0), 24))
        g = e.add(M, S0)
        e.run(12)
        outs.append(e.sites_f64(g) if profile == "fp64" else e.sites(g))
        e.close()
    assert all(np.array_equal(outs[0], o) for o in outs[1:])
    q, ms = eng.autotune(M, S0, eng.params(k=24, mode=1, profile=profile), iters=3)
    assert q.knn_block in (64, 128, 256) and q.proj_block in (64, 128, 256) and q.clip_block in clip
    assert all(v > 0 for v in ms.values())
    from gpu_cvt_b200._lib import CvtError
    with pytest.raises(CvtError):
        eng.Engine(eng.params(k=24, knn_block=96), 1, 10, 100)
    M.close()


def test_fp64_profile_matches_fp64_oracle(eng, oracle, c1):
    m, S0 = c1
    S, st, counts = run_engine(eng, m, S0, 20, 0, 10, profile="fp64")
    r = oracle.lloyd_run(m.V, m.F, S0, 20, 0, 10, profile=oracle.P_FP64)
    assert np.array_equal(S, r["S"])
    assert np.array_equal(counts, r["counts"])


def test_graph_eager_and_threads_same_results(eng, c1, small_torus):
    """The same run launched three ways gives the same sites bit for bit:
    eagerly (use_graph off), through the per-parity graphs (the first
    iteration of each parity runs eagerly while its graph is captured), and
    from two host threads at once, each with its own engine (the second
    stream of an iteration and the capture streams belong to the thread)."""
    import threading

    def run(mesh_np, S0, graph, iters=12):
        m = eng.Mesh(mesh_np.V, mesh_np.F)
        e = eng.Engine(eng.params(k=20, mode=1, profile="mixed", use_graph=graph), 1, len(S0),
                       eng.grid_cells(m, len(S0), 20))
        seg = e.add(m, S0)
        e.run(5)
        e.run(iters - 5)
        out = e.sites(seg)
        e.close()
        m.close()
        return out

    cases = [c1, small_torus]
    ref = [run(m, S0, False) for m, S0 in cases]
    for (m, S0), r in zip(cases, ref):
        assert np.array_equal(run(m, S0, True), r)
    got = [None, None]
    errs = []

    def worker(i):
        try:
            with torch.cuda.device(0):
                got[i] = run(*cases[i], True)
        except Exception as ex:  # reported below
            errs.append(ex)

    th = [threading.Thread(target=worker, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=120)
    assert not errs, errs
    for g, r in zip(got, ref):
        assert g is not None and np.array_equal(g, r)


def test_kept_graphs_reused_across_engines(eng, c1, small_torus):
    """A destroyed engine leaves its instantiated iteration graphs for the
    next engine of the same shape, which loads its own pointers and grid
    sizes into them.  Runs on other meshes and site counts through kept
    graphs equal runs through freshly instantiated ones."""
    from gpu_cvt_b200 import _lib

    def run(mesh_np, S0):
        m = eng.Mesh(mesh_np.V, mesh_np.F)
        e = eng.Engine(eng.params(k=24, mode=1, profile="mixed"), 1, len(S0), eng.grid_cells(m, len(S0), 24))
        seg = e.add(m, S0)
        e.run(8)
        out = e.sites(seg)
        e.close()
        m.close()
        return out

    cases = [small_torus, c1, (small_torus[0], small_torus[1][:1500])]
    fresh = []
    for m, S0 in cases:
        _lib.call("cvt_release_cached_memory")
        fresh.append(run(m, S0))
    for _ in range(2):
        for (m, S0), f in zip(cases, fresh):
            assert np.array_equal(run(m, S0), f)


def test_batched_segments_equal_alone(eng, c1, small_torus):
    """Three meshes in one engine give, per mesh, the same bits as alone."""
    (m1, S1), (m2, S2) = c1, small_torus
    m3 = mg.superquadric(4.0, 8000, axes=(1.0, 0.7, 0.5), name="sq")
    S3 = mg.sample_sites(m3.V, m3.F, 1500, seed=7)
    alone = [run_engine(eng, m, S, 24, 1, 12)[0] for m, S in ((m1, S1), (m2, S2), (m3, S3))]
    meshes = [eng.Mesh(m.V, m.F) for m in (m1, m2, m3)]
    sites = (S1, S2, S3)
    cells = sum(eng.grid_cells(mm, len(S), 24) for mm, S in zip(meshes, sites))
    e = eng.Engine(eng.params(k=24, mode=1), 4, sum(len(S) for S in sites), cells)
    segs = [e.add(mm, S) for mm, S in zip(meshes, sites)]
    e.run(12)
    for sg, a in zip(segs, alone):
        assert np.array_equal(e.sites(sg), a)
    e.close()


def test_admission_mid_run_equals_alone(eng, c1, small_torus):
    """A segment admitted while another is iterating (continuous batching)
    ends identical to running alone; removal frees its slot for reuse."""
    (m1, S1), (m2, S2) = c1, small_torus
    a1 = run_engine(eng, m1, S1, 24, 0, 9)[0]
    a2 = run_engine(eng, m2, S2, 24, 0, 5)[0]
    M1, M2 = eng.Mesh(m1.V, m1.F), eng.Mesh(m2.V, m2.F)
    cells = eng.grid_cells(M1, len(S1), 24) + eng.grid_cells(M2, len(S2), 24)
    e = eng.Engine(eng.params(k=24, mode=0), 2, len(S1) + len(S2), cells)
    g1 = e.add(M1, S1)
    e.run(4)
    g2 = e.add(M2, S2)
    e.run(5)
    assert e.iters(g1) == 9 and e.iters(g2) == 5
    assert np.array_equal(e.sites(g1), a1)
    assert np.array_equal(e.sites(g2), a2)
    e.remove(g1)
    g3 = e.add(M1, S1)
    e.run(9)
    assert np.array_equal(e.sites(g3), a1)
    e.close()


def test_remesh_one_call_equals_engine(eng, c1):
    m, S0 = c1
    out, counts = eng.remesh(m.V, m.F, S0, k=20, mode=0, iters=7, with_counts=True)
    S, _, c2 = run_engine(eng, m, S0, 20, 0, 7)
    assert np.array_equal(out, S) and np.array_equal(counts, c2)


def test_nan_and_tiny_segments(eng, oracle):
    m = mg.icosphere(3)
    S0 = mg.sample_sites(m.V, m.F, 30, seed=4)
    S0[3] = np.nan
    S, st, counts = run_engine(eng, m, S0, 32, 0, 3)
    r = oracle.lloyd_run(m.V, m.F, S0, 32, 0, 3)
    assert np.array_equal(S, r["S"], equal_nan=True)
    assert np.isnan(S[3]).all() and np.isfinite(np.delete(S, 3, 0)).all()
    # MIXED keeps the site that has no centroid instead of propagating NaN
    S2, _, _ = run_engine(eng, m, S0, 32, 0, 3, profile="mixed")
    r2 = oracle.lloyd_run(m.V, m.F, S0, 32, 0, 3, profile=oracle.P_MIXED)
    assert np.array_equal(S2, r2["S"], equal_nan=True)


def test_engine_evaluate_matches_oracle_pipeline(eng, oracle, small_torus):
    """Evaluation after a freezing run: dual mesh, quality and Hausdorff of
    the engine equal the oracle pipeline applied to the oracle's state."""
    m, S0 = small_torus
    M = eng.Mesh(m.V, m.F)
    e = eng.Engine(eng.params(k=24, mode=1), 1, len(S0), eng.grid_cells(M, len(S0), 24))
    g = e.add(M, S0)
    e.run(12)
    ev = e.evaluate(g)
    r = oracle.lloyd_run(m.V, m.F, S0, 24, 1, 12)
    S = r["S"]
    No = oracle.vertex_normals(m.V, m.F)
    nn = oracle.knn_vertices(m.V, S, 1)[:, 0]
    nn = np.where(r["frozen"] > 0, r["knnv"][:, 0], nn)
    U, V = oracle.frames(No, nn)
    ext = S.max(0) - S.min(0)
    R2 = float(np.float32(2.0) * np.float32(0.5) * np.float32(ext.max()))
    F = oracle.extract_faces(S, U, V, r["knn"], R2)
    assert ev["n_faces"] == len(F)
    dH = oracle.hausdorff_one_sided(S, F, m.V, m.F)
    assert abs(ev["dH"] - dH) <= 1e-6 * max(dH, 1e-12)
    q = oracle.quality(S, F)
    assert abs(ev["Qavg"] - q["Qavg"]) < 1e-5
    e.close()
    M.close()


def test_stop_rule_and_poll(eng, c1):
    m, S0 = c1
    M = eng.Mesh(m.V, m.F)
    e = eng.Engine(eng.params(k=20, mode=0), 2, 2 * len(S0), 2 * eng.grid_cells(M, len(S0), 20))
    g1, g2 = e.add(M, S0), e.add(M, S0)
    e.set_stop(g1, -1.0, 7)                  # iteration cap
    e.set_stop(g2, 1e9, 0)                   # first iteration already "converged"
    e.run(12)
    iters, state = e.poll(2)
    assert state == [2, 2] and iters == [7, 1]
    ref = run_engine(eng, m, S0, 20, 0, 7)[0]
    assert np.array_equal(e.sites(g1), ref)
    e.close()


def test_device_sampler_on_surface(eng):
    m = mg.icosphere(4)
    M = eng.Mesh(m.V, m.F)
    t = torch.empty((20000, 3), dtype=torch.float32, device="cuda")
    M.sample_sites(t, 123)
    S = t.cpu().numpy()
    r = np.linalg.norm(S, axis=1)
    assert r.max() <= 1.0 + 1e-6 and r.min() > 0.99
    assert abs(S.mean(0)).max() < 0.02          # area-uniform on a sphere: centred
    t2 = torch.empty_like(t)
    M.sample_sites(t2, 123)
    assert torch.equal(t, t2)


def test_serving_results_equal_alone(eng):
    """Continuous batching: every request's final sites equal the same request
    served alone, first come first served."""
    from gpu_cvt_b200 import server
    meshes, reqs = server.request_stream(n_requests=10, rate=2000.0, site_lo=1000, site_hi=20000, n_meshes=3, seed=9)
    srv = server.RemeshServer(meshes, k=24, mode=1, profile="mixed", hbm_budget=64 << 20, max_segments=8,
                              max_iters=40, chunk=3, keep_results=True)
    stats = srv.run(reqs)
    srv.close()
    import copy
    alone = [copy.copy(r) for r in reqs]
    for r in alone:
        r.result = None
    server.serve_plain(meshes, alone, k=24, mode=1, profile="mixed", max_iters=40, chunk=3, keep_results=True)
    for a, b in zip(reqs, alone):
        assert a.iters == b.iters and np.array_equal(a.result, b.result), a.rid
    assert stats["requests"] == 10 and stats["latency_p99_s"] >= stats["latency_p50_s"]


def test_cli_driver_contract(tmp_path):
    """gpu_cvt <mesh.obj> [mode] [iters]: the reference driver's outputs."""
    from gpu_cvt_b200 import cli, meshgen as mg
    m = mg.icosphere(4)
    obj = tmp_path / "ball.obj"
    mg.save_obj(str(obj), m.V, m.F)
    assert cli.main([str(obj), "1", "12", "--k", "24", "--out-root", str(tmp_path)]) == 0
    d = tmp_path / "experiments" / "output" / "freeze" / "ball"
    rows = (d / "eval_iters.csv").read_text().strip().split("\n")
    assert rows[0] == cli.EVAL_HEADER and len(rows) == 3          # iterations 0 and 10
    assert len(rows[1].split(",")) == 28
    for it in (0, 10):
        V = mg.load_obj(str(d / f"iter_{it:03d}.obj"))
        assert V.nV == m.nV and V.nF > m.nV
        assert len((d / f"iter_{it:03d}_frozen.txt").read_text().split()) == m.nV
        xyz = np.loadtxt(d / f"iter_{it:03d}_sites.xyz")
        assert xyz.shape == (m.nV, 3) and np.allclose(xyz, V.V, atol=1e-5)
    runs = (tmp_path / "experiments" / "runs.csv").read_text().strip().split("\n")
    assert runs[0] == cli.RUNS_HEADER and runs[1].startswith("ball,freeze,")
    dH = float(rows[2].split(",")[9])
    assert 0 < dH < 0.05


def test_c_driver_runs(tmp_path):
    """The plain C driver: engine run + evaluation, then cvt_remesh on the same
    input gives the same sites byte for byte."""
    import subprocess
    from test_host import build_c_driver
    exe = build_c_driver(tmp_path / "remesh_driver")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    f = r.stdout.split()
    vals = dict(zip(f[0::2], f[1::2]))
    assert int(vals["same"]) == 1 and int(vals["faces"]) > 8000
    assert 0 < float(vals["dH"]) < 0.01 and float(vals["Qavg"]) > 0.8


@pytest.mark.parametrize("mode,k", [(0, 24), (1, 32)])
def test_knn_radius_query_fallbacks_clustered(eng, oracle, small_torus, mode, k):
    """Sites far from uniform: 2,000 spread over the torus and 2,000 packed
    into three small patches.  The first iteration's radius comes from the
    segment's mean density, so in the patches it holds far more than the
    64-key buffer and in the sparse part fewer than K+16 sites: both fall
    back to the ring search, and later iterations mix bounded queries with
    fallbacks.  Runs with and without candidate lists agree bit for bit,
    and with the oracle."""
    m, _ = small_torus
    cen = m.V[m.F].mean(axis=1)
    parts = [mg.sample_sites(m.V, m.F, 2000, seed=7)]
    for j, v in enumerate((0, len(m.V) // 3, 2 * len(m.V) // 3)):
        near = np.nonzero(np.linalg.norm(cen - m.V[v], axis=1) < 0.08)[0]
        assert len(near) >= 4
        parts.append(mg.sample_sites(m.V, m.F[near], 667 if j < 2 else 666, seed=11 + j))
    S0 = np.ascontiguousarray(np.concatenate(parts).astype(np.float32))
    assert len(S0) == 4000
    out = {}
    for reuse in (True, False):
        M = eng.Mesh(m.V, m.F)
        e = eng.Engine(eng.params(k=k, mode=mode, profile="mixed", knn_reuse=reuse), 1, len(S0),
                       eng.grid_cells(M, len(S0), k))
        g = e.add(M, S0)
        e.run(25)
        out[reuse] = (e.sites(g), e.state(g)["knn"])
        e.close()
        M.close()
    assert np.array_equal(out[True][0], out[False][0])
    assert np.array_equal(out[True][1], out[False][1])
    r = oracle.lloyd_run(m.V, m.F, S0, k, mode, 25, profile=oracle.P_MIXED)
    assert np.array_equal(out[True][0], r["S"])


@pytest.mark.parametrize("mode,k", [(0, 24), (1, 32), (2, 20)])
def test_knn_candidate_lists_match_full_search(eng, oracle, small_torus, mode, k):
    """Lists taken from the kept candidate lists (knn_reuse, the default) are
    the lists a full search finds: whole runs with and without reuse agree
    bit for bit, and with the oracle."""
    m, S0 = small_torus
    out = {}
    for reuse in (True, False):
        M = eng.Mesh(m.V, m.F)
        e = eng.Engine(eng.params(k=k, mode=mode, profile="mixed", knn_reuse=reuse), 1, len(S0),
                       eng.grid_cells(M, len(S0), k))
        g = e.add(M, S0)
        e.run(40)
        out[reuse] = (e.sites(g), e.state(g)["knn"],
                      [e.stats(g, i)["same"] for i in range(40)])
        e.close()
        M.close()
    assert np.array_equal(out[True][0], out[False][0])
    assert np.array_equal(out[True][1], out[False][1])
    assert out[True][2] == out[False][2]
    r = oracle.lloyd_run(m.V, m.F, S0, k, mode, 40, profile=oracle.P_MIXED)
    assert np.array_equal(out[True][0], r["S"])


@pytest.mark.parametrize("profile", ["mixed", "fp64"])
def test_remesh_batch_matches_single_remeshes(eng, profile):
    """cvt_remesh_batch (meshes ingested by several host threads on their own
    streams, every segment read back with one wait) returns, per mesh, the
    sites of a one-mesh cvt_remesh with the same parameters."""
    meshes = [mg.icosphere(3), mg.torus(1.0, 0.3, 60, 30, noise_sigma=0.002, seed=2),
              mg.superquadric(4.0, 6000, seed=3), mg.icosphere(4, radius=2.0),
              mg.torus(2.0, 0.5, 40, 20, noise_sigma=0.0, seed=4)]
    meshes = meshes + meshes[:4]   # more meshes than ingest threads
    S = [mg.sample_sites(m.V, m.F, 600 + 150 * i, seed=20 + i) for i, m in enumerate(meshes)]
    prm = eng.params(k=24, mode=1, profile=profile)
    outs = eng.remesh_batch([m.V for m in meshes], [m.F for m in meshes], S, prm, 15)
    for m, s, o in zip(meshes, S, outs):
        one = eng.remesh(m.V, m.F, s, iters=15, prm=prm)
        assert np.array_equal(o, one)


def test_remesh_batch_reports_a_bad_mesh(eng):
    """A face index out of range in one mesh of the batch fails the call with
    that mesh's ingest error (raised on the calling thread)."""
    good = mg.icosphere(3)
    bad_F = good.F.copy()
    bad_F[5, 1] = len(good.V) + 7
    S = [mg.sample_sites(good.V, good.F, 300, seed=1)] * 3
    with pytest.raises(Exception, match="face index out of range"):
        eng.remesh_batch([good.V] * 3, [good.F, bad_F, good.F], S, eng.params(k=24, mode=0, profile="mixed"), 3)
