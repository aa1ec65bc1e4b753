"""Host-side logic: procedural fixtures, site sampler, OBJ rules, the C ABI
library loading and exporting every declared symbol (no device calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

from gpu_cvt_b200 import meshgen as mg

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def test_icosphere_counts():
    m = mg.icosphere(5)
    assert (m.nV, m.nF) == (10242, 20480)
    assert np.allclose(np.linalg.norm(m.V, axis=1), 1.0, atol=1e-6)


def test_torus_counts_and_noise():
    t = mg.torus(1.0, 0.3, 200, 100, noise_sigma=0.002, seed=1)
    assert (t.nV, t.nF) == (20000, 40000)
    t0 = mg.torus(1.0, 0.3, 200, 100)
    d = np.linalg.norm(t.V - t0.V, axis=1)
    assert 0.001 < d.std() < 0.003


def test_superellipsoid_is_closed_manifold():
    s = mg.superquadric(8.0, 50_000, jitter_frac=0.01, jitter=1e-3, seed=2)
    F = s.F.astype(np.int64)
    e = np.sort(np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]]), 1)
    _, c = np.unique(e[:, 0] * s.nV + e[:, 1], return_counts=True)
    assert (c == 2).all()
    assert abs(s.nF - 50_000) / 50_000 < 0.05


def test_sampler_deterministic_and_on_surface():
    m = mg.icosphere(5)
    a = mg.sample_sites(m.V, m.F, 2000, seed=0)
    b = mg.sample_sites(m.V, m.F, 2000, seed=0)
    c = mg.sample_sites(m.V, m.F, 2000, seed=1)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    r = np.linalg.norm(a, axis=1)
    assert r.max() <= 1.0 + 1e-6 and r.min() > 0.99


def test_procedural_family_sizes():
    rng = np.random.default_rng(3)
    for _ in range(6):
        m = mg.procedural_family(rng, 5_000, 20_000)
        assert 3_000 <= m.nF <= 30_000


def test_obj_rules(tmp_path):
    p = tmp_path / "q.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 9 9 9\n"
                 "f 1/1/1 2/2/2 3/3/3 4/4/4\nf -5 -4 -2\n")
    m = mg.load_obj(str(p))
    # quad fan-triangulated, negative indices resolved, unused vertex dropped
    assert m.nV == 4
    assert m.F.tolist() == [[0, 1, 2], [0, 2, 3], [0, 1, 3]]
    q = tmp_path / "r.obj"
    mg.save_obj(str(q), m.V, m.F)
    m2 = mg.load_obj(str(q))
    assert np.array_equal(m2.F, m.F) and np.allclose(m2.V, m.V)


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "gpu_cvt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(cvt_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_and_binding_agree():
    from gpu_cvt_b200 import _lib
    assert sorted(_lib.exported_symbols()) == _declared_functions()


def test_library_loads_and_exports_every_symbol():
    from gpu_cvt_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    for name in _declared_functions():
        assert hasattr(lib, name), name
    # pure host calls are safe without a GPU
    from gpu_cvt_b200 import _lib
    L = _lib.load()
    assert L.cvt_version() == 1
    assert L.cvt_status_string(5) == b"capacity exceeded"


def test_invalid_arguments_rejected_without_gpu():
    from gpu_cvt_b200 import _lib, engine
    with pytest.raises(_lib.CvtError):
        _lib.call("cvt_knn_sites", None, 10, 0, None, None, None, None)   # kk = 0
    p = engine.params(k=7)
    h = ctypes.c_void_p()
    st = _lib.load().cvt_engine_create(ctypes.byref(p), 1, 10, 10, ctypes.byref(h))
    assert st == 4 and "k must be one of" in _lib.last_error()


def build_c_driver(out_path):
    """Compile tests/c_driver/remesh_driver.c, a plain C caller of the ABI,
    against include/gpu_cvt.h and link it to libgpucvt.so."""
    import shutil
    import subprocess
    from gpu_cvt_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    _lib.load()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.dirname(_lib.LIB_PATH)
    cmd = [cc, "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(root, "include"),
           os.path.join(root, "tests", "c_driver", "remesh_driver.c"), "-L", libdir, "-lgpucvt",
           "-Wl,-rpath," + libdir, "-lm", "-o", str(out_path)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return str(out_path)


def test_c_driver_compiles_and_links(tmp_path):
    """The C ABI is usable from C as it stands: the driver builds with
    -Wall -Wextra -Werror and links against the library."""
    exe = build_c_driver(tmp_path / "remesh_driver")
    assert os.path.getsize(exe) > 0
