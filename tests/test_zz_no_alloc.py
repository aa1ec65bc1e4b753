"""cvt_knn_sites_noalloc, the site KNN for callers that cannot allocate device
memory at call time (its temporaries live in a fixed array inside the
library), must return what the allocating cvt_knn_sites returns.

Kept in a file of its own, collected last, so a failure here never hides the
other GPU tests; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _knn(name, P, kk, frozen=None):
    from gpu_cvt_b200 import _lib
    n = P.shape[0]
    knn = torch.full((n, kk), -7, dtype=torch.int32, device="cuda")
    dist = torch.full((n, kk), -1.0, dtype=torch.float32, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    fz = None if frozen is None else C.c_void_p(frozen.data_ptr())
    _lib.call(name, C.c_void_p(P.data_ptr()), n, kk, fz, C.c_void_p(knn.data_ptr()), C.c_void_p(dist.data_ptr()), st)
    torch.cuda.synchronize()
    return knn.cpu().numpy(), dist.cpu().numpy()


def test_noalloc_knn_matches_allocating_knn_twice_in_a_row():
    from gpu_cvt_b200 import meshgen as mg
    assert torch.cuda.is_available()
    m = mg.torus(1.0, 0.3, 120, 60, noise_sigma=0.002, seed=1)
    # two different calls back to back: the second must not see the first's
    # leftovers in the shared scratch array
    cases = [(mg.sample_sites(m.V, m.F, 50_000, seed=3), 25, None),
             (mg.sample_sites(mg.icosphere(4).V, mg.icosphere(4).F, 3_000, seed=4), 21, 2)]
    for S, kk, fz_every in cases:
        P = torch.from_numpy(S).cuda()
        frozen = None
        if fz_every:
            f = np.zeros(S.shape[0], np.uint8)
            f[::fz_every] = 1
            frozen = torch.from_numpy(f).cuda()
        a_knn, a_d = _knn("cvt_knn_sites", P, kk, frozen)
        b_knn, b_d = _knn("cvt_knn_sites_noalloc", P, kk, frozen)
        # integer lists: identical; squared distances: identical bits (the
        # same kernels on the same inputs), i.e. within any tolerance
        assert np.array_equal(a_knn, b_knn)
        assert np.array_equal(a_d, b_d)


def test_noalloc_knn_allocates_no_device_memory():
    """The point of the entry point: a warm call takes no device memory.  The
    library's own pool is trimmed first, the outputs are allocated before the
    measurement, and the device's free memory must not move across the call."""
    from gpu_cvt_b200 import _lib, meshgen as mg
    m = mg.icosphere(4)
    P = torch.from_numpy(mg.sample_sites(m.V, m.F, 20_000, seed=5)).cuda()
    _knn("cvt_knn_sites_noalloc", P, 16)            # warm: symbol address, module load
    _lib.call("cvt_release_cached_memory")
    knn = torch.zeros((P.shape[0], 16), dtype=torch.int32, device="cuda")
    dist = torch.zeros((P.shape[0], 16), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.call("cvt_knn_sites_noalloc", C.c_void_p(P.data_ptr()), P.shape[0], 16, None, C.c_void_p(knn.data_ptr()),
              C.c_void_p(dist.data_ptr()), st)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_knn_rejects_oversized_input():
    from gpu_cvt_b200 import _lib
    n = 131072 + 1
    P = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    knn = torch.zeros((n, 5), dtype=torch.int32, device="cuda")
    st = _lib.load().cvt_knn_sites_noalloc(C.c_void_p(P.data_ptr()), n, 5, None, C.c_void_p(knn.data_ptr()), None,
                                          None)
    assert st == 5 and "CVT_NOALLOC_MAX_POINTS" in _lib.last_error()
