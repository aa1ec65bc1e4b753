"""B200-native tangent-plane CVT remesher (restricted-Voronoi Lloyd relaxation).

Compute runs in libgpucvt.so (hand-written sm_100a CUDA behind a C ABI,
include/gpu_cvt.h); this package is the Python host side:

* ``gpu_cvt_b200.engine``  -- resident meshes, the multi-segment Lloyd engine,
                              one-call ``remesh``
* ``gpu_cvt_b200.stages``  -- the reference's stage functions over torch tensors
* ``gpu_cvt_b200.meshgen`` -- seeded procedural meshes, site sampler, OBJ I/O
"""
__version__ = "0.1.0"
