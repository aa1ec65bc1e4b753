"""Run the reference-kernel harness (oracle/_ref/ref_harness) on a workload.

TEST INFRASTRUCTURE ONLY.  The harness binary is built from the reference's
own CUDA headers by ``make -C oracle ref`` and runs on a GPU; this module
writes its input file, runs it and parses its output.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "ref_harness")


def available() -> bool:
    return os.path.exists(BIN)


def run(V, F, S, K, mode, iters, dump=(), knn_mode=1, timeout=1800):
    """knn_mode 0: the reference's hub KNN; 1: exact brute-force KNN with every
    other stage done by the reference's kernels."""
    V = np.ascontiguousarray(V, np.float32)
    F = np.ascontiguousarray(F, np.int32)
    S = np.ascontiguousarray(S, np.float32)
    dump = sorted(int(d) for d in dump if 1 <= d <= iters)
    nV, nF, nS = V.shape[0], F.shape[0], S.shape[0]
    with tempfile.TemporaryDirectory() as td:
        fi, fo = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fi, "wb") as fh:
            fh.write(struct.pack("8i", nV, nF, nS, K, mode, iters, int(knn_mode), len(dump)))
            if dump:
                fh.write(np.asarray(dump, np.int32).tobytes())
            fh.write(V.tobytes())
            fh.write(F.tobytes())
            fh.write(S.tobytes())
        subprocess.run([BIN, fi, fo], check=True, timeout=timeout)
        raw = open(fo, "rb").read()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a.copy()

    it, nd = take(np.int32, 2)
    dumps = take(np.float32, nd * nS * 3).reshape(nd, nS, 3)
    counts = take(np.int32, it * 4).reshape(it, 4)
    knn0 = take(np.uint32, nS * K).reshape(nS, K)
    knnv0 = take(np.int32, nS * 5).reshape(nS, 5)
    cent0 = take(np.float32, nS * 3).reshape(nS, 3)
    frozen = take(np.uint8, nS)
    tier = take(np.uint8, nS)
    stage_ms = take(np.float32, it * 6).reshape(it, 6)
    quality = take(np.float32, 6)
    dH = float(take(np.float32, 1)[0])
    nfaces = int(take(np.int32, 1)[0])
    wall_ms = float(take(np.float32, 1)[0])
    return dict(dump_iters=np.asarray(dump, np.int32), S=dumps, counts=counts, knn0=knn0, knnv0=knnv0,
                cent0=cent0, frozen=frozen, tier=tier, stage_ms=stage_ms, quality=quality, dH=dH,
                nfaces=nfaces, wall_ms=wall_ms)
