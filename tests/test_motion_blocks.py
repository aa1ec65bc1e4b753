"""The coarse motion blocks that the candidate-list check reads.

k_knn_verify (gpu_cvt_b200/csrc/cvt_engine.cuh, knn_verify_half) bounds how
far any site outside a candidate list can have come by the largest motion
recorded in the 2 x 2 x 2 coarse blocks (kBlockCells = 4 grid cells per
block edge) nearest the site's old position: per axis the block of its cell
and the neighbour on the side of the nearer block face.  Its proof needs
every point within half a block edge (less 1e-3 of it) of the position to
fall into one of those blocks, with cells computed in float32 exactly as
grid_coord computes them (floor((x - lo) * inv_h), clamped to the grid).
This restates that arithmetic and checks the claim per axis on random grids.
"""
import numpy as np

BLOCK = 4


def cell(x, lo, inv_h, dim):
    f = np.floor((x.astype(np.float32) - lo) * inv_h)
    return np.where(f >= 0, np.where(f < dim, f, dim - 1), 0).astype(np.int64)


def test_nearest_two_blocks_cover_half_a_block():
    rng = np.random.default_rng(1)
    f32 = np.float32
    tested = 0
    for _ in range(100):
        lo = f32(rng.uniform(-5, 5))
        h = f32(10 ** rng.uniform(-4, -1))
        inv_h = f32(1) / h
        dim = int(rng.integers(8, 400))
        p = (lo + rng.uniform(0, dim, 2000).astype(f32) * h).astype(f32)
        c = cell(p, lo, inv_h, dim)
        b0 = c // BLOCK - np.where(c % BLOCK < BLOCK // 2, 1, 0)
        q = (p + rng.uniform(-1, 1, 2000).astype(f32) * f32(0.999 * BLOCK / 2) * h).astype(f32)
        inside = (q >= lo) & (q < lo + dim * h)
        bq = cell(q, lo, inv_h, dim) // BLOCK
        assert np.all(((bq == b0) | (bq == b0 + 1))[inside])
        tested += int(inside.sum())
    assert tested > 150_000


def test_one_block_alone_does_not_cover():
    """The neighbour block is needed: a point half a block edge away can sit
    in the other neighbour than the position's own block."""
    f32 = np.float32
    lo, h = f32(0.0), f32(0.01)
    inv_h, dim = f32(1) / h, 64
    p = np.array([lo + f32(4.5) * h], f32)          # cell 4: first cell of block 1
    q = (p - f32(0.9 * BLOCK / 2) * h).astype(f32)  # 1.8 cells to the left: block 0
    assert cell(p, lo, inv_h, dim)[0] // BLOCK == 1
    assert cell(q, lo, inv_h, dim)[0] // BLOCK == 0
    c = cell(p, lo, inv_h, dim)[0]
    assert c // BLOCK - (1 if c % BLOCK < BLOCK // 2 else 0) == 0  # the pair chosen is {0, 1}
