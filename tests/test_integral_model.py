"""The integral scan's tile decomposition, restated in numpy (no GPU).

integral.cu computes D = the inclusive 2-D prefix sum in three passes over
128 x 32 tiles: (1) per-row tile sums RowSum and each tile's bottom-row local
integral LB; (2) RowLeft = exclusive scan of RowSum across the tiles of a row,
ColTop = exclusive scan of LB over the bands; (3) per tile, Top(x) = ColTop(x)
+ the sum of ColTop at the last column of every tile left of x, then each row
adds RowLeft and its prefix within the tile to the running column sums. This
test checks that algebra against np.cumsum on integer inputs (exact) for sizes
with partial tiles on both edges, so that the kernels' arithmetic is pinned
independently of the GPU.
"""
import numpy as np
import pytest

TW, TH = 128, 32


def tiled_integral(S):
    H, W = S.shape
    nbx, nby = -(-W // TW), -(-H // TH)
    S = S.astype(np.int64)
    rowsum = np.zeros((H, nbx), np.int64)
    lb = np.zeros((nby, W), np.int64)
    for by in range(nby):
        for bx in range(nbx):
            t = S[by * TH:(by + 1) * TH, bx * TW:(bx + 1) * TW]
            rowsum[by * TH:by * TH + t.shape[0], bx] = t.sum(axis=1)
            lb[by, bx * TW:bx * TW + t.shape[1]] = np.cumsum(t.sum(axis=0))
    rowleft = np.cumsum(rowsum, axis=1) - rowsum
    coltop = np.cumsum(lb, axis=0) - lb
    D = np.zeros((H, W), np.int64)
    for by in range(nby):
        for bx in range(nbx):
            x0, x1 = bx * TW, min(W, (bx + 1) * TW)
            y0, y1 = by * TH, min(H, (by + 1) * TH)
            left_tiles = sum(coltop[by, min(W, (j + 1) * TW) - 1] for j in range(bx))
            acc = coltop[by, x0:x1] + left_tiles
            for y in range(y0, y1):
                acc = acc + rowleft[y, bx] + np.cumsum(S[y, x0:x1])
                D[y, x0:x1] = acc
    return D


@pytest.mark.parametrize("H,W", [(1, 1), (31, 127), (32, 128), (33, 129), (70, 300),
                                 (100, 520)])
def test_tiled_decomposition_is_the_integral(H, W):
    rng = np.random.default_rng(H * 1000 + W)
    S = rng.integers(0, 256, (H, W))
    want = np.cumsum(np.cumsum(S.astype(np.int64), axis=0), axis=1)
    assert np.array_equal(tiled_integral(S), want)
