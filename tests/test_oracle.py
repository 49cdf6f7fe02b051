"""The CPU oracle, pinned against the reference's own kernel sources.

The reference has no golden vectors of its own; the fixtures in
tests/golden were produced by the reference's cl-files/ImageProximity.cl and
cl-files/Integral.cl compiled for the host (tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cases():
    z = np.load(os.path.join(GOLDEN, "proximity.npz"))
    keys = sorted({k.split("_")[0] for k in z.files})
    return z, keys


def test_restatement_matches_reference_fixtures():
    """Both arithmetic forms of the C restatement equal the reference's
    outputs bit for bit, on every stored case (8 types x channels x 5
    measures x shapes, _Cached and plain kernels)."""
    z, keys = _cases()
    n = 0
    for k in keys:
        S, T = z[k + "_S"], z[k + "_T"]
        for m in range(5):
            for fused, suffix in ((False, ""), (True, "_fma")):
                ref = z[f"{k}_m{m}{suffix}"]
                got = O.proximity_refexact(m, S, T, fused=fused)
                assert got.dtype == ref.dtype
                assert np.array_equal(got, ref, equal_nan=True), (k, m, fused)
                n += 1
    assert n == len(keys) * 10


def test_exact_oracle_consistent_with_reference():
    """Where the reference's float sums are exact (8-bit sources, integer
    measures, small templates) the exact oracle equals it; elsewhere they agree
    to float accuracy."""
    z, keys = _cases()
    for k in keys:
        S, T = z[k + "_S"], z[k + "_T"]
        for m in range(5):
            ref = z[f"{k}_m{m}"].astype(np.float64)
            ex = O.proximity_exact(m, S, T)
            fin = np.isfinite(ex) & np.isfinite(ref)
            assert np.array_equal(np.isfinite(ex), np.isfinite(ref)) or m in (1, 4)
            scale = np.abs(ex[fin]).max() + 1e-30
            tol = 1e-3 if S.dtype in (np.uint32, np.int32) else 2e-5
            if S.dtype == np.float64:
                tol = 1e-12
            assert np.max(np.abs(ex[fin] - ref[fin])) <= tol * scale, (k, m)


def test_u8_small_template_exact_equals_reference():
    rng = np.random.default_rng(7)
    S = rng.integers(0, 256, (40, 37), dtype=np.uint8)
    T = rng.integers(0, 256, (16, 16), dtype=np.uint8)
    for m in (0, 2, 3):
        ref = O.proximity_reference(m, S, T)
        ex = O.proximity_exact(m, S, T)
        assert np.array_equal(ref.astype(np.float64), ex)


def test_known_answers_3x3():
    """Hand-computed values on a 3x3 image with a 2x2 template.

    S = [[1,2,3],[4,5,6],[7,8,9]], T = [[1,2],[3,4]]; the window of output
    (x, y) covers S[y-1..y][x-1..x] (anchor -tw/2, -th/2), zero outside."""
    S = np.arange(1, 10, dtype=np.uint8).reshape(3, 3)
    T = np.array([[1, 2], [3, 4]], dtype=np.uint8)
    Sp = np.zeros((4, 4))
    Sp[1:, 1:] = S
    cc = np.zeros((3, 3)); sd = np.zeros((3, 3)); ad = np.zeros((3, 3)); ss = np.zeros((3, 3))
    for y in range(3):
        for x in range(3):
            win = Sp[y:y + 2, x:x + 2]
            cc[y, x] = (win * T).sum()
            sd[y, x] = ((win - T) ** 2).sum()
            ad[y, x] = np.abs(win - T).sum()
            ss[y, x] = (win ** 2).sum()
    # e.g. output (0,0): window [[0,0],[0,1]] -> CrossCorr = 4, SqrDistance = 1+4+9+9 = 23
    assert cc[0, 0] == 4 and sd[0, 0] == 23 and ad[0, 0] == 9
    assert cc[2, 2] == 5 * 1 + 6 * 2 + 8 * 3 + 9 * 4 == 77
    tt = 30.0
    expect = {0: sd, 1: sd / np.sqrt(ss * tt), 2: ad, 3: cc, 4: cc / np.sqrt(ss * tt)}
    for m, e in expect.items():
        got = O.proximity_refexact(m, S, T).astype(np.float64)
        np.testing.assert_allclose(got, e, rtol=1e-6)
        np.testing.assert_allclose(O.proximity_exact(m, S, T), e, rtol=1e-15)
        if O.ref_available():
            np.testing.assert_allclose(O.proximity_reference(m, S, T).astype(np.float64), e,
                                       rtol=1e-6)


def test_norm_of_zero_window_matches_reference():
    """A window of zeros gives 0/0 (NaN) or x/0 (inf) exactly as the reference."""
    S = np.zeros((6, 6), np.float32)
    T = np.ones((3, 3), np.float32)
    for m in (1, 4):
        got = O.proximity_refexact(m, S, T)
        assert np.isnan(got[3, 3]) or np.isinf(got[3, 3])
        if O.ref_available():
            ref = O.proximity_reference(m, S, T)
            assert np.array_equal(np.isnan(ref), np.isnan(got))


def test_integral_exact_matches_reference_fixtures():
    z = np.load(os.path.join(GOLDEN, "integral.npz"))
    ids = sorted({k.split("_")[0] for k in z.files})
    for i in ids:
        S = z[i + "_S"]
        for sqr in (0, 1):
            ex = O.integral_exact(S, sqr)
            k64 = f"{i}_sqr{sqr}_f641"
            ref64 = z[k64]
            if S.dtype.kind != "f":
                # integer sums below 2^53: the reference's F64 scan is exact
                assert np.array_equal(ref64, ex), k64
            else:
                np.testing.assert_allclose(ref64, ex, rtol=1e-12, atol=1e-9)
            k32 = f"{i}_sqr{sqr}_f640"
            if k32 in z.files:
                ref32 = z[k32].astype(np.float64)
                # the reference accumulates in float: exact below 2^24 only
                np.testing.assert_allclose(ref32, ex, rtol=2e-6, atol=1e-3)


@pytest.mark.skipif(not O.ref_available(), reason="reference kernels not built")
@pytest.mark.parametrize("W,H", [(1, 1), (63, 7), (64, 8), (65, 9), (200, 3)])
def test_integral_reference_edge_sizes(W, H):
    rng = np.random.default_rng(W * 1000 + H)
    S = rng.integers(0, 256, (H, W), dtype=np.uint8)
    for sqr in (0, 1):
        assert np.array_equal(O.integral_reference(S, sqr, 1), O.integral_exact(S, sqr))


def test_backward_oracle_matches_finite_differences():
    rng = np.random.default_rng(3)
    S = rng.random((9, 11))
    T = rng.random((3, 4))
    g = rng.standard_normal((9, 11))
    for m in (0, 4):
        dS, dT = O.proximity_backward(m, S, T, g)

        def f(S_, T_):
            return float((O.proximity_exact(m, S_, T_) * g).sum())
        h = 1e-6
        for (i, j) in [(0, 0), (1, 2), (2, 3)]:
            Tp, Tm = T.copy(), T.copy()
            Tp[i, j] += h; Tm[i, j] -= h
            fd = (f(S, Tp) - f(S, Tm)) / (2 * h)
            assert abs(fd - dT[i, j]) <= 1e-6 * max(1.0, abs(fd))
        for (i, j) in [(0, 0), (4, 5), (8, 10)]:
            Sp, Sm = S.copy(), S.copy()
            Sp[i, j] += h; Sm[i, j] -= h
            fd = (f(Sp, T) - f(Sm, T)) / (2 * h)
            assert abs(fd - dS[i, j]) <= 1e-6 * max(1.0, abs(fd))


def test_index_reduce_oracle_matches_brute_force_without_ties():
    """With a unique extreme, the reference's reduction order does not matter:
    the oracle's (value, x, y) equals numpy's argmin / argmax."""
    rng = np.random.default_rng(21)
    for shape in [(37, 300), (16, 256), (1, 1), (70, 513)]:
        a = rng.permutation(shape[0] * shape[1]).reshape(shape).astype(np.float32) - 1000.0
        for name, fn in [("MinIndx", np.argmin), ("MaxIndx", np.argmax),
                         ("MinAbsIndx", lambda v: np.argmin(np.abs(v))),
                         ("MaxAbsIndx", lambda v: np.argmax(np.abs(v)))]:
            v, x, y = O.index_reduce(name, a)
            iy, ix = np.unravel_index(fn(a), a.shape)
            ref = a[iy, ix] if "Abs" not in name else abs(a[iy, ix])
            assert (x, y) == (ix, iy) and v == ref, (name, shape)


def test_index_reduce_oracle_tie_order():
    """Ties follow the reference's reduction tree. Across 256 x 16 groups the
    first group in row-major group order wins. Inside a group, a work-item
    (lx, ly) keeps its first pixel of a tie along x, and the tree folds
    lid + s into lid (s = 128 .. 1), an equal value never replacing: below,
    row 9's candidate (lid 145) reaches lid 17 at the first level, before row
    7's (lid 113, via lid 49 at s = 64) meets it at s = 32, so row 9 wins."""
    a = np.zeros((40, 600), np.uint8) + 9
    a[30, 5] = a[3, 100] = a[3, 516] = 1   # groups (x0, y1), (x0, y0), (x2, y0)
    assert O.index_reduce("MinIndx", a) == (1.0, 100, 3)
    b = np.zeros((16, 256), np.uint8) + 9
    b[7, 33] = b[7, 17] = b[9, 1] = 1
    assert O.index_reduce("MinIndx", b) == (1.0, 1, 9)
