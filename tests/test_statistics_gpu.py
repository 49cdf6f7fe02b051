"""Index reductions (ocipMinIndx, ocipMaxIndx, ocipMinAbsIndx, ocipMaxAbsIndx)
through the C ABI: value and coordinates equal the oracle's restatement of
the reference's reduction order, ties and NaNs included, for every type."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

NAMES = ["MinIndx", "MaxIndx", "MinAbsIndx", "MaxAbsIndx"]


def check(ocip, a):
    img = ocip.Image(a)
    prog = ocip.prepare_statistics(img)
    try:
        for name in NAMES:
            rc, v, x, y = ocip.index_reduce(name, prog, img)
            assert rc == 0, name
            ev, ex, ey = O.index_reduce(name, a)
            assert (x, y) == (ex, ey), (name, a.dtype, (x, y), (ex, ey))
            assert v == ev or (np.isnan(v) and np.isnan(ev)), (name, v, ev)
    finally:
        prog.release()
        img.release()


@pytest.mark.parametrize("dtype", [np.uint8, np.int8, np.uint16, np.int16, np.uint32, np.int32,
                                   np.float32, np.float64])
def test_types_and_ties(ocip, ctx, dtype):
    ctx.make_current()
    rng = np.random.default_rng(3)
    for shape in [(37, 300), (16, 256), (100, 1000), (1, 5)]:
        lo = -4 if np.issubdtype(dtype, np.signedinteger) or dtype in (np.float32, np.float64) else 0
        a = rng.integers(lo, 4, shape).astype(dtype)  # few values: many ties
        check(ocip, a)
    if np.issubdtype(dtype, np.signedinteger):
        a = rng.integers(-3, 3, (50, 70)).astype(dtype)
        a[10, 20] = np.iinfo(dtype).min  # abs() of the most negative value
        check(ocip, a)


def test_nan_and_random_floats(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(4)
    a = rng.standard_normal((300, 700)).astype(np.float32)
    check(ocip, a)
    a[rng.integers(0, 300, 40), rng.integers(0, 700, 40)] = np.nan
    a[0, 0] = np.nan
    check(ocip, a)


def test_best_match_on_a_score_map(ocip, ctx):
    """The template's own location is the arg-min of SqrDistance and the
    arg-max of CrossCorr_Norm."""
    import bench
    ctx.make_current()
    S = bench.blob_field(500, 300, nblobs=30, seed=5)
    y0, x0 = 120, 230
    T = S[y0:y0 + 31, x0:x0 + 31].copy()
    ctx.set_path(ocip.PATH_TENSOR)
    sq = ocip.match("SqrDistance", S, T)
    cc = ocip.match("CrossCorr_Norm", S, T)
    ctx.set_path(ocip.PATH_PLAIN)
    for m, name in ((sq, "MinIndx"), (cc, "MaxIndx")):
        img = ocip.Image(m)
        prog = ocip.prepare_statistics(img)
        rc, v, x, y = ocip.index_reduce(name, prog, img)
        prog.release()
        img.release()
        assert rc == 0 and (x, y) == (x0 + 15, y0 + 15), (name, x, y)


def test_multichannel_is_refused(ocip, ctx):
    ctx.make_current()
    img = ocip.Image(np.zeros((10, 10, 3), np.uint8))
    prog = ocip.prepare_statistics(img)
    rc, _, _, _ = ocip.index_reduce("MinIndx", prog, img)
    prog.release()
    img.release()
    assert rc == ocip.CL_INVALID_VALUE
