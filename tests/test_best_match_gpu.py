"""ocipProximityIndx: a measure's best match in one call, through the C ABI.

The answer (value, x, y) must equal ocipMinIndx / ocipMaxIndx / ocipMinAbsIndx
/ ocipMaxAbsIndx on the map the one-pair call writes, ties included (those
follow the reference's reduction order, cl-files/Statistics.cl). On the
tensor path the reduction runs in the scoring kernel's epilogue; maps with
NaN scores, the plain path and templates beyond 64 x 64 take the written map.
"""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu

MEAS = ["SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr", "CrossCorr_Norm"]
OPS = ["MinIndx", "MaxIndx", "MinAbsIndx", "MaxAbsIndx"]


def reference_answer(ocip, m, op, S, T):
    """The one-pair call's map, reduced by the statistics entry point."""
    Si, Ti = ocip.Image(S), ocip.Image(T)
    Di = ocip.Image(np.zeros(S.shape, np.float32))
    ocip.check(ocip.proximity(m, Si, Ti, Di), m)
    prog = ocip.prepare_statistics(Di)
    rc, v, x, y = ocip.index_reduce(op, prog, Di)
    ocip.check(rc, op)
    prog.release()
    for h in (Si, Ti, Di):
        h.release()
    return v, x, y


def fused_answer(ocip, m, op, S, T, with_dest):
    Si, Ti = ocip.Image(S), ocip.Image(T)
    out = np.zeros(S.shape, np.float32)
    Di = ocip.Image(out) if with_dest else None
    rc, v, x, y = ocip.proximity_index(m, op, Si, Ti, Di)
    ocip.check(rc, "ocipProximityIndx")
    if Di is not None:
        Di.read()
        Di.release()
    Si.release()
    Ti.release()
    return (v, x, y), (out if with_dest else None)


@pytest.mark.parametrize("m", [0, 1, 3, 4])
def test_u8_ties_match_the_index_reduction(ocip, tensor, m):
    rng = np.random.default_rng(m)
    S = rng.integers(0, 4, (170, 600), dtype=np.uint8)  # many equal scores
    T = rng.integers(0, 4, (9, 12), dtype=np.uint8)
    for op in OPS:
        ref = reference_answer(ocip, MEAS[m], op, S, T)
        got, _ = fused_answer(ocip, MEAS[m], op, S, T, with_dest=False)
        assert got == ref, (MEAS[m], op, got, ref)
        assert tensor.last_path() == ocip.PATH_TENSOR


@pytest.mark.parametrize("m", [0, 1, 3, 4])
def test_f32_blob_field_with_and_without_dest(ocip, tensor, m):
    S = bench.blob_field(700, 530, nblobs=30, seed=m)
    T = S[100:131, 420:451].copy()
    for op in OPS:
        ref = reference_answer(ocip, MEAS[m], op, S, T)
        got, _ = fused_answer(ocip, MEAS[m], op, S, T, with_dest=False)
        assert got == ref, (MEAS[m], op, got, ref)
    got, out = fused_answer(ocip, MEAS[m], "MaxIndx", S, T, with_dest=True)
    assert got == reference_answer(ocip, MEAS[m], "MaxIndx", S, T)
    assert np.array_equal(out, ocip.match(MEAS[m], S, T), equal_nan=True)


def test_best_match_finds_the_template(ocip, tensor):
    S = bench.blob_field(900, 700, nblobs=40, seed=9)
    T = S[300:331, 500:531].copy()
    Si, Ti = ocip.Image(S), ocip.Image(T)
    rc, v, x, y = ocip.proximity_index("CrossCorr_Norm", "MaxIndx", Si, Ti)
    assert rc == 0 and (x, y) == (515, 315) and abs(v - 1.0) < 1e-5
    rc, v, x, y = ocip.proximity_index("SqrDistance", "MinIndx", Si, Ti)
    assert rc == 0 and (x, y) == (515, 315)
    Si.release()
    Ti.release()


def test_nan_scores_take_the_map_path(ocip, tensor):
    """A black region gives CrossCorr_Norm = 0/0: the answer is the map
    reduction's, whose NaN handling depends on where the NaNs lie."""
    rng = np.random.default_rng(3)
    S = rng.integers(0, 256, (120, 300), dtype=np.uint8)
    S[:, :60] = 0
    T = rng.integers(1, 256, (8, 8), dtype=np.uint8)
    for op in OPS:
        ref = reference_answer(ocip, "CrossCorr_Norm", op, S, T)
        got, _ = fused_answer(ocip, "CrossCorr_Norm", op, S, T, with_dest=False)
        assert (np.isnan(got[0]) and np.isnan(ref[0]) and got[1:] == ref[1:]) or got == ref, \
            (op, got, ref)


def test_plain_path_and_large_templates(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(5)
    S = rng.integers(0, 6, (200, 300), dtype=np.uint8)
    T = rng.integers(0, 6, (70, 66), dtype=np.uint8)  # beyond 64 x 64: map path
    for path in (ocip.PATH_PLAIN, ocip.PATH_TENSOR):
        ctx.set_path(path)
        for op in ("MinIndx", "MaxIndx"):
            assert fused_answer(ocip, "CrossCorr", op, S, T, False)[0] == \
                reference_answer(ocip, "CrossCorr", op, S, T)
    ctx.set_path(ocip.PATH_PLAIN)


def test_argument_checks(ocip, ctx):
    ctx.make_current()
    S = ocip.Image(np.zeros((40, 50), np.float32))
    T = ocip.Image(np.zeros((5, 5), np.float32))
    D64 = ocip.Image(np.zeros((40, 50), np.float64))
    import ctypes
    v, x, y = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    args = (ctypes.byref(v), ctypes.byref(x), ctypes.byref(y))
    assert ocip.lib.ocipProximityIndx(7, 0, S.handle, T.handle, None, *args) == ocip.CL_INVALID_VALUE
    assert ocip.lib.ocipProximityIndx(3, 9, S.handle, T.handle, None, *args) == ocip.CL_INVALID_VALUE
    assert ocip.lib.ocipProximityIndx(3, 0, S.handle, T.handle, D64.handle, *args) == \
        ocip.CL_INVALID_VALUE
    assert ocip.lib.ocipProximityIndx(3, 0, S.handle, T.handle, None, None, None, None) == \
        ocip.CL_INVALID_VALUE
    for h in (S, T, D64):
        h.release()
