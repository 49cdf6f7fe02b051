"""Integral / SqrIntegral on the GPU, through the C ABI, against the oracle.

Bars: integer sources are accumulated exactly, so an F64 destination equals
the exact integral (values below 2^53) and an F32 destination equals it
rounded once; float sources are accumulated in FP64 (relative error at the
level of FP64 rounding). The reference's own F64 output (tests/golden) equals
the exact integral for integer sources.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gpu_integral(ocip, S, sqr, out_dtype):
    out = np.zeros(S.shape, out_dtype)
    Si, Di = ocip.Image(S), ocip.Image(out)
    prog = ocip.prepare_integral(Si)
    ocip.integral(prog, Si, Di, sqr=sqr)
    Di.read()
    prog.release()
    return out


def check(S, sqr, got):
    ex = O.integral_exact(S, sqr)
    if S.dtype.kind == "f" or (S.dtype.itemsize == 4 and sqr):
        np.testing.assert_allclose(got.astype(np.float64), ex,
                                   rtol=1e-12 if got.dtype == np.float64 else 1e-7,
                                   atol=1e-9)
    elif got.dtype == np.float64:
        assert np.array_equal(got, ex)
    else:
        assert np.array_equal(got, ex.astype(np.float32))


@pytest.mark.parametrize("dtype", [np.uint8, np.int8, np.uint16, np.int16, np.uint32,
                                   np.int32, np.float32, np.float64])
@pytest.mark.parametrize("sqr", [False, True])
def test_integral_types(ocip, ctx, dtype, sqr):
    ctx.make_current()
    rng = np.random.default_rng(int(sqr) * 10 + np.dtype(dtype).num)
    H, W = 300, 517
    if np.dtype(dtype).kind == "f":
        S = rng.standard_normal((H, W)).astype(dtype)
    else:
        info = np.iinfo(dtype)
        S = rng.integers(info.min, int(info.max) + 1, (H, W), dtype=np.int64).astype(dtype)
    for out in (np.float32, np.float64):
        check(S, sqr, gpu_integral(ocip, S, sqr, out))


@pytest.mark.parametrize("W,H", [(1, 1), (255, 63), (256, 64), (257, 65), (1000, 3), (3, 1000)])
def test_integral_edge_sizes(ocip, ctx, W, H):
    ctx.make_current()
    rng = np.random.default_rng(W + 7 * H)
    S = rng.integers(0, 256, (H, W), dtype=np.uint8)
    for sqr in (False, True):
        check(S, sqr, gpu_integral(ocip, S, sqr, np.float64))


def test_integral_matches_reference_golden(ocip, ctx):
    ctx.make_current()
    z = np.load(os.path.join(GOLDEN, "integral.npz"))
    ids = sorted({k.split("_")[0] for k in z.files})
    for i in ids:
        S = z[i + "_S"]
        for sqr in (0, 1):
            got = gpu_integral(ocip, S, bool(sqr), np.float64)
            ref = z[f"{i}_sqr{sqr}_f641"]
            if S.dtype.kind != "f":
                assert np.array_equal(got, ref)
            else:
                np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-9)


def test_integral_multichannel(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(21)
    S = rng.integers(0, 65536, (70, 90, 4)).astype(np.uint16)
    for sqr in (False, True):
        check(S, sqr, gpu_integral(ocip, S, sqr, np.float64))


def test_integral_large_u16_sqr_exact(ocip, ctx):
    """3840x2160 U16 squares: the total reaches ~3.6e16 > 2^53 for a full
    white image, so FP64 accumulation would round; int64 does not."""
    ctx.make_current()
    S = np.full((2160, 3840), 65535, np.uint16)
    got = gpu_integral(ocip, S, True, np.float64)
    # the exact value of the last pixel is 2160*3840*65535^2
    exact = 2160 * 3840 * 65535 ** 2
    assert int(got[-1, -1]) == int(np.float64(exact))
    assert got[0, 0] == 65535.0 ** 2


def test_integral_error_codes(ocip, ctx):
    ctx.make_current()
    S = ocip.Image(np.zeros((8, 8), np.uint8))
    prog = ocip.prepare_integral(S)
    bad_type = ocip.Image(np.zeros((8, 8), np.int32))
    bad_size = ocip.Image(np.zeros((8, 9), np.float32))
    assert ocip.lib.ocipIntegral(prog.handle, S.handle, bad_type.handle) == ocip.CL_INVALID_VALUE
    assert ocip.lib.ocipIntegral(prog.handle, S.handle, bad_size.handle) == ocip.CL_INVALID_IMAGE_SIZE
    assert ocip.lib.ocipIntegral(None, S.handle, bad_size.handle) == ocip.CL_INVALID_PROGRAM
    prog.release()
