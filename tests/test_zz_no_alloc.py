"""ocipIntegralNoAlloc: the Integral entry point that allocates no device memory.

It serves callers that cannot let a library call cudaMalloc (their device
memory belongs to another allocator, or allocation while running would block
them). Its scratch is a fixed array shared by every call, so these tests run
it twice in a row on different images and compare each result with the
regular ocipIntegral / ocipSqrIntegral, which must agree exactly (both
accumulate exactly and round once), and with the oracle's exact integral.
Two more cases nearly fill the array (one channel at 7300 x 7300, two
channels at 5100 x 5100), checked on sampled rows including the last row
and column. This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _device_image(ocip, arr):
    img = ocip.Image(arr)
    img.send()
    ptr, pitch = img.device_ptr()
    return img, ptr, pitch


def _regular(ocip, S, sqr, out_dtype):
    out = np.zeros(S.shape, out_dtype)
    Si, Di = ocip.Image(S), ocip.Image(out)
    prog = ocip.prepare_integral(Si)
    ocip.integral(prog, Si, Di, sqr=sqr)
    Di.read()
    prog.release()
    return out


def _no_alloc(ocip, ctx, S, sqr, out_dtype):
    Si, sp, spitch = _device_image(ocip, S)
    out = np.zeros(S.shape, out_dtype)
    Di, dp, dpitch = _device_image(ocip, out)
    ctx.finish()
    rc = ocip.lib.ocipIntegralNoAlloc(int(sqr), Si.desc, ctypes.c_void_p(sp), spitch,
                                      Di.desc, ctypes.c_void_p(dp), dpitch,
                                      ctypes.c_void_p(ctx.stream()))
    ocip.check(rc, "ocipIntegralNoAlloc")
    Di.read()
    Si.release()
    Di.release()
    return out


def test_no_alloc_matches_regular_entry_point_twice(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(77)
    # first call: U8 squares into F64
    S1 = rng.integers(0, 256, (300, 517), dtype=np.uint8)
    a = _no_alloc(ocip, ctx, S1, True, np.float64)
    assert np.array_equal(a, _regular(ocip, S1, True, np.float64))
    assert np.array_equal(a, O.integral_exact(S1, True))
    # second call reuses the same scratch: F32 sums into F32, another size
    S2 = rng.standard_normal((129, 1000)).astype(np.float32)
    b = _no_alloc(ocip, ctx, S2, False, np.float32)
    assert np.array_equal(b, _regular(ocip, S2, False, np.float32))
    # FP64 accumulation rounded once into F32: within one F32 rounding
    ex = O.integral_exact(S2, False)
    np.testing.assert_allclose(b.astype(np.float64), ex, rtol=1.2e-7,
                               atol=1.2e-7 * np.abs(ex).max())


def _sampled_rows(H):
    """First rows, a spread of interior rows and the last rows."""
    rows = set(range(3)) | set(range(H - 3, H)) | set(np.linspace(0, H - 1, 40).astype(int))
    return sorted(rows)


@pytest.mark.parametrize("H,W,nch", [(7300, 7300, 1), (5100, 5100, 2)])
def test_no_alloc_near_its_scratch_limit(ocip, ctx, H, W, nch):
    """Images whose scratch nearly fills the fixed array: exact U8 sums of
    squares into F64, equal to the oracle on sampled rows (the last row and
    column included), then a second call on the same array."""
    ctx.make_current()
    rng = np.random.default_rng(H + nch)
    shape = (H, W) if nch == 1 else (H, W, nch)
    S = rng.integers(0, 256, shape, dtype=np.uint8)
    got = _no_alloc(ocip, ctx, S, True, np.float64)
    ex = O.integral_exact(S, True)
    rows = _sampled_rows(H)
    assert np.array_equal(got[rows], ex[rows])
    assert np.array_equal(got[:, -1], ex[:, -1])
    # second call on the same scratch, the plain sums
    got2 = _no_alloc(ocip, ctx, S, False, np.float64)
    ex2 = O.integral_exact(S, False)
    assert np.array_equal(got2[rows], ex2[rows])
    assert np.array_equal(got2[:, -1], ex2[:, -1])


def test_no_alloc_refuses_images_beyond_its_scratch(ocip, ctx):
    ctx.make_current()
    desc = ocip.SImage(8192, 8192, 8192, 1, ocip.U8)
    dst = ocip.SImage(8192, 8192, 8192 * 8, 1, ocip.F64)
    # refused on the host before any device work: the pointers are never used
    rc = ocip.lib.ocipIntegralNoAlloc(1, desc, ctypes.c_void_p(16), 8192, dst,
                                      ctypes.c_void_p(16), 8192 * 8, None)
    assert rc == ocip.CL_INVALID_IMAGE_SIZE
    assert b"fixed limit" in ocip.lib.ocipGetLastErrorMessage()
