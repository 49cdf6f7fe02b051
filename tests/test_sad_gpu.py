"""AbsDistance of 8-bit sources (U8, S8): the packed-byte SAD kernel against
the oracle.

Every |S - T| of an 8-bit source is an integer in [0, 255], so the kernel's
uint32 sums are exact; the result must equal the exact sum rounded once to
the destination type (bit-identical), for every template width (the last
4/8-byte chunk is masked), image width (right-edge tiles), channel count and
destination type. Templates too large for the kernel's shared memory go to
the plain kernel, with the same results.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def exact_abs(S, T, out_dtype):
    return O.proximity_exact(2, S, T).astype(out_dtype)


def rand8(rng, shape, dtype):
    info = np.iinfo(dtype)
    return rng.integers(info.min, int(info.max) + 1, shape).astype(dtype)


@pytest.mark.parametrize("dtype", [np.uint8, np.int8])
@pytest.mark.parametrize("tw", [1, 3, 4, 5, 7, 8, 9, 15, 17, 31, 33])
def test_template_widths(ocip, plain, tw, dtype):
    rng = np.random.default_rng(700 + tw)
    S = rand8(rng, (77, 301), dtype)
    T = rand8(rng, (6, tw), dtype)
    got = ocip.match("AbsDistance", S, T)
    assert np.array_equal(got, exact_abs(S, T, np.float32))


@pytest.mark.parametrize("dtype", [np.uint8, np.int8])
@pytest.mark.parametrize("W,H,tw,th", [(1, 1, 1, 1), (256, 32, 16, 16), (257, 33, 16, 16),
                                       (600, 70, 31, 31), (40, 300, 7, 40)])
def test_image_edges(ocip, plain, W, H, tw, th, dtype):
    rng = np.random.default_rng(W * 1000 + H)
    S = rand8(rng, (H, W), dtype)
    T = rand8(rng, (th, tw), dtype)
    got = ocip.match("AbsDistance", S, T)
    assert np.array_equal(got, exact_abs(S, T, np.float32))


@pytest.mark.parametrize("dtype", [np.uint8, np.int8])
@pytest.mark.parametrize("nch", [2, 4])
def test_channels_and_f64_destination(ocip, plain, nch, dtype):
    rng = np.random.default_rng(40 + nch)
    S = rand8(rng, (45, 270, nch), dtype)
    T = rand8(rng, (11, 13, nch), dtype)
    assert np.array_equal(ocip.match("AbsDistance", S, T), exact_abs(S, T, np.float32))
    assert np.array_equal(ocip.match("AbsDistance", S, T, np.float64),
                          exact_abs(S, T, np.float64))


def overlap(n, t):
    """Window pixels inside [0, n) for each output of a length-n axis and a
    t-long window anchored at -(t // 2)."""
    x = np.arange(n)[:, None] + np.arange(t)[None, :] - t // 2
    return ((x >= 0) & (x < n)).sum(axis=1)


@pytest.mark.parametrize("H,W,th,tw", [(70, 1000, 66, 1000), (310, 330, 300, 300)])
def test_all_terms_255_and_sums_beyond_float(ocip, plain, H, W, th, tw):
    """An all-255 image against an all-0 template makes every in-image term
    255, so the exact map is 255 x (window pixels inside the image). Both
    cases sum past 2^24, where float accumulation would round: 66 x 1000 runs
    on the SAD kernel, 300 x 300 exceeds its shared memory and runs on the
    plain kernel."""
    S = np.full((H, W), 255, np.uint8)
    T = np.zeros((th, tw), np.uint8)
    want = (255.0 * overlap(H, th)[:, None] * overlap(W, tw)[None, :])
    assert want.max() > 2**24
    got = ocip.match("AbsDistance", S, T)
    assert np.array_equal(got, want.astype(np.float32))


def test_s8_extremes(ocip, plain):
    """-128 against 127 gives the largest signed term, 255, in every tap."""
    S = np.full((40, 300), -128, np.int8)
    S[:, 1::2] = 127
    T = np.full((9, 21), 127, np.int8)
    T[::2] = -128
    got = ocip.match("AbsDistance", S, T)
    assert np.array_equal(got, exact_abs(S, T, np.float32))


def test_matches_reference_kernel(ocip, plain):
    """The cfg-1 shape (512x512, 16x16 template) equals the reference's own
    kernel source compiled for the host."""
    rng = np.random.default_rng(11)
    S = rng.integers(0, 256, (512, 512), dtype=np.uint8)
    T = np.clip(S[40:56, 300:316].astype(np.int32) + rng.integers(-8, 9, (16, 16)),
                0, 255).astype(np.uint8)
    got = ocip.match("AbsDistance", S, T)
    ref = O.proximity_reference(2, S, T) if O.ref_available() else exact_abs(S, T, np.float32)
    assert np.array_equal(got, ref)
