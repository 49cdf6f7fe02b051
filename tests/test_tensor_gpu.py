"""Tensor-core (tcgen05) ImageProximity path, through the C ABI.

Bars:
  * U8 sources (i8 MMA, exact s32 sums, exact window statistics): results are
    bit-identical to the plain path, which equals the reference wherever the
    reference's float sums are exact;
  * F32 and U16 sources (split BF16 hi/lo, three MMAs, FP64 window
    statistics): relative error <= 1e-5 against the long-double oracle for
    CrossCorr and CrossCorr_Norm; SqrDistance[_Norm] (which cancel to 0 at a
    match) within 1e-5 of the scale of their terms, sum S^2 + sum T^2 of the
    window (divided by sqrt(sum S^2 * sum T^2) for the _Norm form);
  * 2-4 channel sources: the same bars per channel (the channels are split
    into planes and run as one launch).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

MEAS = ["SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr", "CrossCorr_Norm"]
TOL = 1e-5


def run(ocip, ctx, m, S, T, path, out_dtype=None):
    ctx.set_path(path)
    got = ocip.match(MEAS[m], S, T, out_dtype)
    return got, ctx.last_path()


def f32_check(got, S, T, m):
    ex = O.proximity_exact(m, S, T)
    if m in (0, 1):
        # SqrDistance[_Norm] cancel to 0 at a match: error relative to the
        # scale of the terms, (sum S^2 + sum T^2) [/ sqrt(sum S^2 * sum T^2)].
        ss, _, tt = O.window_terms_exact(S, T)
        tt = tt if S.ndim == 3 else tt[0]
        scale = ss + tt
        if m == 1:
            scale = scale / np.sqrt(ss * tt)
        fin = np.isfinite(scale)
        err = np.abs(got[fin] - ex[fin]) / np.maximum(scale[fin], 1e-30)
    else:
        fin = np.isfinite(ex)
        assert np.array_equal(np.isfinite(got), fin)
        err = np.abs(got[fin] - ex[fin]) / np.maximum(np.abs(ex[fin]), 1e-30)
    assert err.max() <= TOL, f"{MEAS[m]}: max rel err {err.max():.3g}"
    return float(err.max())


@pytest.mark.parametrize("th,tw", [(31, 31), (16, 16), (1, 1), (3, 7), (17, 40), (32, 32),
                                   (64, 64), (64, 5), (9, 64)])
def test_u8_tensor_equals_plain(ocip, ctx, th, tw):
    ctx.make_current()
    rng = np.random.default_rng(th * 100 + tw)
    S = rng.integers(0, 256, (150, 301), dtype=np.uint8)
    T = rng.integers(0, 256, (th, tw), dtype=np.uint8)
    for m in (0, 1, 3, 4):
        plain, p1 = run(ocip, ctx, m, S, T, ocip.PATH_PLAIN)
        tens, p2 = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
        assert p1 == ocip.PATH_PLAIN and p2 == ocip.PATH_TENSOR
        assert np.array_equal(plain, tens, equal_nan=True), MEAS[m]
        # and against the exact oracle directly: integer scores bit-exact, the
        # _Norm ratios within 2 FP32 rounding units of the exact value
        ex = O.proximity_exact(m, S, T)
        if m in (0, 3):
            assert np.array_equal(tens, ex.astype(np.float32)), MEAS[m]
        else:
            fin = np.isfinite(ex) & (ex != 0)
            assert np.array_equal(np.isnan(tens), np.isnan(ex.astype(np.float32))), MEAS[m]
            rel = np.abs(tens[fin].astype(np.float64) - ex[fin]) / np.abs(ex[fin])
            assert rel.max() <= 2.0 ** -22, MEAS[m]
    ctx.set_path(ocip.PATH_PLAIN)


def test_u8_cfg1_exact_against_reference(ocip, ctx):
    """512x512 U8, 16x16 template cut with noise: tensor path == reference."""
    ctx.make_current()
    rng = np.random.default_rng(1)
    S = rng.integers(0, 256, (512, 512), dtype=np.uint8)
    T = np.clip(S[100:116, 200:216].astype(np.int32) + np.round(rng.normal(0, 4, (16, 16))),
                0, 255).astype(np.uint8)
    for m in (0, 1, 3, 4):
        got, path = run(ocip, ctx, m, S, T, ocip.PATH_AUTO)
        assert path == ocip.PATH_TENSOR
        ref = O.proximity_reference(m, S, T) if O.ref_available() else O.proximity_refexact(m, S, T)
        assert np.array_equal(got, ref, equal_nan=True), MEAS[m]
    ctx.set_path(ocip.PATH_PLAIN)


def test_u8_tall_image_many_bands(ocip, ctx):
    """Enough rows for several bands per strip; exact integer results."""
    ctx.make_current()
    rng = np.random.default_rng(2)
    S = rng.integers(0, 256, (2600, 140), dtype=np.uint8)
    T = rng.integers(0, 256, (24, 24), dtype=np.uint8)
    got, path = run(ocip, ctx, 3, S, T, ocip.PATH_TENSOR)
    assert path == ocip.PATH_TENSOR
    assert np.array_equal(got, O.proximity_exact(3, S, T).astype(np.float32))
    ctx.set_path(ocip.PATH_PLAIN)


@pytest.mark.parametrize("th,tw", [(31, 31), (16, 16), (8, 8), (17, 40), (32, 32),
                                   (64, 64), (40, 9), (2, 64)])
def test_f32_tensor_accuracy(ocip, ctx, th, tw):
    ctx.make_current()
    rng = np.random.default_rng(th * 7 + tw)
    S = rng.random((130, 263)).astype(np.float32)
    T = rng.random((th, tw)).astype(np.float32)
    for m in (0, 1, 3, 4):
        got, path = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
        assert path == ocip.PATH_TENSOR
        f32_check(got, S, T, m)
    ctx.set_path(ocip.PATH_PLAIN)


def test_f32_blob_field_crop_accuracy(ocip, ctx):
    """The benchmark's data (blob field + noise, template cut from it) on a
    crop: max relative error per measure."""
    import bench
    ctx.make_current()
    S = bench.blob_field(600, 500, nblobs=20, seed=3)
    T = S[200:231, 300:331].copy()
    for m in (0, 1, 3, 4):
        got, path = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
        assert path == ocip.PATH_TENSOR
        f32_check(got, S, T, m)
    ctx.set_path(ocip.PATH_PLAIN)


def test_f32_signed_values(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(4)
    S = rng.standard_normal((97, 200)).astype(np.float32)
    T = rng.standard_normal((12, 13)).astype(np.float32)
    got, _ = run(ocip, ctx, 3, S, T, ocip.PATH_TENSOR)
    ex = O.proximity_exact(3, S, T)
    # with signed data the sum can cancel: compare against the sum of |S*T|
    absref = O.proximity_exact(3, np.abs(S), np.abs(T))
    assert (np.abs(got - ex) / absref).max() <= TOL
    ctx.set_path(ocip.PATH_PLAIN)


def test_fallbacks_to_plain(ocip, ctx):
    """AbsDistance, types without a tensor form, small F32 templates and
    templates wider than 1024 columns are served by the plain path even when
    the tensor path is requested."""
    ctx.make_current()
    rng = np.random.default_rng(5)
    S = rng.random((80, 90)).astype(np.float32)
    T = rng.random((7, 7)).astype(np.float32)
    _, path = run(ocip, ctx, 2, S, T, ocip.PATH_TENSOR)
    assert path == ocip.PATH_PLAIN
    S4 = rng.random((40, 50, 4)).astype(np.float32)
    _, path = run(ocip, ctx, 3, S4, rng.random((5, 5, 4)).astype(np.float32), ocip.PATH_TENSOR)
    assert path == ocip.PATH_PLAIN
    Si16 = rng.integers(-100, 100, (40, 50), dtype=np.int16)
    _, path = run(ocip, ctx, 3, Si16, rng.integers(-9, 9, (9, 9), dtype=np.int16),
                  ocip.PATH_TENSOR)
    assert path == ocip.PATH_PLAIN
    # AUTO keeps U16 (split, not exact) on the plain path
    S16 = rng.integers(0, 65535, (40, 50), dtype=np.uint16)
    _, path = run(ocip, ctx, 3, S16, rng.integers(0, 65535, (9, 9), dtype=np.uint16),
                  ocip.PATH_AUTO)
    assert path == ocip.PATH_PLAIN
    # templates wider than the row-energy pass takes (1024 columns)
    _, path = run(ocip, ctx, 3, rng.random((12, 1100)).astype(np.float32),
                  rng.random((2, 1030)).astype(np.float32), ocip.PATH_TENSOR)
    assert path == ocip.PATH_PLAIN
    # AUTO keeps F32 on the plain path (not bit-exact on the tensor path)
    _, path = run(ocip, ctx, 3, S, T, ocip.PATH_AUTO)
    assert path == ocip.PATH_PLAIN
    # F32 templates under 64 taps stay on the plain path
    _, path = run(ocip, ctx, 3, S, rng.random((5, 3)).astype(np.float32), ocip.PATH_TENSOR)
    assert path == ocip.PATH_PLAIN
    ctx.set_path(ocip.PATH_PLAIN)


def test_f64_destination(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(6)
    S = rng.integers(0, 256, (64, 140), dtype=np.uint8)
    T = rng.integers(0, 256, (8, 8), dtype=np.uint8)
    got, path = run(ocip, ctx, 0, S, T, ocip.PATH_TENSOR, out_dtype=np.float64)
    assert path == ocip.PATH_TENSOR
    assert np.array_equal(got, O.proximity_exact(0, S, T))
    ctx.set_path(ocip.PATH_PLAIN)


@pytest.mark.parametrize("nch", [2, 3, 4])
@pytest.mark.parametrize("th,tw", [(16, 16), (31, 31), (64, 64), (5, 40)])
def test_u8_multichannel_tensor_equals_plain(ocip, ctx, nch, th, tw):
    ctx.make_current()
    rng = np.random.default_rng(nch * 1000 + th * 10 + tw)
    S = rng.integers(0, 256, (90, 300, nch), dtype=np.uint8)
    T = rng.integers(0, 256, (th, tw, nch), dtype=np.uint8)
    for m in (0, 1, 3, 4):
        plain, p1 = run(ocip, ctx, m, S, T, ocip.PATH_PLAIN)
        tens, p2 = run(ocip, ctx, m, S, T, ocip.PATH_AUTO)
        assert p1 == ocip.PATH_PLAIN and p2 == ocip.PATH_TENSOR
        assert np.array_equal(plain, tens, equal_nan=True), (MEAS[m], nch)
    ctx.set_path(ocip.PATH_PLAIN)


@pytest.mark.parametrize("nch", [1, 4])
@pytest.mark.parametrize("th,tw", [(31, 31), (64, 64), (12, 40), (40, 12)])
def test_u16_tensor_accuracy(ocip, ctx, nch, th, tw):
    ctx.make_current()
    rng = np.random.default_rng(nch * 100 + th + tw)
    shape = (70, 270, nch) if nch > 1 else (70, 270)
    tshape = (th, tw, nch) if nch > 1 else (th, tw)
    S = rng.integers(0, 65536, shape, dtype=np.uint16)
    T = rng.integers(0, 65536, tshape, dtype=np.uint16)
    for m in (0, 1, 3, 4):
        got, path = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
        assert path == ocip.PATH_TENSOR
        f32_check(got, S, T, m)
    ctx.set_path(ocip.PATH_PLAIN)


@pytest.mark.parametrize("nch", [3, 4])
def test_f32_multichannel_accuracy(ocip, ctx, nch):
    ctx.make_current()
    rng = np.random.default_rng(nch)
    S = rng.random((80, 290, nch)).astype(np.float32)
    T = rng.random((20, 24, nch)).astype(np.float32)
    for m in (0, 1, 3, 4):
        got, path = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
        assert path == ocip.PATH_TENSOR
        f32_check(got, S, T, m)
    ctx.set_path(ocip.PATH_PLAIN)


def cfg5_images(dtype):
    """3840x2160x4 field as in the multi-channel config: uniform noise plus a
    blob field (U8), or the field scaled to 0-65535 (U16); 64x64x4 template
    cut at a seeded offset."""
    import bench
    rng = np.random.default_rng(55)
    field = np.stack([bench.blob_field(3840, 2160, nblobs=60, seed=60 + c) for c in range(4)], -1)
    field = field / field.max()
    if dtype == np.uint8:
        S = np.clip(rng.integers(0, 128, field.shape) + 127 * field, 0, 255).astype(np.uint8)
    else:
        S = np.round(field * 65535).astype(np.uint16)
    y, x = 700, 1900
    return S, S[y:y + 64, x:x + 64].copy()


def test_cfg5_u8_full_size_tensor_equals_plain(ocip, ctx):
    """Full-size 3840x2160x4 U8, 64x64x4 template: the tensor path's _Norm maps
    are bit-identical to the plain path's (exact integer sums on both)."""
    ctx.make_current()
    S, T = cfg5_images(np.uint8)
    for m in (1, 4):
        plain, _ = run(ocip, ctx, m, S, T, ocip.PATH_PLAIN)
        tens, path = run(ocip, ctx, m, S, T, ocip.PATH_AUTO)
        assert path == ocip.PATH_TENSOR
        assert np.array_equal(plain, tens, equal_nan=True), MEAS[m]
    ctx.set_path(ocip.PATH_PLAIN)


def test_cfg5_u16_full_size_accuracy_on_crops(ocip, ctx):
    """Full-size 3840x2160x4 U16 on the tensor path, checked against the
    long-double oracle on crops (interior, corner and edges)."""
    ctx.make_current()
    S, T = cfg5_images(np.uint16)
    for m in (1, 4):
        got, path = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
        assert path == ocip.PATH_TENSOR
        for (y, x) in [(700, 1900), (0, 0), (2160 - 48, 3840 - 48), (1000, 0)]:
            # the window of output (y..y+n, x..x+n) needs 64 rows/cols around it
            y0, x0 = max(0, y - 64), max(0, x - 64)
            y1, x1 = min(2160, y + 48 + 64), min(3840, x + 48 + 64)
            crop_ex = O.proximity_exact(m, S[y0:y1, x0:x1], T)
            sub = got[y:y + 48, x:x + 48]
            ex = crop_ex[y - y0:y - y0 + 48, x - x0:x - x0 + 48]
            # crop borders only where the crop is the image border
            if m == 1:
                ss, _, tt = O.window_terms_exact(S[y0:y1, x0:x1], T)
                scale = ((ss + tt) / np.sqrt(ss * tt))[y - y0:y - y0 + 48, x - x0:x - x0 + 48]
                err = np.abs(sub - ex) / scale
            else:
                err = np.abs(sub - ex) / np.abs(ex)
            assert err.max() <= TOL, (MEAS[m], y, x, err.max())
    ctx.set_path(ocip.PATH_PLAIN)


@pytest.mark.parametrize("dtype,th,tw,nch", [(np.float32, 16, 16, 1), (np.float32, 31, 31, 1),
                                             (np.float32, 64, 64, 1), (np.float32, 48, 33, 1),
                                             (np.uint16, 40, 48, 2), (np.uint8, 24, 24, 1),
                                             (np.uint8, 64, 64, 3)])
def test_tall_bands_many_blocks(ocip, ctx, dtype, th, tw, nch):
    """One work item per strip covering all 420 rows: the running sums go
    round their TMEM ring many times and the energy ring is reused many times.
    U8 stays bit-identical to the plain path; F32 and U16 stay within the
    1e-5 bar."""
    ctx.make_current()
    rng = np.random.default_rng(th * 31 + tw + nch)
    H, W = 420, 200 if th > 32 else 300
    shape = (H, W, nch) if nch > 1 else (H, W)
    tshape = (th, tw, nch) if nch > 1 else (th, tw)
    if dtype == np.float32:
        S = rng.random(shape).astype(np.float32)
        T = rng.random(tshape).astype(np.float32)
    else:
        hi = 256 if dtype == np.uint8 else 65536
        S = rng.integers(0, hi, shape, dtype=dtype)
        T = rng.integers(0, hi, tshape, dtype=dtype)
    ctx.set_band_height(H)
    try:
        for m in (0, 1, 3, 4):
            got, path = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
            assert path == ocip.PATH_TENSOR
            if dtype == np.uint8:
                plain, _ = run(ocip, ctx, m, S, T, ocip.PATH_PLAIN)
                assert np.array_equal(plain, got, equal_nan=True), MEAS[m]
            else:
                f32_check(got, S, T, m)
    finally:
        ctx.set_band_height(0)
        ctx.set_path(ocip.PATH_PLAIN)


def test_band_height_does_not_change_results(ocip, ctx):
    """Items of 17, 64 or 150 rows, or the whole image, give the automatic
    choice's maps: bit-identical for U8 (exact sums), within the 1e-5 bar for
    F32 (the blocks of partial sums start at each band's first row). A negative
    height is refused."""
    ctx.make_current()
    rng = np.random.default_rng(23)
    S8 = rng.integers(0, 256, (300, 280), dtype=np.uint8)
    T8 = rng.integers(0, 256, (20, 23), dtype=np.uint8)
    Sf = rng.random((300, 280)).astype(np.float32)
    Tf = rng.random((20, 23)).astype(np.float32)
    try:
        ref8 = {m: run(ocip, ctx, m, S8, T8, ocip.PATH_TENSOR)[0] for m in (0, 3)}
        for rows in (17, 64, 150, 300):
            ctx.set_band_height(rows)
            for m in (0, 3):
                got, path = run(ocip, ctx, m, S8, T8, ocip.PATH_TENSOR)
                assert path == ocip.PATH_TENSOR
                assert np.array_equal(got, ref8[m]), (MEAS[m], rows)
            for m in (1, 4):
                got, _ = run(ocip, ctx, m, Sf, Tf, ocip.PATH_TENSOR)
                f32_check(got, Sf, Tf, m)
        assert ocip.lib.ocipSetProximityBandHeight(-1) == ocip.CL_INVALID_VALUE
    finally:
        ctx.set_band_height(0)
        ctx.set_path(ocip.PATH_PLAIN)


def test_bounded_wait_expires_and_context_stays_usable(ocip, ctx):
    """A kernel waits on a barrier nothing arrives on: the bounded wait
    expires (about 1 ms here), the kernel returns, the error surfaces as
    CL_OUT_OF_RESOURCES at the next synchronisation, and the context keeps
    working."""
    ctx.make_current()
    assert ocip.lib.ocipTestBoundedWait(2_000_000) == ocip.CL_OUT_OF_RESOURCES
    assert ocip.lib.ocipFinish() == 0  # the flag was cleared
    rng = np.random.default_rng(17)
    S = rng.integers(0, 256, (64, 300), dtype=np.uint8)
    T = rng.integers(0, 256, (9, 9), dtype=np.uint8)
    got, path = run(ocip, ctx, 3, S, T, ocip.PATH_TENSOR)
    assert path == ocip.PATH_TENSOR
    assert np.array_equal(got, O.proximity_exact(3, S, T).astype(np.float32))
    ctx.set_path(ocip.PATH_PLAIN)
