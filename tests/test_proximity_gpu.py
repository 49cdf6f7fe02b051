"""ImageProximity on the GPU, through the C ABI, against the oracle.

Bars (see the plain kernel's header comment for why they hold):
  * F32 / F64 sources: bit-identical to the reference kernel source with every
    acc += a*b contracted to one fma (tests/golden, oracle fused form);
  * 8/16-bit integer sources: bit-identical to the exact integer value rounded
    once to F32 (for the _Norm measures, within 2 ulp of the exact ratio);
  * 32-bit integer sources: double accumulation, within 1e-12 relative.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MEAS = ["SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr", "CrossCorr_Norm"]


def run(ocip, measure, S, T, out_dtype=None):
    return ocip.match(MEAS[measure], S, T, out_dtype)


def ulp_diff32(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, np.int64(-2**31) - a, a)
    b = np.where(b < 0, np.int64(-2**31) - b, b)
    return np.abs(a - b)


def check_against_oracle(got, S, T, m, fixture_fma=None):
    kind = S.dtype
    if kind in (np.float32, np.float64):
        ref = fixture_fma if fixture_fma is not None else O.proximity_refexact(m, S, T, fused=True)
        assert got.dtype == ref.dtype
        assert np.array_equal(got, ref, equal_nan=True), \
            f"max diff {np.nanmax(np.abs(got.astype(np.float64) - ref))}"
        return
    ex = O.proximity_exact(m, S, T)
    if kind in (np.uint32, np.int32):
        fin = np.isfinite(ex)
        np.testing.assert_allclose(got[fin].astype(np.float64), ex[fin], rtol=1e-6)
        return
    want = ex.astype(np.float32)
    if m in (1, 4):
        fin = np.isfinite(want)
        assert np.array_equal(np.isfinite(got), fin)
        assert ulp_diff32(got[fin], want[fin]).max() <= 2
    else:
        assert np.array_equal(got, want)


def test_golden_matrix_plain(ocip, plain):
    """Every fixture case: 8 types x {1,2,4} channels x 5 measures x shapes."""
    z = np.load(os.path.join(GOLDEN, "proximity.npz"))
    keys = sorted({k.split("_")[0] for k in z.files})
    for k in keys:
        S, T = z[k + "_S"], z[k + "_T"]
        for m in range(5):
            got = run(ocip, m, S, T)
            check_against_oracle(got, S, T, m, fixture_fma=z[f"{k}_m{m}_fma"]
                                 if S.dtype.kind == "f" else None)


def test_u8_matches_reference_bit_exact(ocip, plain):
    """cfg-1 shape: 512x512 U8, 16x16 template cut from it with noise; the
    integer-valued measures are exact and equal the reference's own output."""
    rng = np.random.default_rng(1)
    S = rng.integers(0, 256, (512, 512), dtype=np.uint8)
    y, x = 100, 200
    T = np.clip(S[y:y + 16, x:x + 16].astype(np.int32) + np.round(rng.normal(0, 4, (16, 16))),
                0, 255).astype(np.uint8)
    for m in range(5):
        got = run(ocip, m, S, T)
        ref = O.proximity_reference(m, S, T) if O.ref_available() else \
            O.proximity_refexact(m, S, T)
        assert np.array_equal(got, ref, equal_nan=True), MEAS[m]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("tw,th", [(31, 31), (8, 3), (33, 17), (1, 40)])
def test_float_bit_exact_random_shapes(ocip, plain, dtype, tw, th):
    rng = np.random.default_rng(tw * 100 + th)
    S = rng.random((300, 277)).astype(dtype)
    T = rng.random((th, tw)).astype(dtype)
    for m in range(5):
        check_against_oracle(run(ocip, m, S, T), S, T, m)


def test_tall_template_uses_row_bands(ocip, plain):
    """A template too tall for one shared-memory band is processed in bands;
    results stay bit-exact."""
    rng = np.random.default_rng(5)
    S = rng.random((300, 200)).astype(np.float32)
    T = rng.random((250, 60)).astype(np.float32)
    for m in (0, 3, 4):
        check_against_oracle(run(ocip, m, S, T), S, T, m)


@pytest.mark.parametrize("nch", [2, 3, 4])
@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32])
def test_multichannel(ocip, plain, nch, dtype):
    rng = np.random.default_rng(nch)
    if dtype == np.float32:
        S = rng.random((50, 61, nch)).astype(dtype)
        T = rng.random((9, 12, nch)).astype(dtype)
    else:
        hi = 256 if dtype == np.uint8 else 65536
        S = rng.integers(0, hi, (50, 61, nch)).astype(dtype)
        T = rng.integers(0, hi, (9, 12, nch)).astype(dtype)
    for m in range(5):
        check_against_oracle(run(ocip, m, S, T), S, T, m)


def test_large_u8_template_exact_beyond_float(ocip, plain):
    """64x64 U8: sums exceed 2^24, where the reference's float accumulation
    rounds; the result here is the exact integer rounded once."""
    rng = np.random.default_rng(9)
    S = rng.integers(0, 256, (130, 140), dtype=np.uint8)
    T = rng.integers(0, 256, (64, 64), dtype=np.uint8)
    for m in (0, 2, 3):
        got = run(ocip, m, S, T)
        assert np.array_equal(got, O.proximity_exact(m, S, T).astype(np.float32))


def test_host_step_larger_than_row(ocip, plain):
    rng = np.random.default_rng(11)
    big = rng.random((40, 64)).astype(np.float32)
    S = big[:, :50]  # row step 256 bytes, 50 pixels wide
    T = rng.random((5, 6)).astype(np.float32)
    Si = ocip.Image(S, step=S.strides[0])
    Ti = ocip.Image(np.ascontiguousarray(T))
    out = np.zeros((40, 50), np.float32)
    Di = ocip.Image(out)
    ocip.cross_corr(Si, Ti, Di)
    Di.read()
    check_against_oracle(out, np.ascontiguousarray(S), T, 3)


def test_f64_destination_for_f32_source(ocip, plain):
    rng = np.random.default_rng(12)
    S = rng.random((30, 40)).astype(np.float32)
    T = rng.random((4, 5)).astype(np.float32)
    got = run(ocip, 3, S, T, out_dtype=np.float64)
    ref = O.proximity_refexact(3, S, T, fused=True).astype(np.float64)
    assert np.array_equal(got, ref)


def test_error_codes_follow_reference_order(ocip, plain):
    u8 = np.zeros((10, 10), np.uint8)
    f32 = np.zeros((10, 10), np.float32)
    S = ocip.Image(u8)
    big = ocip.Image(np.zeros((11, 10), np.uint8))
    T16 = ocip.Image(np.zeros((3, 3), np.uint16))
    T = ocip.Image(np.zeros((3, 3), np.uint8))
    D = ocip.Image(f32)
    D_small = ocip.Image(np.zeros((9, 10), np.float32))
    D_u8 = ocip.Image(np.zeros((10, 10), np.uint8))
    D_2ch = ocip.Image(np.zeros((10, 10, 2), np.float32))
    for name in MEAS:
        assert ocip.proximity(name, S, big, D) == ocip.CL_INVALID_VALUE          # template > source
        assert ocip.proximity(name, S, T16, D) == ocip.CL_INVALID_VALUE          # type mismatch
        assert ocip.proximity(name, S, T, D_small) == ocip.CL_INVALID_IMAGE_SIZE  # size
        assert ocip.proximity(name, S, T, D_2ch) == ocip.CL_INVALID_VALUE        # channels
        assert ocip.proximity(name, S, T, D_u8) == ocip.CL_INVALID_VALUE         # non-float dest
        # first failing check wins: size is checked after type
        assert ocip.proximity(name, S, T16, D_small) == ocip.CL_INVALID_VALUE
        assert ocip.proximity(name, S, T, D) == ocip.CL_SUCCESS
    import ctypes
    bogus = ctypes.c_void_p(0)
    assert ocip.lib.ocipCrossCorr(S.handle, bogus, D.handle) == ocip.CL_INVALID_MEM_OBJECT


def test_fft_named_entry_points(ocip, plain):
    """ocip*FFT: same measures, the FFT path's own check order and codes
    (C++/programs/ImageProximityFFT.cpp:112-210)."""
    rng = np.random.default_rng(13)
    S = rng.random((64, 70)).astype(np.float32)
    T = rng.random((20, 21)).astype(np.float32)
    Si, Ti = ocip.Image(S), ocip.Image(T)
    out = np.zeros_like(S)
    Di = ocip.Image(out)
    prog = ocip.prepare_proximity_fft(Si, Ti)
    fns = {"SqrDistanceFFT": 0, "SqrDistanceFFT_Norm": 1, "CrossCorrFFT": 3, "CrossCorrFFT_Norm": 4}
    for name, m in fns.items():
        rc = getattr(ocip.lib, "ocip" + name)(prog.handle, Si.handle, Ti.handle, Di.handle)
        assert rc == 0
        Di.read()
        ex = O.proximity_exact(m, S, T)
        scale = np.abs(ex).max()
        assert np.max(np.abs(out - ex)) <= 1e-5 * scale
    big = ocip.Image(np.zeros((65, 70), np.float32))
    assert ocip.lib.ocipCrossCorrFFT(prog.handle, Si.handle, big.handle, Di.handle) == \
        ocip.CL_IMAGE_FORMAT_NOT_SUPPORTED
    T64 = ocip.Image(np.zeros((3, 3), np.float64))
    assert ocip.lib.ocipCrossCorrFFT(prog.handle, Si.handle, T64.handle, Di.handle) == \
        ocip.CL_IMAGE_FORMAT_MISMATCH
    prog.release()


def test_reads_overlap_later_kernels(ocip, ctx):
    """Five maps queued, then read one by one: each read waits only for its own
    writer (later kernels still run), and every map equals a lone call's."""
    ctx.make_current()
    ctx.set_path(ocip.PATH_AUTO)
    try:
        rng = np.random.default_rng(5)
        S = rng.random((700, 900)).astype(np.float32)
        T = S[100:131, 200:231].copy()
        Si, Ti = ocip.Image(S), ocip.Image(T)
        outs = [np.zeros(S.shape, np.float32) for _ in MEAS]
        Ds = [ocip.Image(o) for o in outs]
        for rep in range(2):
            for o in outs:
                o[:] = np.nan
            for m, D in zip(MEAS, Ds):
                ocip.check(ocip.proximity(m, Si, Ti, D), m)
            for D in Ds:
                D.read()
            for m, o in zip(MEAS, outs):
                assert np.array_equal(o, ocip.match(m, S, T), equal_nan=True), (rep, m)
        for D in Ds:
            D.release()
        Si.release()
        Ti.release()
    finally:
        ctx.set_path(ocip.PATH_PLAIN)
