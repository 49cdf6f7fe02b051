"""Templates larger than 64 x 64 on the tensor path, through the C ABI.

They run as tiles of at most 64 x 64 whose product sums accumulate in an F64
map, and a scoring pass adds the window and template energies. Bars as for
the one-launch tensor path: U8 bit-identical to the plain path (exact integer
sums, the plain path's final formulas); F32 and U16 within 1e-5 of the
long-double oracle (SqrDistance[_Norm] against the scale of their terms).
The FFT-named entry points, which the reference provides for large
templates, serve them on the tensor path.
"""
import numpy as np
import pytest

import bench
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MEAS = ["SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr", "CrossCorr_Norm"]
TOL = 1e-5


def run(ocip, ctx, m, S, T, path):
    ctx.set_path(path)
    got = ocip.match(MEAS[m], S, T)
    return got, ctx.last_path()


def check_rows(got, S, T, m, rows):
    e = bench.error_rows(m, S, T, got, rows)
    key = "max_scaled" if m in (0, 1) else "max_rel"
    assert e[key] <= TOL, (MEAS[m], e)


@pytest.mark.parametrize("th,tw", [(128, 128), (200, 40), (70, 65), (40, 200)])
def test_f32_large_templates(ocip, ctx, th, tw):
    ctx.make_current()
    S = bench.blob_field(520, 360, nblobs=30, seed=th + tw)
    T = S[100:100 + th, 150:150 + tw].copy()
    rows = sorted({0, 1, 180, 359} | set(np.linspace(0, 359, 8).astype(int).tolist()) |
                  {100 + th // 2})
    for m in (0, 1, 3, 4):
        got, path = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
        assert path == ocip.PATH_TENSOR, MEAS[m]
        check_rows(got, S, T, m, rows)
    ctx.set_path(ocip.PATH_PLAIN)


@pytest.mark.parametrize("th,tw,nch", [(100, 70, 1), (65, 130, 1), (80, 80, 3)])
def test_u8_large_templates_equal_plain(ocip, ctx, th, tw, nch):
    ctx.make_current()
    rng = np.random.default_rng(th * tw + nch)
    shape = (230, 300, nch) if nch > 1 else (230, 300)
    S = rng.integers(0, 256, shape, dtype=np.uint8)
    T = S[40:40 + th, 60:60 + tw].copy()
    for m in (0, 1, 3, 4):
        plain, p1 = run(ocip, ctx, m, S, T, ocip.PATH_PLAIN)
        tens, p2 = run(ocip, ctx, m, S, T, ocip.PATH_AUTO)
        assert p1 == ocip.PATH_PLAIN and p2 == ocip.PATH_TENSOR
        assert np.array_equal(plain, tens, equal_nan=True), MEAS[m]
    # and the integer sums themselves
    got, _ = run(ocip, ctx, 3, S, T, ocip.PATH_TENSOR)
    rows = [0, 57, 229]
    ex = O.proximity_exact_rows(3, S, T, rows).astype(np.float32)
    assert np.array_equal(got[rows], ex)
    ctx.set_path(ocip.PATH_PLAIN)


def test_u16_two_channels_large_template(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(91)
    S = rng.integers(0, 65536, (150, 260, 2), dtype=np.uint16)
    T = S[20:110, 30:120].copy()
    rows = [0, 64, 65, 149]
    for m in (0, 1, 3, 4):
        got, path = run(ocip, ctx, m, S, T, ocip.PATH_TENSOR)
        assert path == ocip.PATH_TENSOR
        check_rows(got, S, T, m, rows)
    ctx.set_path(ocip.PATH_PLAIN)


def test_fft_entry_points_serve_large_templates_on_tensor_cores(ocip, ctx):
    """ocipCrossCorrFFT_Norm and the other FFT-named calls on a 128 x 128 and a
    200 x 40 F32 template: tensor path, within the 1e-5 bar."""
    ctx.make_current()
    S = bench.blob_field(400, 330, nblobs=25, seed=5)
    Si = ocip.Image(S)
    out = np.zeros_like(S)
    Di = ocip.Image(out)
    fns = {"SqrDistanceFFT": 0, "SqrDistanceFFT_Norm": 1, "CrossCorrFFT": 3,
           "CrossCorrFFT_Norm": 4}
    for th, tw in ((128, 128), (200, 40)):
        T = S[60:60 + th, 90:90 + tw].copy()
        Ti = ocip.Image(T)
        prog = ocip.prepare_proximity_fft(Si, Ti)
        rows = [0, 60 + th // 2, 200, 329]
        for name, m in fns.items():
            rc = getattr(ocip.lib, "ocip" + name)(prog.handle, Si.handle, Ti.handle, Di.handle)
            assert rc == 0
            assert ctx.last_path() == ocip.PATH_TENSOR, name
            Di.read()
            check_rows(out, S, T, m, rows)
        prog.release()
        Ti.release()
    Si.release()
    Di.release()
