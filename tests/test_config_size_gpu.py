"""Parity at the configurations' full sizes, through the C ABI.

The other GPU tests pin every path on small images against the oracle; these
run the benchmark configurations at full size and check full-width rows of
the maps (spread over the map, plus the rows around the match) against the
exact oracle:

  * 4096x4096 F32 blob field, 31x31 template (tensor path): per-output
    relative error <= 1e-5 for CrossCorr[_Norm] (non-negative data), and
    within 1e-5 of the scale of the cancelling terms for SqrDistance[_Norm];
  * the same field made zero-mean (signed data): a dot product that cancels
    has no per-output relative bound, so the bar is 1e-5 of sum |S||T| (over
    sqrt(sum S^2 sum T^2) for CrossCorr_Norm);
  * 16 x 2048x2048 U8 batch config: all 64 templates (sides 8-64) against one
    full image in one batch, bit-exact against the integer oracle on sampled
    rows;
  * 32 x 1024x1024 F32 differentiation config: one full-size pair, gradients
    against FP64 central finite differences (h = 1e-3) on 64 seeded
    coordinates, relative error per coordinate <= 1e-4;
  * 3840x2160x4 U8, 64x64x4 template: the _Norm maps against the exact
    oracle (exact integer sums rounded once).
"""
import numpy as np
import pytest

import bench
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MEAS = bench.MEAS_ALL
TOL = 1e-5


def maps_of(ocip, ctx, path, measures, S, T, out_dtype=np.float32):
    maps, used = bench._run_maps(ocip, ctx, path, measures, S, T, out_dtype)
    ctx.set_path(ocip.PATH_PLAIN)
    return maps, used


@pytest.fixture(scope="module")
def cfg2():
    S, T, off = bench.workload(seed=1234, with_offset=True)
    return S, T, off


def test_cfg2_full_size_rows_and_match(ocip, ctx, cfg2):
    ctx.make_current()
    S, T, (ty, tx) = cfg2
    rows = bench.check_rows(S.shape[0], T.shape[0], n=64, match_row=ty + 15)
    meas = ["SqrDistance", "SqrDistance_Norm", "CrossCorr", "CrossCorr_Norm"]
    maps, used = maps_of(ocip, ctx, ocip.PATH_TENSOR, meas, S, T)
    for m in meas:
        assert used[m] == "tensor"
        e = bench.error_rows(MEAS.index(m), S, T, maps[m], rows)
        if m.startswith("CrossCorr"):
            assert e["max_rel"] <= TOL, (m, e)
        else:
            assert e["max_scaled"] <= TOL, (m, e)
    # the best match is where the template was cut
    cc = maps["CrossCorr_Norm"]
    assert np.unravel_index(np.nanargmax(cc), cc.shape) == (ty + 15, tx + 15)
    sq = maps["SqrDistance"]
    assert np.unravel_index(np.argmin(sq), sq.shape) == (ty + 15, tx + 15)


def test_cfg2_zero_mean_signed_rows(ocip, ctx, cfg2):
    ctx.make_current()
    S, _, (ty, tx) = cfg2
    S0 = (S - np.float32(S.mean(dtype=np.float64))).astype(np.float32)
    T0 = S0[ty:ty + 31, tx:tx + 31].copy()
    rows = bench.check_rows(S.shape[0], 31, n=32, match_row=ty + 15)
    meas = ["SqrDistance", "SqrDistance_Norm", "CrossCorr", "CrossCorr_Norm"]
    maps, used = maps_of(ocip, ctx, ocip.PATH_TENSOR, meas, S0, T0)
    for m in meas:
        assert used[m] == "tensor"
        e = bench.error_rows(MEAS.index(m), S0, T0, maps[m], rows)
        assert e["max_scaled"] <= TOL, (m, e)


def test_cfg3_full_image_all_64_templates(ocip, ctx):
    """One full 2048x2048 U8 image of the batch config against all 64
    templates in one batch per measure; sampled rows of every map (first and
    last rows included) equal the integer oracle."""
    ctx.make_current()
    imgs, tmpls = bench.batch_workload()
    S = imgs[0]
    Si = ocip.Image(S)
    Ti = [ocip.Image(t) for t in tmpls]
    rows = sorted({0, 1, 1000, 2046, 2047} | set(np.linspace(0, 2047, 6).astype(int).tolist()))
    try:
        for m in ("CrossCorr", "SqrDistance"):
            outs = [np.zeros(S.shape, np.float32) for _ in tmpls]
            Ds = [ocip.Image(o) for o in outs]
            b = ocip.prepare_batch(m, [Si], Ti, Ds)
            ocip.check(b.run(), "ocipRunProximityBatch")
            for D in Ds:
                D.read()
            b.release()
            for D in Ds:
                D.release()
            for j, t in enumerate(tmpls):
                ex = O.proximity_exact_rows(m, S, t, rows).astype(np.float32)
                assert np.array_equal(outs[j][rows], ex), (m, j, t.shape)
    finally:
        Si.release()
        for t in Ti:
            t.release()


def gpu_gradients(ocip, S, T, G1, G2):
    """dL/dS and dL/dT from ocipProximityBackward (the CrossCorr_Norm map it
    needs comes from the forward call)."""
    Si, Ti, g1, g2 = ocip.Image(S), ocip.Image(T), ocip.Image(G1), ocip.Image(G2)
    n2 = ocip.Image(np.zeros(S.shape, np.float32))
    dS, dT = np.zeros(S.shape, np.float32), np.zeros(T.shape, np.float32)
    dSi, dTi = ocip.Image(dS), ocip.Image(dT)
    try:
        ocip.check(ocip.cross_corr_norm(Si, Ti, n2), "forward")
        ocip.check(ocip.proximity_backward(Si, Ti, g1, g2, n2, dSi, dTi), "ocipProximityBackward")
        dSi.read()
        dTi.read()
    finally:
        for k in (Si, Ti, g1, g2, n2, dSi, dTi):
            k.release()
    return dS, dT


def _fd_loss_parts(S, T, G1, G2):
    """FP64 maps of the forward: C = sum S T (exact oracle), E_S (window sums
    of S^2), E_T."""
    S64, T64 = S.astype(np.float64), T.astype(np.float64)
    C = O.proximity_exact(3, S, T)
    E = bench.window_energy_rows(S, T.shape[1], T.shape[0], list(range(S.shape[0])))
    return S64, T64, C, E, float((T64 ** 2).sum())


def _loss(G1, G2, C, E, et):
    return float((G1 * (E - 2 * C + et)).sum() + (G2 * (C / np.sqrt(E * et))).sum())


def test_cfg4_full_size_finite_differences_per_coordinate(ocip, ctx):
    """1024x1024 blob field with a 32x32 template (its crop + N(0, 0.02)),
    upstream gradients N(0, 1): dL/dS and dL/dT of
    L = sum G1 SqrDistance + sum G2 CrossCorr_Norm from the C ABI against
    FP64 central differences with h = 1e-3 at 32 image and 32 template
    coordinates. A perturbed pixel changes C and the window energies only
    where its windows reach, so L(+h) and L(-h) are evaluated exactly from the
    FP64 maps updated there.

    Bar, per coordinate: |g - fd| <= 1e-4 |fd| + 8 u sum|terms|, where
    sum|terms| is the sum of the magnitudes of the terms the gradient adds up
    and u = 2^-24 the FP32 rounding unit; and at least 60 of the 64
    coordinates within 1e-4 relative alone. The second term matters only
    where the gradient cancels: an image coordinate whose gradient is 1/2800
    of its terms (kappa = sum|terms| / |g| = 2800) is below the resolution
    of FP32 values of those terms at 1e-4, in any FP32 evaluation order (and
    the FP64 central difference itself, with its O(h^2) truncation, is only
    good to ~1e-4 there)."""
    ctx.make_current()
    ctx.set_path(ocip.PATH_TENSOR)
    rng = np.random.default_rng(4)
    H = W = 1024
    th = tw = 32
    S = bench.blob_field(W, H, nblobs=60, seed=400)
    y, x = (int(v) for v in rng.integers(0, H - th, 2))
    T = (S[y:y + th, x:x + tw] + rng.normal(0, 0.02, (th, tw))).astype(np.float32)
    G1 = rng.standard_normal((H, W)).astype(np.float32)
    G2 = rng.standard_normal((H, W)).astype(np.float32)
    dS, dT = gpu_gradients(ocip, S, T, G1, G2)
    ctx.set_path(ocip.PATH_PLAIN)
    S64, T64, C, E, et = _fd_loss_parts(S, T, G1, G2)
    g1, g2 = G1.astype(np.float64), G2.astype(np.float64)
    h = 1e-3
    ax, ay = tw // 2, th // 2
    rows = []  # (tensor, coordinate, fd, gpu, kappa)
    for _ in range(32):
        py, px = int(rng.integers(0, H)), int(rng.integers(0, W))
        # outputs whose window holds (px, py)
        x0, x1 = max(0, px + ax - tw + 1), min(W - 1, px + ax)
        y0, y1 = max(0, py + ay - th + 1), min(H - 1, py + ay)
        ys, xs = np.mgrid[y0:y1 + 1, x0:x1 + 1]
        tv = T64[py - ys + ay, px - xs + ax]
        c, e = C[y0:y1 + 1, x0:x1 + 1], E[y0:y1 + 1, x0:x1 + 1]
        G1l, G2l = g1[y0:y1 + 1, x0:x1 + 1], g2[y0:y1 + 1, x0:x1 + 1]
        s = S64[py, px]
        Lp = _loss(G1l, G2l, c + h * tv, e + 2 * h * s + h * h, et)
        Lm = _loss(G1l, G2l, c - h * tv, e - 2 * h * s + h * h, et)
        fd = (Lp - Lm) / (2 * h)
        # terms of dL/dS(p): 2 G1 (S(p) - T), G2 (T - N S(p) / E_S) / sqrt(E_S E_T)
        q = np.sqrt(e * et)
        mag = (np.abs(2 * G1l * s) + np.abs(2 * G1l * tv) + np.abs(G2l * tv / q) +
               np.abs(G2l * (c / q) * s / e)).sum()
        rows.append(("S", (py, px), fd, float(dS[py, px]), mag / abs(fd)))
    Sp = np.pad(S64, ((th, th), (tw, tw)))
    q = np.sqrt(E * et)
    for _ in range(32):
        kh, kw = int(rng.integers(0, th)), int(rng.integers(0, tw))
        # C(x, y) gains h S(x + kw - ax, y + kh - ay) (zero outside)
        shift = Sp[th + kh - ay:th + kh - ay + H, tw + kw - ax:tw + kw - ax + W]
        t = T64[kh, kw]
        Lp = _loss(g1, g2, C + h * shift, E, et + 2 * h * t + h * h)
        Lm = _loss(g1, g2, C - h * shift, E, et - 2 * h * t + h * h)
        fd = (Lp - Lm) / (2 * h)
        mag = (np.abs(2 * g1 * shift) + np.abs(2 * g1 * t) + np.abs(g2 * shift / q) +
               np.abs(g2 * (C / q) * t / et)).sum()
        rows.append(("T", (kh, kw), fd, float(dT[kh, kw]), mag / abs(fd)))
    u = 2.0 ** -24
    for name, coord, fd, g, kappa in rows:
        err = abs(g - fd)
        assert err <= 1e-4 * abs(fd) + 8 * u * kappa * abs(fd), (name, coord, fd, g, kappa)
    within = sum(1 for r in rows if abs(r[3] - r[2]) <= 1e-4 * abs(r[2]))
    assert within >= 60, f"only {within} of 64 coordinates within 1e-4 relative"


def test_cfg5_u8_full_size_against_oracle(ocip, ctx):
    """3840x2160x4 U8 with a 64x64x4 template on the tensor path: the _Norm
    maps are the exact integer sums with one final rounding, so each output is
    within one F32 rounding of the exact oracle."""
    ctx.make_current()
    S, T, (y5, _) = bench.cfg5_images(np.uint8)
    rows = sorted({0, 1, 2158, 2159, y5 + 32} | set(np.linspace(32, 2127, 5).astype(int).tolist()))
    maps, used = maps_of(ocip, ctx, ocip.PATH_AUTO, ["SqrDistance_Norm", "CrossCorr_Norm"], S, T)
    for m, got in maps.items():
        assert used[m] == "tensor"
        ex = O.proximity_exact_rows(m, S, T, rows)
        g = got[rows].astype(np.float64)
        fin = np.isfinite(ex)
        assert np.array_equal(np.isfinite(g), fin), m
        err = np.abs(g[fin] - ex[fin])
        assert (err <= 6e-8 * np.abs(ex[fin]) + 1e-30).all(), (m, float(err.max()))
