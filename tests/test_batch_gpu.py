"""Batched matching (ocipPrepareProximityBatch / ocipRunProximityBatch): every
(image, template) pair of a batch in one persistent launch on the tensor path,
replayed from a CUDA graph.

Bars: U8 batches are bit-identical to the one-pair plain path (exact integer
sums on both) and to the exact oracle; F32 batches are within 1e-5 of the
long-double oracle (the tensor path's bar); every replay gives the same maps.
"""
import numpy as np
import pytest

from oracle import oracle as O
from test_tensor_gpu import f32_check

pytestmark = pytest.mark.gpu

MEAS = ["SqrDistance", "SqrDistance_Norm", "AbsDistance", "CrossCorr", "CrossCorr_Norm"]


def run_batch(ocip, measure, srcs, tmpls, out_dtype=np.float32):
    imgs = [ocip.Image(s) for s in srcs]
    tps = [ocip.Image(t) for t in tmpls]
    outs = [np.zeros(s.shape, out_dtype) for s in srcs for _ in tmpls]
    dsts = [ocip.Image(o) for o in outs]
    b = ocip.prepare_batch(measure, imgs, tps, dsts)
    try:
        ocip.check(b.run(), "ocipRunProximityBatch")
        for d in dsts:
            d.read()
        first = [o.copy() for o in outs]
        ocip.check(b.run(), "ocipRunProximityBatch")  # graph replay
        for d in dsts:
            d.read()
        for o, f in zip(outs, first):
            assert np.array_equal(o, f, equal_nan=True)
        info = b.info(tmpls[0].shape[1], tmpls[0].shape[0])
    finally:
        b.release()
        for x in imgs + tps + dsts:
            x.release()
    return outs, info


def test_u8_batch_uneven_templates_equal_plain(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(11)
    srcs = [rng.integers(0, 256, (300, 260), dtype=np.uint8),
            rng.integers(0, 256, (190, 333), dtype=np.uint8)]
    tmpls = [rng.integers(0, 256, (s, s), dtype=np.uint8) for s in (8, 12, 16, 24, 32, 48, 64)]
    tmpls.append(rng.integers(0, 256, (5, 40), dtype=np.uint8))
    for m in (3, 0, 4, 1):
        outs, (nitems, bh) = run_batch(ocip, MEAS[m], srcs, tmpls)
        assert nitems > 0 and bh > 0
        ctx.set_path(ocip.PATH_PLAIN)
        for i, s in enumerate(srcs):
            for j, t in enumerate(tmpls):
                ref = ocip.match(MEAS[m], s, t)
                assert np.array_equal(outs[i * len(tmpls) + j], ref, equal_nan=True), \
                    (MEAS[m], i, t.shape)


def test_u8_batch_exact_against_oracle(ocip, ctx):
    """cfg-3 style at reduced size: templates cut from the images with +-8
    noise; CrossCorr and SqrDistance maps equal the int64 oracle."""
    ctx.make_current()
    rng = np.random.default_rng(12)
    srcs = [rng.integers(0, 256, (256, 256), dtype=np.uint8) for _ in range(3)]
    tmpls = []
    for _ in range(6):
        s = int(rng.choice([8, 12, 16, 24, 32, 48, 64]))
        k = int(rng.integers(0, 3))
        y, x = rng.integers(0, 256 - s, 2)
        t = srcs[k][y:y + s, x:x + s].astype(np.int32) + rng.integers(-8, 9, (s, s))
        tmpls.append(np.clip(t, 0, 255).astype(np.uint8))
    for m in (3, 0):
        outs, _ = run_batch(ocip, MEAS[m], srcs, tmpls)
        for i, s in enumerate(srcs):
            for j, t in enumerate(tmpls):
                ex = O.proximity_exact(m, s, t).astype(np.float32)
                assert np.array_equal(outs[i * len(tmpls) + j], ex), (MEAS[m], i, j)


def test_f32_batch_accuracy(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(13)
    srcs = [rng.random((140, 300)).astype(np.float32), rng.random((140, 300)).astype(np.float32)]
    tmpls = [rng.random((s, s)).astype(np.float32) for s in (9, 31, 64)]
    for m in (3, 4, 0, 1):
        outs, _ = run_batch(ocip, MEAS[m], srcs, tmpls)
        for i, s in enumerate(srcs):
            for j, t in enumerate(tmpls):
                f32_check(outs[i * len(tmpls) + j], s, t, m)


def test_u8_batch_multichannel_equals_plain(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(14)
    srcs = [rng.integers(0, 256, (120, 270, 4), dtype=np.uint8) for _ in range(2)]
    tmpls = [rng.integers(0, 256, (s, s, 4), dtype=np.uint8) for s in (16, 33)]
    outs, _ = run_batch(ocip, "CrossCorr_Norm", srcs, tmpls)
    ctx.set_path(ocip.PATH_PLAIN)
    for i, s in enumerate(srcs):
        for j, t in enumerate(tmpls):
            assert np.array_equal(outs[i * len(tmpls) + j], ocip.match("CrossCorr_Norm", s, t),
                                  equal_nan=True)


def test_batch_f64_destinations(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(15)
    srcs = [rng.integers(0, 256, (64, 300), dtype=np.uint8)]
    tmpls = [rng.integers(0, 256, (10, 10), dtype=np.uint8)]
    outs, _ = run_batch(ocip, "SqrDistance", srcs, tmpls, out_dtype=np.float64)
    assert np.array_equal(outs[0], O.proximity_exact(0, srcs[0], tmpls[0]))


def test_batch_checks(ocip, ctx):
    ctx.make_current()
    rng = np.random.default_rng(16)
    S = ocip.Image(rng.integers(0, 256, (100, 120), dtype=np.uint8))
    T = ocip.Image(rng.integers(0, 256, (9, 9), dtype=np.uint8))
    D = ocip.Image(np.zeros((100, 120), np.float32))
    Dsmall = ocip.Image(np.zeros((90, 120), np.float32))
    Tbig = ocip.Image(rng.integers(0, 256, (65, 65), dtype=np.uint8))
    Tf = ocip.Image(rng.random((9, 9)).astype(np.float32))
    try:
        assert ocip.Batch("AbsDistance", [S], [T], [D]).rc == ocip.CL_INVALID_VALUE
        assert ocip.Batch("CrossCorr", [S], [Tbig], [D]).rc == ocip.CL_INVALID_VALUE
        assert ocip.Batch("CrossCorr", [S], [Tf], [D]).rc == ocip.CL_INVALID_VALUE
        assert ocip.Batch("CrossCorr", [S], [T], [Dsmall]).rc == ocip.CL_INVALID_IMAGE_SIZE
        assert ocip.Batch("CrossCorr", [], [T], [D]).rc == ocip.CL_INVALID_VALUE
        b = ocip.prepare_batch("CrossCorr", [S], [T], [D])
        n0 = ocip.launch_count()
        ocip.check(b.run(), "run")
        ctx.finish()
        assert ocip.launch_count() == n0 + 1  # one persistent kernel per run
        b.release()
    finally:
        for x in (S, T, D, Dsmall, Tbig, Tf):
            x.release()
