"""Row-band split of one image on the GPU, through the C ABI: each part's
band (its source rows plus the template's halo) computed as its own image
gives the whole image's map at the part's rows.

Parts run one after another on one GPU here; on several GPUs each runs in its
own process and context. Bars: plain F32 bit-identical to the whole-image
plain map (same per-output arithmetic), U8 tensor path bit-identical to the
exact oracle, F32 tensor path within 1e-5 relative of it."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def stitched(bands, measure, S, T, parts):
    out = None
    for p in range(parts):
        bm = bands.BandMatch(S, T, p, parts)
        try:
            bm.run(measure)
            rows = bm.owned()
        finally:
            bm.release()
        out = rows if out is None else np.concatenate([out, rows])
    return out


@pytest.mark.parametrize("parts", [1, 2, 3, 5])
def test_plain_f32_bands_equal_the_whole_map(plain, ocip, parts):
    from openclipp_b200 import bands
    rng = np.random.default_rng(parts)
    S = rng.random((301, 257)).astype(np.float32)
    T = S[100:131, 40:71].copy()
    for m in ("CrossCorr_Norm", "SqrDistance", "AbsDistance"):
        whole = ocip.match(m, S, T)
        got = stitched(bands, m, S, T, parts)
        assert np.array_equal(got, whole), m


@pytest.mark.parametrize("parts", [2, 4])
def test_tensor_u8_bands_are_exact(tensor, ocip, parts):
    from openclipp_b200 import bands
    rng = np.random.default_rng(10 + parts)
    S = rng.integers(0, 256, (517, 300), dtype=np.uint8)
    T = S[200:224, 17:41].copy()
    for m in ("CrossCorr", "SqrDistance", "CrossCorr_Norm"):
        got = stitched(bands, m, S, T, parts)
        assert tensor.last_path() == ocip.PATH_TENSOR
        want = ocip.match(m, S, T)
        assert np.array_equal(got, want), m
        if m != "CrossCorr_Norm":
            assert np.array_equal(got, O.proximity_exact(m, S, T).astype(np.float32)), m


@pytest.mark.parametrize("parts", [3])
def test_tensor_f32_bands_within_bar(tensor, ocip, parts):
    from openclipp_b200 import bands
    rng = np.random.default_rng(99)
    S = (rng.random((400, 320)) + 0.1).astype(np.float32)
    T = S[150:181, 60:91].copy()
    got = stitched(bands, "CrossCorr", S, T, parts)
    ex = O.proximity_exact("CrossCorr", S, T)
    assert np.max(np.abs(got - ex) / np.abs(ex)) <= 1e-5


def test_device_view_holds_the_owned_rows(plain, ocip):
    import torch
    from openclipp_b200 import bands
    rng = np.random.default_rng(5)
    S = rng.random((200, 128)).astype(np.float32)
    T = S[20:37, 30:47].copy()
    bm = bands.BandMatch(S, T, 1, 3)
    try:
        bm.run("CrossCorr")
        torch.cuda.ExternalStream(bands.ocip_stream()).synchronize()
        dev = torch.as_tensor(bm.device_view(), device="cuda").cpu().numpy()
        assert np.array_equal(dev, bm.owned())
        whole = ocip.match("CrossCorr", S, T)
        assert np.array_equal(dev, whole[bm.y0:bm.y1])
    finally:
        bm.release()
