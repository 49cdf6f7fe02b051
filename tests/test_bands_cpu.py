"""Row-band split of one image across GPUs: the partition (C ABI host
arithmetic, no GPU) and the stitching of the bands, on CPU.

The per-band maps here come from the oracle, standing in for each GPU's
ImageProximity call; what is under test is the band arithmetic of
ocipGetProximityBand and openclipp_b200.bands.gather_rows over gloo."""
import os
import socket

import numpy as np
import pytest

from oracle import oracle as O


def _bands():
    from openclipp_b200 import bands
    return bands


@pytest.mark.parametrize("H,th", [(1, 1), (7, 5), (64, 16), (100, 31), (4096, 31), (513, 64)])
@pytest.mark.parametrize("parts", [1, 2, 3, 4, 7, 8])
def test_partition_covers_rows_with_their_windows(H, th, parts):
    B = _bands()
    ay = th // 2
    owned = []
    for p in range(parts):
        y0, y1, s0, s1 = B.band(H, th, p, parts)
        owned.append((y0, y1))
        if y1 == y0:
            assert s0 == s1 == y0
            continue
        # every row of every owned window that lies in the image is in the band
        assert s0 <= max(0, y0 - ay) and s1 >= min(H, y1 - ay + th - 1)
        assert 0 <= s0 and s1 <= H and s1 - s0 >= th
        # the band is no larger than its windows, widened to the template height
        assert s1 - s0 <= max(th, (y1 - y0) + th - 1)
    assert owned[0][0] == 0 and owned[-1][1] == H
    assert all(owned[i][1] == owned[i + 1][0] for i in range(parts - 1))
    sizes = [b - a for a, b in owned]
    assert max(sizes) - min(sizes) <= 1


def test_invalid_arguments_are_refused():
    from openclipp_b200 import ocip
    B = _bands()
    for args in [(10, 0, 0, 1), (10, 11, 0, 1), (10, 3, 1, 1), (10, 3, -1, 2), (10, 3, 0, 0)]:
        with pytest.raises(ocip.OcipError) as e:
            B.band(*args)
        assert e.value.code == ocip.CL_INVALID_VALUE


@pytest.mark.parametrize("measure", ["SqrDistance", "CrossCorr_Norm", "AbsDistance"])
@pytest.mark.parametrize("parts", [2, 3, 5])
def test_band_maps_stitch_into_the_whole_map(measure, parts):
    """The map of each part's source band, at the part's rows, equals the whole
    image's map there: zero padding falls only outside the whole image."""
    B = _bands()
    rng = np.random.default_rng(parts)
    S = rng.integers(0, 256, (61, 40), dtype=np.uint8)
    T = S[10:23, 5:16].copy()
    whole = O.proximity_exact(measure, S, T)
    stitched = np.full_like(whole, np.nan)
    for p in range(parts):
        y0, y1, s0, s1 = B.band(S.shape[0], T.shape[0], p, parts)
        band = O.proximity_exact(measure, np.ascontiguousarray(S[s0:s1]), T)
        stitched[y0:y1] = band[y0 - s0:y1 - s0]
    assert np.array_equal(stitched, whole, equal_nan=True)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    from openclipp_b200 import bands as B
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        rng = np.random.default_rng(7)
        S = rng.random((45, 33)).astype(np.float32)
        T = S[4:13, 9:20].copy()
        y0, y1, s0, s1 = B.band(S.shape[0], T.shape[0], rank, world)
        band = O.proximity_exact("CrossCorr", np.ascontiguousarray(S[s0:s1]), T)
        full = B.gather_rows(torch.from_numpy(band[y0 - s0:y1 - s0].copy()), S.shape[0],
                             T.shape[0], rank, world)
        if rank == 0:
            np.save(os.path.join(out_dir, "map.npy"), full.numpy())
            np.save(os.path.join(out_dir, "want.npy"), O.proximity_exact("CrossCorr", S, T))
        else:
            assert full is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_their_bands(tmp_path, world):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    got = np.load(tmp_path / "map.npy")
    want = np.load(tmp_path / "want.npy")
    assert np.array_equal(got, want)
