"""The packed-byte SAD kernel's word algebra, restated in numpy (no GPU).

proximity_sad.cu sums |S - T| over a template row in 8-byte chunks: for output
i of a lane it takes the window bytes starting at offset 8*chunk + i as two
little-endian words (bytes 0-3 and 4-7 of the chunk, formed by byte_perm from
the 16 window bytes the lane loaded), adds the bytewise absolute differences
against the template chunk's two words, and in the last chunk masks both window
words to the template's valid bytes (the template is zero-padded to a multiple
of 8). This test checks that the chunked, masked sum equals the direct sum for
every template width 1..40 and both signednesses.
"""
import numpy as np
import pytest


def word(b, k):
    """Bytes b[k:k+4] as a little-endian uint32 (b is a uint8 array)."""
    return int(b[k]) | int(b[k + 1]) << 8 | int(b[k + 2]) << 16 | int(b[k + 3]) << 24


def sad4(a, b, signed):
    x = np.frombuffer(np.uint32(a).tobytes(), np.uint8)
    y = np.frombuffer(np.uint32(b).tobytes(), np.uint8)
    if signed:
        x, y = x.view(np.int8), y.view(np.int8)
    return int(np.abs(x.astype(np.int32) - y.astype(np.int32)).sum())


def kernel_row_sum(win, tmpl, tw, i, signed):
    """One output's sum over one template row, as the kernel forms it."""
    tw8 = -(-tw // 8) * 8
    t = np.zeros(tw8, np.uint8)
    t[:tw] = tmpl
    nc = tw8 // 8
    rem = tw - 8 * (nc - 1)
    m0 = 0xFFFFFFFF if rem >= 4 else (1 << (8 * rem)) - 1
    m1 = 0xFFFFFFFF if rem >= 8 else (0 if rem <= 4 else (1 << (8 * (rem - 4))) - 1)
    acc = 0
    for ch in range(nc):
        w0, w1 = word(win, 8 * ch + i), word(win, 8 * ch + i + 4)
        if ch == nc - 1:
            w0, w1 = w0 & m0, w1 & m1
        acc += sad4(w0, word(t, 8 * ch), signed) + sad4(w1, word(t, 8 * ch + 4), signed)
    return acc


@pytest.mark.parametrize("signed", [False, True])
def test_chunked_masked_sum_equals_direct_sum(signed):
    rng = np.random.default_rng(5 + signed)
    for tw in range(1, 41):
        tw8 = -(-tw // 8) * 8
        win = rng.integers(0, 256, 8 + tw8 + 8).astype(np.uint8)  # lane window + slack
        tmpl = rng.integers(0, 256, tw).astype(np.uint8)
        for i in range(8):
            s = win[i:i + tw]
            if signed:
                direct = int(np.abs(s.view(np.int8).astype(np.int32)
                                    - tmpl.view(np.int8).astype(np.int32)).sum())
            else:
                direct = int(np.abs(s.astype(np.int32) - tmpl.astype(np.int32)).sum())
            assert kernel_row_sum(win, tmpl, tw, i, signed) == direct, (tw, i)
