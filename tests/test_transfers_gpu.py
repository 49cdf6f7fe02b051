"""Host transfers of caller buffers (the reference's Send/Read,
C++/Buffer.cpp:123-194), through the C ABI.

A pageable host buffer (a numpy array: malloc'd memory, as a reference
program passes) is page-locked once its image has made four transfers, and
unregistered when the image is released; a buffer that is already page-locked
is used as it is. Results are the same either way.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

_CU_POINTER_ATTRIBUTE_MEMORY_TYPE = 2
_CU_MEMORYTYPE_HOST = 1


def is_page_locked(arr):
    cuda = ctypes.CDLL("libcuda.so.1")
    v = ctypes.c_uint(0)
    rc = cuda.cuPointerGetAttribute(ctypes.byref(v), _CU_POINTER_ATTRIBUTE_MEMORY_TYPE,
                                    ctypes.c_uint64(arr.ctypes.data))
    return rc == 0 and v.value == _CU_MEMORYTYPE_HOST


def test_reused_pageable_buffers_are_page_locked_and_released(ocip, plain):
    rng = np.random.default_rng(3)
    S = rng.integers(0, 256, (300, 500), dtype=np.uint8)
    T = S[10:26, 20:36].copy()
    out = np.zeros(S.shape, np.float32)
    assert not is_page_locked(S) and not is_page_locked(out)
    Si, Ti, Di = ocip.Image(S), ocip.Image(T), ocip.Image(out)
    for k in range(6):
        S[:] = rng.integers(0, 256, S.shape, dtype=np.uint8)
        Si.send()
        ocip.check(ocip.cross_corr(Si, Ti, Di), "ocipCrossCorr")
        Di.read()
        assert np.array_equal(out, O.proximity_exact(3, S, T).astype(np.float32)), k
        # page-locked from the fourth transfer on
        assert is_page_locked(S) == (k >= 3) and is_page_locked(out) == (k >= 3), k
    for x in (Si, Ti, Di):
        x.release()
    assert not is_page_locked(S) and not is_page_locked(out)


def test_page_locked_buffers_are_used_as_given(ocip, plain):
    import torch
    rng = np.random.default_rng(4)
    S = torch.empty((200, 260), dtype=torch.float32, pin_memory=True).numpy()
    S[:] = rng.random(S.shape, dtype=np.float32)
    T = S[5:20, 7:30].copy()
    assert is_page_locked(S)
    got = ocip.match("SqrDistance", S, T)
    want = O.proximity_refexact(0, S, T, fused=True)
    assert np.array_equal(got, want)
    assert is_page_locked(S)  # the library did not unregister the caller's pinned memory
