"""lzk_msm_g1_noalloc: the G1 MSM for callers that cannot let the library
allocate device memory (its scratch is a fixed array the library reserves on
each GPU).  Called through the C ABI and compared with lzk_msm_g1, the
allocating entry point, on two calls in a row with different inputs, so a
second call over the shared scratch must not see the first call's data.
The first test plays the caller the entry point exists for: it makes the
set-up call (n = 0), then takes nearly all of the GPU's free memory, as a
process whose own allocator reserves the device at start-up would, and only
then runs an MSM through the entry point.  Kept in a file of its own that
runs last."""
import ctypes

import numpy as np
import pytest

from helpers import bases, scalars

pytestmark = pytest.mark.gpu

MAX_POINTS = 65536
MARGIN = 64 << 20        # device bytes left free while the memory is taken


def _call_noalloc(s, b, n, window_bits=0, out=None):
    from liblightzk_b200 import _capi, device
    if out is None:
        out = device.empty((3, 4))
    st = _capi.lib().lzk_msm_g1_noalloc(s.data_ptr(), b.data_ptr(), n, out.data_ptr(), window_bits, None)
    return st, out


def _call_alloc(s, b, n, window_bits=0):
    from liblightzk_b200 import _capi, device
    out = device.empty((3, 4))
    cfg = _capi.MsmCfg()
    cfg.window_bits = window_bits
    _capi.call("lzk_msm_g1", s.data_ptr(), b.data_ptr(), n, out.data_ptr(), ctypes.byref(cfg), None)
    return out


def _same(orc, a, b):
    from liblightzk_b200 import device
    A = orc.jac_to_aff(1, device.to_host(a)[None])
    B = orc.jac_to_aff(1, device.to_host(b)[None])
    return bool((A == B).all())


def _take_device_memory(torch):
    """allocate device memory until at most about MARGIN bytes stay free"""
    hog = []
    chunk = 1 << 34
    while chunk >= (8 << 20):
        free, _ = torch.cuda.mem_get_info()
        if free <= MARGIN + chunk:
            chunk //= 2
            continue
        try:
            hog.append(torch.empty(chunk, dtype=torch.uint8, device="cuda"))
        except RuntimeError:
            chunk //= 2
    return hog


def test_noalloc_after_setup_with_device_memory_taken(cuda, orc, rng_state):
    import torch
    from liblightzk_b200 import device
    n = 4096
    sh, bh = scalars(orc, n, rng_state), bases(orc, 1, n, rng_state)
    expect = orc.jac_to_aff(1, orc.msm(1, sh, bh)[None])
    s, b = device.to_device(sh), device.to_device(bh)
    out = device.empty((3, 4))
    st, _ = _call_noalloc(s, b, 0, out=out)          # the set-up call
    assert st == 0
    torch.cuda.synchronize()
    hog = _take_device_memory(torch)
    try:
        free, _ = torch.cuda.mem_get_info()
        assert free < 2 * MARGIN, f"could not take the device memory ({free} bytes still free)"
        for _ in range(2):
            st, _ = _call_noalloc(s, b, n, out=out)
            assert st == 0, f"status {st} with the device memory taken"
            torch.cuda.synchronize()
            assert (orc.jac_to_aff(1, device.to_host(out)[None]) == expect).all()
    finally:
        del hog
        torch.cuda.empty_cache()


def test_noalloc_matches_allocating_msm_twice(cuda, orc, rng_state):
    import torch
    from liblightzk_b200 import device
    for n, c in ((MAX_POINTS, 0), (3000, 12)):
        s = device.to_device(scalars(orc, n, rng_state))
        b = device.to_device(bases(orc, 1, n, rng_state))
        st, got = _call_noalloc(s, b, n, c)
        assert st == 0
        torch.cuda.synchronize()
        assert _same(orc, got, _call_alloc(s, b, n, c))
    # the second call above reused the scratch of the first; check it
    # against the oracle as well
    sh, bh = device.to_host(s), device.to_host(b)
    assert (orc.jac_to_aff(1, device.to_host(got)[None]) == orc.jac_to_aff(1, orc.msm(1, sh, bh)[None])).all()


def test_noalloc_refuses_oversized_requests(cuda, orc, rng_state):
    from liblightzk_b200 import device
    s = device.to_device(np.zeros((4, 4), np.uint64))
    b = device.to_device(np.zeros((4, 2, 4), np.uint64))
    st, _ = _call_noalloc(s, b, MAX_POINTS + 1)
    assert st == -1                      # LZK_EINVAL, nothing queued
    st, _ = _call_noalloc(s, b, 4, 20)   # window whose scratch exceeds the array
    assert st == -1
