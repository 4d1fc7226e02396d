"""The tuning table (lzk_tune_set / lzk_tune_get): defaults, validation and
clearing, on the CPU (no device calls); and on the GPU, that every allowed
value of each knob gives results equal to the oracle's (the knobs change how
work is split, never what is computed) and that the autotuner installs what
it measured and a saved table loads back."""
import numpy as np
import pytest

from helpers import bases, same_point, scalars
from oracle import FR

WINDOW, CHUNK, RUN, NTT_BLOCK, TABLE_WINDOW, TABLE_CHUNK, TABLE_RUN = range(7)


def _lib():
    from liblightzk_b200 import _capi
    return _capi.lib()


def test_defaults_validation_and_clearing():
    L = _lib()
    assert L.lzk_tune_get(CHUNK, 1, 20) == 64 and L.lzk_tune_get(RUN, 2, 20) == 4
    assert L.lzk_tune_get(NTT_BLOCK, 0, 22) == 2048 and L.lzk_tune_get(WINDOW, 1, 20) == 0
    for knob, bad in ((CHUNK, 48), (CHUNK, 4), (CHUNK, 1024), (RUN, 3), (RUN, 32), (NTT_BLOCK, 128),
                      (NTT_BLOCK, 8192), (WINDOW, 1), (WINDOW, 25), (7, 1)):
        assert L.lzk_tune_set(knob, 1, 16, bad) == -1, (knob, bad)
    assert L.lzk_tune_set(CHUNK, 3, 16, 32) == -1          # no group 3
    assert L.lzk_tune_set(CHUNK, 1, 33, 32) == -1          # no size class 33
    assert L.lzk_tune_set(CHUNK, 1, 16, 128) == 0 and L.lzk_tune_get(CHUNK, 1, 16) == 128
    assert L.lzk_tune_get(CHUNK, 2, 16) == 64              # per group
    assert L.lzk_tune_set(CHUNK, 1, 16, 0) == 0 and L.lzk_tune_get(CHUNK, 1, 16) == 64
    assert L.lzk_tune_set(NTT_BLOCK, 5, 12, 1024) == 0 and L.lzk_tune_get(NTT_BLOCK, 1, 12) == 1024
    assert L.lzk_tune_set(NTT_BLOCK, 0, 12, 0) == 0 and L.lzk_tune_get(NTT_BLOCK, 0, 12) == 2048
    assert L.lzk_msm_set_window(1, 14, 9) == 0 and L.lzk_tune_get(WINDOW, 1, 14) == 9
    assert L.lzk_msm_set_window(1, 14, 0) == 0
    # tables have their own entries
    assert L.lzk_tune_get(TABLE_CHUNK, 1, 20) == 64 and L.lzk_tune_get(TABLE_RUN, 1, 20) == 4
    assert L.lzk_tune_set(TABLE_RUN, 1, 20, 8) == 0 and L.lzk_tune_get(TABLE_RUN, 1, 20) == 8
    assert L.lzk_tune_get(RUN, 1, 20) == 4
    assert L.lzk_tune_set(TABLE_RUN, 1, 20, 0) == 0
    assert L.lzk_tune_set(TABLE_WINDOW, 2, 18, 17) == 0 and L.lzk_tune_get(TABLE_WINDOW, 2, 18) == 17
    assert L.lzk_tune_set(TABLE_WINDOW, 2, 18, 0) == 0
    assert L.lzk_tune_set(TABLE_CHUNK, 1, 20, 24) == -1 and L.lzk_tune_set(7, 1, 20, 4) == -1


@pytest.mark.gpu
@pytest.mark.parametrize("group", [1, 2])
def test_msm_knobs_keep_results(cuda, orc, rng_state, group):
    from liblightzk_b200 import device, msm
    n = 20000 if group == 1 else 3000
    s, b = scalars(orc, n, rng_state), bases(orc, group, n, rng_state)
    want = orc.msm(group, s, b)
    ds, db = device.to_device(s), device.to_device(b)
    lg = int(np.ceil(np.log2(n)))
    L = _lib()
    try:
        for chunk in (8, 32, 64, 128, 512):
            for run in (1, 2, 4, 8, 16):
                assert L.lzk_tune_set(CHUNK, group, lg, chunk) == 0 and L.lzk_tune_set(RUN, group, lg, run) == 0
                for c in (7, 12):
                    got = device.to_host(msm.msm(group, ds, db, window_bits=c))
                    assert same_point(orc, group, got, want), (chunk, run, c)
        # a precomputed table too (one shared bucket set, its own entries)
        t = msm.precompute(group, db, 13, msm.windows_for(13), n)
        for chunk, run in ((16, 16), (256, 1)):
            L.lzk_tune_set(TABLE_CHUNK, group, lg, chunk)
            L.lzk_tune_set(TABLE_RUN, group, lg, run)
            got = device.to_host(msm.msm_precomputed(group, ds, t, 13, msm.windows_for(13), n))
            assert same_point(orc, group, got, want), (chunk, run, "table")
    finally:
        for k in (CHUNK, RUN, TABLE_CHUNK, TABLE_RUN):
            L.lzk_tune_set(k, group, lg, 0)


@pytest.mark.gpu
def test_ntt_block_keeps_results(cuda, orc, rng_state):
    from liblightzk_b200 import device, ntt
    L = _lib()
    try:
        for k in (1, 5, 9, 12, 13, 17):
            a = orc.rand_field(FR, 1 << k, rng_state)
            for blk in (256, 512, 1024, 2048, 4096):
                assert L.lzk_tune_set(NTT_BLOCK, 0, k, blk) == 0
                for d in range(4):
                    x = device.to_device(a)
                    ntt.ntt(x, k, d)
                    assert (device.to_host(x) == orc.ntt(a, k, d)).all(), (k, blk, d)
    finally:
        for k in (1, 5, 9, 12, 13, 17):
            L.lzk_tune_set(NTT_BLOCK, 0, k, 0)


@pytest.mark.gpu
def test_autotuner_installs_and_saves(cuda, tmp_path):
    from liblightzk_b200 import autotune
    L = _lib()
    t = autotune.tune_msm(1, log_ns=[10, 12], spread=1, reps=1, chunks=(32, 64), runs=(4, 8))
    n = autotune.tune_ntt([12], reps=1, blocks=(1024, 2048))
    for lg, e in t.items():
        assert (L.lzk_tune_get(WINDOW, 1, lg), L.lzk_tune_get(RUN, 1, lg), L.lzk_tune_get(CHUNK, 1, lg)) == \
            (e["window"], e["run"], e["chunk"])
    assert L.lzk_tune_get(NTT_BLOCK, 0, 12) == n[12][0]
    path = tmp_path / "table.json"
    autotune.save(path)
    for lg in (10, 12):
        for k in (WINDOW, RUN, CHUNK):
            L.lzk_tune_set(k, 1, lg, 0)
    L.lzk_tune_set(NTT_BLOCK, 0, 12, 0)
    autotune.load(path)
    for lg, e in t.items():
        assert L.lzk_tune_get(WINDOW, 1, lg) == e["window"] and L.lzk_tune_get(CHUNK, 1, lg) == e["chunk"]
    assert L.lzk_tune_get(NTT_BLOCK, 0, 12) == n[12][0]
    for lg in (10, 12):
        for k in (WINDOW, RUN, CHUNK):
            L.lzk_tune_set(k, 1, lg, 0)
    L.lzk_tune_set(NTT_BLOCK, 0, 12, 0)
