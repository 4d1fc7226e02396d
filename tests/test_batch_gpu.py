"""Batched MSMs and NTTs of uneven sizes (lzk_batch_plan_*): every result of
the batch equals the oracle's, eagerly and through the captured CUDA graph
(first run captures, second replays) after the inputs changed in place, with
plain bases and with the shifted-copy tables of LZK_BATCH_FIXED_BASES, and
with the MSM phases as one persistent launch (LZK_BATCH_PERSISTENT: runs are
eager whatever use_graph says)."""
import numpy as np
import pytest

from helpers import bases, scalars
from oracle import FR

pytestmark = pytest.mark.gpu


def _dev(a):
    from liblightzk_b200 import device
    return device.to_device(a)


def _host(t):
    from liblightzk_b200 import device
    return device.to_host(t)


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("fixed_bases", [False, True])
@pytest.mark.parametrize("group", [1, 2])
def test_batch_plan(cuda, orc, rng_state, group, fixed_bases, persistent):
    import torch

    from liblightzk_b200 import batch
    if group == 1:
        sizes, wins = [0, 1, 5, 100, 1000, 3000, 20000], [0, 0, 4, 0, 9, 12, 0]
        nspec = [(5, 0), (5, 0), (10, 3), (13, 1), (12, 2)]
    else:
        sizes, wins = [3, 200, 1500], [0, 6, 0]
        nspec = [(4, 1)]
    host_b = [bases(orc, group, n, rng_state) if n else np.zeros((0, 2, 4) if group == 1 else (0, 2, 2, 4), np.uint64)
              for n in sizes]
    dev_s = [_dev(np.zeros((n, 4), np.uint64)) for n in sizes]
    dev_b = [_dev(b) for b in host_b]
    outs = [torch.empty((3, 4) if group == 1 else (3, 2, 4), dtype=torch.int64, device="cuda") for _ in sizes]
    dev_n = [_dev(np.zeros((1 << k, 4), np.uint64)) for k, _ in nspec]
    plan = batch.BatchPlan(group, [(s, b, o, w) for s, b, o, w in zip(dev_s, dev_b, outs, wins)],
                           [(d, k, di) for d, (k, di) in zip(dev_n, nspec)], fixed_bases=fixed_bases,
                           persistent=persistent)
    stream = torch.cuda.Stream()
    for mode in ("eager", "capture", "replay"):
        hs = [scalars(orc, n, rng_state) if n else np.zeros((0, 4), np.uint64) for n in sizes]
        hn = [orc.rand_field(FR, 1 << k, rng_state) for k, _ in nspec]
        for d, h in zip(dev_s, hs):
            d.copy_(_dev(h))
        for d, h in zip(dev_n, hn):
            d.copy_(_dev(h))
        torch.cuda.synchronize()
        plan.run(use_graph=(mode != "eager"), stream=stream)
        torch.cuda.synchronize()
        for n, h, b, o in zip(sizes, hs, host_b, outs):
            expect = orc.msm(group, h, b) if n else None
            got = orc.jac_to_aff(group, _host(o)[None])
            if n:
                assert (got == orc.jac_to_aff(group, expect[None])).all(), (mode, n)
            else:
                assert got.sum() == 0
        for (k, di), h, d in zip(nspec, hn, dev_n):
            assert (_host(d) == orc.ntt(h, k, di)).all(), (mode, k, di)
    assert plan.device_bytes() > 0
    plan.close()


def test_autotuner_installs_measured_widths(cuda):
    from liblightzk_b200 import _capi, autotune, msm
    table = autotune.tune(1, log_ns=[10, 12], spread=1, reps=1)
    for lg, (best, res) in table.items():
        assert best in res and msm.autotune_window(1, 1 << lg) == best
        _capi.call("lzk_msm_set_window", 1, lg, 0)


def test_persistent_barrier_timeout_is_reported(cuda, orc, rng_state):
    """The persistent launch's grid barriers wait with a bound.  With one
    arrival that never comes and a short poll limit (the test hook
    lzk_debug_persistent_barrier), every block gives up at the first barrier
    and leaves, and the run returns LZK_ETIMEOUT (-3) without any fault; the
    next run with normal barriers gives the oracle's result."""
    import torch

    from liblightzk_b200 import LzkError, _capi, batch
    n = 3000
    hb = bases(orc, 1, n, rng_state)
    hs = scalars(orc, n, rng_state)
    s, b = _dev(hs), _dev(hb)
    out = torch.empty((3, 4), dtype=torch.int64, device="cuda")
    plan = batch.BatchPlan(1, [(s, b, out)], [], persistent=True)
    stream = torch.cuda.Stream()
    _capi.call("lzk_debug_persistent_barrier", 1, 4096)
    try:
        with pytest.raises(LzkError) as e:
            plan.run(stream=stream)
        assert e.value.status == -3
    finally:
        _capi.call("lzk_debug_persistent_barrier", 0, 0)
    plan.run(stream=stream)
    torch.cuda.synchronize()
    want = orc.jac_to_aff(1, orc.msm(1, hs, hb)[None])
    assert (orc.jac_to_aff(1, _host(out)[None]) == want).all()
    plan.close()
