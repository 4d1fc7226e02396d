"""Measured window-width autotuner for plain-base MSMs.

For each size class 2^log_n the tuner times the cost model's window width
and its neighbours on the device (CUDA events, random inputs, median of a few
runs) and installs the fastest in the library's table (lzk_msm_set_window),
which every autotuned MSM and batch plan then uses.
"""
import numpy as np
import torch

from . import _capi, msm, synth


def _time(fn, reps):
    ts = []
    for _ in range(reps + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts[1:]))


def tune(group=1, log_ns=range(10, 21), spread=2, reps=3, seed=11, install=True):
    """returns {log_n: (best_c, {c: ms})}"""
    table = {}
    top = max(log_ns)
    sc_all = synth.random_fr(1 << top, seed, 90)
    bases_all = synth.fixed_base(group, synth.random_fr(1 << top, seed, 91))
    for lg in log_ns:
        n = 1 << lg
        _capi.call("lzk_msm_set_window", group, lg, 0)      # model value as the centre
        c0 = msm.autotune_window(group, n)
        res = {}
        for c in range(max(2, c0 - spread), min(22, c0 + spread) + 1):
            res[c] = _time(lambda c=c: msm.msm(group, sc_all[:n], bases_all[:n], window_bits=c), reps)
        best = min(res, key=res.get)
        table[lg] = (best, res)
        if install:
            _capi.call("lzk_msm_set_window", group, lg, best)
    return table
