"""Batched MSMs and NTTs of uneven sizes (lzk_batch_plan_* in include/lzk.h).

    plan = BatchPlan(1, msms=[(scalars, bases, out), ...], ntts=[(data, log_n, direction), ...])
    plan.run(use_graph=True, stream=s)     # first run captures a CUDA graph, later runs replay it

`workload_config3` builds the batched-operator workload of the benchmark:
64 G1 MSMs with sizes log-uniform in [2^10, 2^20] and 32 Fr NTTs with sizes
2^k, k uniform in 12..22, uniform random scalars, points and coefficients.
"""
import ctypes

import numpy as np
import torch

from . import _capi
from .device import ptr, stream_ptr


FIXED_BASES = 0x1
PERSISTENT = 0x2


class BatchPlan:
    def __init__(self, group, msms=(), ntts=(), fixed_bases=False, persistent=False):
        """fixed_bases: build the MSMs' shifted-copy tables now (the bases are
        not read again; see LZK_BATCH_FIXED_BASES); persistent: the MSM phases
        after the digit sort as one persistent launch (LZK_BATCH_PERSISTENT;
        runs are then synchronous and never captured)"""
        self.group = group
        self._keep = (list(msms), list(ntts))
        md = (_capi.MsmDesc * max(len(msms), 1))()
        for i, m in enumerate(msms):
            s, b, o = m[:3]
            md[i].scalars, md[i].bases, md[i].n, md[i].out = ptr(s), ptr(b), int(s.shape[0]), ptr(o)
            md[i].window_bits = m[3] if len(m) > 3 else 0
        nd = (_capi.NttDesc * max(len(ntts), 1))()
        for i, (d, k, direction) in enumerate(ntts):
            nd[i].data, nd[i].log_n, nd[i].direction = ptr(d), k, direction
        h = ctypes.c_void_p()
        _capi.call("lzk_batch_plan_create_ex", group, md if msms else None, len(msms), nd if ntts else None,
                   len(ntts), (FIXED_BASES if fixed_bases else 0) | (PERSISTENT if persistent else 0),
                   ctypes.byref(h))
        self.handle = h

    def run(self, use_graph=False, stream=None):
        _capi.call("lzk_batch_plan_run", self.handle, 1 if use_graph else 0, stream_ptr(stream))

    def device_bytes(self):
        return int(_capi.lib().lzk_batch_plan_device_bytes(self.handle))

    def close(self):
        if self.handle:
            _capi.call("lzk_batch_plan_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def workload_config3(seed=3, n_msm=64, n_ntt=32, msm_log=(10, 20), ntt_log=(12, 22), device="cuda"):
    """inputs of the batched-operator benchmark; bases are slices of one
    pool of 2^msm_log[1] random points"""
    from .synth import fixed_base, random_fr
    rng = np.random.default_rng(seed)
    sizes = np.rint(2.0 ** rng.uniform(msm_log[0], msm_log[1], n_msm)).astype(np.int64)
    logs = rng.integers(ntt_log[0], ntt_log[1] + 1, n_ntt)
    pool = fixed_base(1, random_fr(1 << msm_log[1], seed, 40, device=device))
    msms = []
    for i, n in enumerate(sizes):
        start = int(rng.integers(0, (1 << msm_log[1]) - n + 1))
        sc = random_fr(int(n), seed, 41 + i, device=device)
        out = torch.empty((3, 4), dtype=torch.int64, device=device)
        msms.append((sc, pool[start:start + n], out))
    ntts = []
    for i, k in enumerate(logs):
        ntts.append((random_fr(1 << int(k), seed, 200 + i, device=device), int(k), int(rng.integers(0, 4))))
    return msms, ntts, pool
