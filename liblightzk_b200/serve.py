"""Prove-request serving over resident provers (lzk_server_* in include/lzk.h).

    srv = Server(budget_bytes, max_inflight=4)
    cid = srv.add(prover)                       # a groth16.Prover, kept alive by the caller
    rid = srv.submit(cid, z_host, r, s)         # z_host: numpy uint64 (n_vars, 4)
    proof = srv.wait(rid)                       # numpy uint64 (48,)

`poisson_run` drives the serving benchmark: requests arriving as a Poisson
process over several resident circuits, each with a witness drawn from a
pool of pre-solved witnesses (pinned host memory) and fresh (r, s).
"""
import ctypes
import time

import numpy as np
import torch

from . import _capi
from .groth16 import PROOF_WORDS, fr_struct


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64), ("queued", ctypes.c_uint64), ("running", ctypes.c_uint64),
                ("device_bytes", ctypes.c_size_t), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("proofs_per_s", ctypes.c_double)]


class ServerCfg(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_inflight", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


REQ_WITNESS_PINNED = 1
LZK_EBUSY, LZK_ECANCELED, LZK_EREJECTED = -6, -7, -8


class Server:
    def __init__(self, budget_bytes, max_inflight=4):
        cfg = ServerCfg(budget_bytes, max_inflight, 0)
        h = ctypes.c_void_p()
        _capi.call("lzk_server_create", ctypes.byref(cfg), ctypes.byref(h))
        self.handle = h
        self.provers = []

    def add(self, prover):
        cid = ctypes.c_uint32()
        _capi.call("lzk_server_add_circuit", self.handle, prover.handle, ctypes.byref(cid))
        self.provers.append(prover)
        return cid.value

    def add_key_file(self, circuit, path, mode=0, window_bits=0):
        """make a resident prover for `circuit` from its key file (the loaded
        key is freed once the prover has built its tables) and add it"""
        from .groth16 import LoadedKey, Prover
        key = LoadedKey(path)
        try:
            prover = Prover(circuit, key, mode=mode, window_bits=window_bits)
        finally:
            key.close()
        return self.add(prover)

    def submit(self, cid, z, r, s, pinned=False):
        """z: numpy uint64 (n_vars, 4) or a pinned CPU torch tensor (pinned=True: it must
        stay unchanged until the request completes)"""
        rid = ctypes.c_uint64()
        zp = z.data_ptr() if isinstance(z, torch.Tensor) else np.ascontiguousarray(z, dtype=np.uint64).ctypes.data
        rr, ss = fr_struct(r), fr_struct(s)
        _capi.call("lzk_server_submit", self.handle, cid, zp, ctypes.byref(rr), ctypes.byref(ss),
                   REQ_WITNESS_PINNED if pinned else 0, ctypes.byref(rid))
        return rid.value

    def poll(self, rid):
        """(status, proof numpy (48,) or None, latency_ms)"""
        buf = np.zeros(PROOF_WORDS, np.uint64)
        lat = ctypes.c_double()
        st = _capi.lib().lzk_server_poll(self.handle, rid, buf.ctypes.data, ctypes.byref(lat))
        return st, (buf if st == 0 else None), lat.value

    def wait(self, rid, timeout_s=600.0):
        t0 = time.time()
        while True:
            st, proof, lat = self.poll(rid)
            if st != LZK_EBUSY:
                if st != 0:
                    raise _capi.LzkError(st, "lzk_server_poll")
                return proof
            if time.time() - t0 > timeout_s:
                raise TimeoutError(f"request {rid}")
            time.sleep(0.0005)

    def cancel(self, rid):
        return _capi.lib().lzk_server_cancel(self.handle, rid)

    def wait_idle(self, timeout_ms=600000):
        return _capi.lib().lzk_server_wait_idle(self.handle, timeout_ms)

    def stats(self):
        st = ServerStats()
        _capi.call("lzk_server_get_stats", self.handle, ctypes.byref(st))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def reset_stats(self):
        _capi.call("lzk_server_reset_stats", self.handle)

    def close(self):
        if self.handle:
            _capi.call("lzk_server_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_run(server, circuits, witness_pools, rate_per_s, n_requests, seed=5, mix=None):
    """submit n_requests Poisson arrivals (rate_per_s) over circuit ids
    `circuits` (chosen by `mix` probabilities, uniform by default), each with
    a pooled pinned witness and fresh (r, s); returns the server stats after
    all complete"""
    from .synth import random_fr
    from .device import to_host
    rng = np.random.default_rng(seed)
    rs = to_host(random_fr(2 * n_requests, seed, 777)).reshape(n_requests, 2, 4)
    gaps = rng.exponential(1.0 / rate_per_s, n_requests)
    which = rng.choice(len(circuits), n_requests, p=mix)
    server.reset_stats()
    ids = []
    t = time.perf_counter()
    for i in range(n_requests):
        t += gaps[i]
        delay = t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        pool = witness_pools[which[i]]
        z = pool[i % len(pool)]
        ids.append(server.submit(circuits[which[i]], z, rs[i, 0], rs[i, 1], pinned=True))
    server.wait_idle()
    for rid in ids:
        server.poll(rid)
    return server.stats()
