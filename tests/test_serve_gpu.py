"""Serving loop (lzk_server_*): every proof served in a mix of concurrent
requests over several resident circuits equals the proof of the same
(witness, r, s) computed alone; memory-budget admission (rejection of a
request that can never fit, a circuit that does not fit, eviction of idle
contexts of other circuits) and cancellation of queued requests."""
import numpy as np
import pytest

from helpers import same_point
from oracle import FR

pytestmark = pytest.mark.gpu


def _circuit(log_m, seed):
    from liblightzk_b200 import groth16, synth
    c = synth.Circuit(log_m, seed=seed, n_public=1, n_free=16, block=16)
    pk = synth.ProvingKey(c, seed=seed + 1)
    return c, pk, groth16.Prover(c, pk, mode=groth16.STANDARD, window_bits=8)


def _same_proof(orc, a, b):
    from liblightzk_b200.groth16 import split_proof
    A1, B1, C1 = split_proof(a)
    A2, B2, C2 = split_proof(b)
    return same_point(orc, 1, A1, A2) and same_point(orc, 2, B1, B2) and same_point(orc, 1, C1, C2)


def test_mix_equals_alone(cuda, orc, rng_state):
    from liblightzk_b200 import device, serve
    circs = [_circuit(lg, 10 + lg) for lg in (6, 8, 10)]
    wits = [[device.to_host(c.witness(100 + i)) for i in range(2)] for c, _, _ in circs]
    jobs = []
    for i in range(12):
        k = i % 3
        r, s = orc.rand_field(FR, 2, rng_state)
        jobs.append((k, wits[k][i % 2], r, s))
    alone = [device.to_host(circs[k][2].prove(device.to_device(z), r, s)) for k, z, r, s in jobs]
    srv = serve.Server(budget_bytes=64 << 30, max_inflight=4)
    cids = [srv.add(p) for _, _, p in circs]
    ids = [srv.submit(cids[k], z, r, s) for k, z, r, s in jobs]
    served = [srv.wait(rid) for rid in ids]
    for a, b in zip(alone, served):
        assert _same_proof(orc, a, b)
    st = srv.stats()
    assert st["completed"] == 12 and st["rejected"] == 0 and st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()


def test_budget_admission_and_eviction(cuda, orc, rng_state):
    from liblightzk_b200 import device, serve
    (c1, _, p1), (c2, _, p2) = _circuit(7, 40), _circuit(7, 50)
    r1, r2 = p1.device_bytes(), p2.device_bytes()
    # size of one serving context, measured
    srv = serve.Server(budget_bytes=64 << 30, max_inflight=1)
    cid = srv.add(p1)
    srv.wait(srv.submit(cid, device.to_host(c1.witness(1)), *orc.rand_field(FR, 2, rng_state)))
    ctx = srv.stats()["device_bytes"] - r1
    srv.close()
    assert ctx > 0
    # no room for any proof context: the request is rejected, not queued forever
    srv = serve.Server(budget_bytes=r1 + ctx // 2, max_inflight=2)
    cid = srv.add(p1)
    rid = srv.submit(cid, device.to_host(c1.witness(1)), *orc.rand_field(FR, 2, rng_state))
    srv.wait_idle()
    assert srv.poll(rid)[0] == serve.LZK_EREJECTED
    assert srv.stats()["rejected"] == 1
    srv.close()
    # two resident circuits and room for one context: the idle context of one
    # circuit is released when the other needs one
    srv = serve.Server(budget_bytes=r1 + r2 + ctx + ctx // 2, max_inflight=1)
    a, b = srv.add(p1), srv.add(p2)
    for k in range(4):
        cid, circ, prov = (a, c1, p1) if k % 2 == 0 else (b, c2, p2)
        z = device.to_host(circ.witness(k))
        r, s = orc.rand_field(FR, 2, rng_state)
        got = srv.wait(srv.submit(cid, z, r, s))
        assert _same_proof(orc, got, device.to_host(prov.prove(device.to_device(z), r, s)))
        assert srv.stats()["device_bytes"] <= r1 + r2 + ctx + ctx // 2
    assert srv.stats()["completed"] == 4
    srv.close()
    # a circuit whose resident tables exceed the budget is refused
    srv = serve.Server(budget_bytes=r1 // 2, max_inflight=1)
    with pytest.raises(Exception):
        srv.add(p1)
    srv.close()


def test_cancel_queued(cuda, orc, rng_state):
    from liblightzk_b200 import device, serve
    c, _, p = _circuit(10, 60)
    z = device.to_host(c.witness(3))
    srv = serve.Server(budget_bytes=64 << 30, max_inflight=1)
    cid = srv.add(p)
    ids = [srv.submit(cid, z, *orc.rand_field(FR, 2, rng_state)) for _ in range(6)]
    cancelled = srv.cancel(ids[-1])
    srv.wait_idle()
    statuses = [srv.poll(rid)[0] for rid in ids]
    assert statuses[:5] == [0] * 5
    assert (cancelled == 0 and statuses[5] == serve.LZK_ECANCELED) or (cancelled == serve.LZK_EBUSY and statuses[5] == 0)
    srv.close()
