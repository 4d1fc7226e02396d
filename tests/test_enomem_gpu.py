"""Out-of-memory on every create path, forced from the host.

lzk_debug_fail_allocations(k) lets k more device allocations succeed and
fails the rest as if the device were out of memory.  For every k below what
a call needs, prover creation, batch-plan creation, key loading and an MSM
with library-managed scratch must return LZK_ENOMEM, release what they had
allocated (free device memory back to where it was) and leave the library
usable; a server whose context allocation fails rejects the request and
serves the next one once memory is back.  (The reference has no error path
here: its containers assert, xpu-vector.cuh:18.)  No GPU fault is involved:
the failure is made on the host before cudaMalloc is reached."""
import ctypes

import numpy as np
import pytest

from helpers import same_point
from oracle import FR

pytestmark = pytest.mark.gpu

ENOMEM, EREJECTED = -2, -8
SLACK = 8 << 20           # the CUDA pool and runtime may keep a few MB


def _fail_after(k):
    from liblightzk_b200 import _capi
    _capi.lib().lzk_debug_fail_allocations(k)


def _sweep(make, limit=80):
    """make() under k = 0, 1, ... allowed allocations until it succeeds;
    returns the number of failing k (each must be LZK_ENOMEM)"""
    from liblightzk_b200 import LzkError
    fails = 0
    for k in range(limit):
        _fail_after(k)
        try:
            obj = make()
        except LzkError as e:
            assert e.status == ENOMEM, f"k = {k}: status {e.status}"
            fails += 1
            continue
        finally:
            _fail_after(-1)
        return fails, obj
    raise AssertionError("never succeeded")


def _free():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


@pytest.fixture(scope="module")
def small_circuit(cuda):
    from liblightzk_b200 import synth
    circ = synth.Circuit(8, seed=31, n_public=1, n_free=16, block=16)
    return circ, synth.ProvingKey(circ, seed=32), circ.witness(33)


@pytest.mark.parametrize("mode", [0, 1])
def test_prover_creation(orc, small_circuit, mode):
    from liblightzk_b200 import groth16
    circ, pk, z = small_circuit
    groth16.Prover(circ, pk, mode=mode, window_bits=8).close()     # per-device tables now exist
    free0 = _free()
    fails, prover = _sweep(lambda: groth16.Prover(circ, pk, mode=mode, window_bits=8))
    assert fails >= 10
    prover.close()
    assert _free() >= free0 - SLACK, "device memory leaked by failed creations"
    # the library still proves, and correctly
    r, s = orc.rand_field(FR, 2, np.array([34], np.uint64))
    p0 = groth16.Prover(circ, pk, mode=mode, window_bits=8)
    A, B, C = groth16.split_proof(p0.prove(z, r, s))
    p0.close()
    from liblightzk_b200 import device
    h = device.to_host
    keys = {"a_query": h(pk.a), "b1_query": h(pk.b1), "b2_query": h(pk.b2), "l_query": h(pk.l),
            "h_query": h(pk.h), "alpha1": h(pk.alpha1), "beta1": h(pk.beta1), "delta1": h(pk.delta1),
            "beta2": h(pk.beta2), "delta2": h(pk.delta2)}
    eA, eB, eC = orc.groth16_prove([m.host() for m in circ.mats], circ.M, circ.n_vars, circ.n_public, circ.log_m,
                                   keys, h(z), r, s, mode)
    assert same_point(orc, 1, A, eA) and same_point(orc, 2, B, eB) and same_point(orc, 1, C, eC)


def test_batch_plan_creation(cuda, orc):
    from liblightzk_b200 import batch, device, synth
    msms = []
    for i, lg in enumerate((10, 12, 9)):
        n = 1 << lg
        msms.append((synth.random_fr(n, 41, i), synth.fixed_base(1, synth.random_fr(n, 42, i)),
                     device.empty((3, 4))))
    ntts = [(synth.random_fr(1 << 12, 43, 0), 12, 2), (synth.random_fr(1 << 10, 43, 1), 10, 1)]
    batch.BatchPlan(1, msms, ntts).close()
    free0 = _free()
    fails, plan = _sweep(lambda: batch.BatchPlan(1, msms, ntts))
    assert fails >= 2
    plan.run(use_graph=False)
    for s, b, o in msms:
        want = orc.msm(1, device.to_host(s), device.to_host(b))
        assert same_point(orc, 1, device.to_host(o), want)
    plan.close()
    assert _free() >= free0 - SLACK


def test_msm_scratch_and_key_load(cuda, orc, small_circuit, tmp_path):
    from liblightzk_b200 import LzkError, device, groth16, msm, synth
    n = 5000
    s = synth.random_fr(n, 51, 0)
    b = synth.fixed_base(1, synth.random_fr(n, 51, 1))
    want = orc.msm(1, device.to_host(s), device.to_host(b))
    _fail_after(0)
    try:
        with pytest.raises(LzkError) as e:
            msm.msm(1, s, b)
        assert e.value.status == ENOMEM
    finally:
        _fail_after(-1)
    assert same_point(orc, 1, device.to_host(msm.msm(1, s, b)), want)
    circ, pk, _ = small_circuit
    path = tmp_path / "k.pk"
    groth16.save_key(path, pk, circ)
    free0 = _free()
    _fail_after(0)
    try:
        with pytest.raises(LzkError) as e:
            groth16.LoadedKey(path)
        assert e.value.status == ENOMEM
    finally:
        _fail_after(-1)
    assert _free() >= free0 - SLACK
    groth16.LoadedKey(path).close()


def test_server_rejects_then_recovers(orc, small_circuit):
    from liblightzk_b200 import LzkError, device, groth16, serve
    circ, pk, z = small_circuit
    prover = groth16.Prover(circ, pk, mode=groth16.STANDARD, window_bits=8)
    r, s = orc.rand_field(FR, 2, np.array([35], np.uint64))
    A0, B0, C0 = groth16.split_proof(prover.prove(z, r, s))
    srv = serve.Server(4 << 30, max_inflight=2)
    cid = srv.add(prover)
    zh = device.to_host(z)
    _fail_after(0)
    try:
        rid = srv.submit(cid, zh, r, s)
        with pytest.raises(LzkError) as e:
            srv.wait(rid, timeout_s=60)
        assert e.value.status == EREJECTED
    finally:
        _fail_after(-1)
    A1, B1, C1 = groth16.split_proof(srv.wait(srv.submit(cid, zh, r, s), timeout_s=60))
    srv.close()
    prover.close()
    assert same_point(orc, 1, A0, A1) and same_point(orc, 2, B0, B1) and same_point(orc, 1, C0, C1)
