"""The batched-operator and serving configurations at their benchmark sizes,
against the oracle.

* Batched operators: the exact workload the bench times (64 G1 MSMs of
  2^10..2^20 points drawn log-uniformly, over slices of one pool of 2^20
  random points, and 32 Fr NTTs of 2^12..2^22 elements in all four
  directions), run as one plan through its captured CUDA graph, with plain
  bases and with shifted-copy tables built at creation, and as the
  persistent launch over the tables; every MSM
  result equals the oracle's MSM (the reference checks its MSM the same
  way, GPU against CPU, test/msm-check.cu:45-58) and every NTT output the
  oracle's transform, element for element.
* Serving: three resident circuits of 2^16, 2^18 and 2^20 constraints
  (built like the benchmark circuit), a burst of requests over all three
  with several in flight; every served proof equals the proof of the same
  (witness, r, s) made alone, and one served 2^20 proof equals the oracle's
  whole proof (SpMV, H chain, the five MSMs and Phase 6, groth16.cuh:
  154-222)."""
import numpy as np
import pytest

from helpers import same_point
from oracle import FR

pytestmark = pytest.mark.gpu


def _host(t):
    from liblightzk_b200 import device
    return device.to_host(t)


def test_batched_workload_against_oracle(cuda, orc):
    """the plan forms: plain bases, shifted-copy tables built at creation, and
    tables with the MSM phases as one persistent launch"""
    import torch

    from liblightzk_b200 import batch
    msms, ntts, pool = batch.workload_config3()
    sizes = [int(s.shape[0]) for s, _, _ in msms]
    assert len(msms) == 64 and max(sizes) > (1 << 19) and min(sizes) >= (1 << 10)
    assert len(ntts) == 32 and max(k for _, k, _ in ntts) >= 21
    ntt_in = [_host(d) for d, _, _ in ntts]
    want_msm = [orc.msm(1, _host(s), _host(b)) for s, b, _ in msms]
    want_ntt = [orc.ntt(h, k, di) for (_, k, di), h in zip(ntts, ntt_in)]
    stream = torch.cuda.Stream()
    for fixed, persistent in ((False, False), (True, False), (True, True)):
        plan = batch.BatchPlan(1, msms, ntts, fixed_bases=fixed, persistent=persistent)
        for _ in range(2):        # captures the graph, then replays it on fresh NTT inputs
            for (d, _, _), h in zip(ntts, ntt_in):
                d.copy_(torch.from_numpy(h.view(np.int64)).to(d.device))
            torch.cuda.synchronize()
            plan.run(use_graph=True, stream=stream)
            torch.cuda.synchronize()
        for (s, b, o), want in zip(msms, want_msm):
            assert same_point(orc, 1, _host(o), want), f"MSM of {s.shape[0]} points ({fixed=}, {persistent=})"
        for (d, k, di), want in zip(ntts, want_ntt):
            assert (_host(d) == want).all(), f"NTT 2^{k} direction {di} ({fixed=}, {persistent=})"
        plan.close()


def test_serving_mix_at_benchmark_sizes(cuda, orc):
    from liblightzk_b200 import device, groth16, serve, synth
    logs = (16, 18, 20)
    circs, keys, provers, wits = [], [], [], []
    for lg in logs:
        c = synth.Circuit(lg, seed=lg)
        pk = synth.ProvingKey(c, seed=lg + 1)
        circs.append(c)
        keys.append(pk)
        provers.append(groth16.Prover(c, pk, mode=groth16.STANDARD, window_bits=17))
        wits.append([_host(c.witness(1000 + i)) for i in range(2)])
    rng = np.array([71], np.uint64)
    jobs = []
    for i in range(9):
        k = [2, 0, 1, 2, 1, 0, 2, 2, 1][i]
        r, s = orc.rand_field(FR, 2, rng)
        jobs.append((k, wits[k][i % 2], r, s))
    alone = [_host(provers[k].prove(device.to_device(z), r, s)) for k, z, r, s in jobs]
    srv = serve.Server(budget_bytes=96 << 30, max_inflight=4)
    cids = [srv.add(p) for p in provers]
    rids = [srv.submit(cids[k], z, r, s) for k, z, r, s in jobs]
    served = [srv.wait(rid) for rid in rids]
    assert srv.stats()["completed"] == len(jobs)
    srv.close()
    for (k, _, _, _), a, b in zip(jobs, alone, served):
        A1, B1, C1 = groth16.split_proof(a)
        A2, B2, C2 = groth16.split_proof(b)
        assert same_point(orc, 1, A1, A2) and same_point(orc, 2, B1, B2) and same_point(orc, 1, C1, C2), \
            f"served 2^{logs[k]} proof differs from the same proof made alone"
    # one served 2^20 proof against the oracle's whole proof
    k, z, r, s = jobs[0]
    c, pk = circs[k], keys[k]
    h = _host
    keyset = {"a_query": h(pk.a), "b1_query": h(pk.b1), "b2_query": h(pk.b2), "l_query": h(pk.l),
              "h_query": h(pk.h), "alpha1": h(pk.alpha1), "beta1": h(pk.beta1), "delta1": h(pk.delta1),
              "beta2": h(pk.beta2), "delta2": h(pk.delta2)}
    eA, eB, eC = orc.groth16_prove([m.host() for m in c.mats], c.M, c.n_vars, c.n_public, c.log_m, keyset, z, r, s,
                                   groth16.STANDARD)
    A, B, C = groth16.split_proof(served[0])
    assert same_point(orc, 1, A, eA) and same_point(orc, 2, B, eB) and same_point(orc, 1, C, eC)
    for p in provers:
        p.close()
