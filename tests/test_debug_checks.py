"""The bounds-checking debug build (liblzk_b200_debug.so, LZK_DEBUG_CHECKS).

On the CPU: the release library reports its checks compiled out and its
error word as 0 (no device call).  On the GPU, in a child process that loads
the debug library: plain and table MSMs in G1 and G2, the prover's presorted
and concatenated MSMs (one small proof in each mode) and a batch plan all
give the oracle's results with every index check passing (error word 0)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEBUG_LIB = os.path.join(ROOT, "liblightzk_b200", "liblzk_b200_debug.so")

CHILD = r'''
import sys, numpy as np, torch
sys.path.insert(0, ROOT)
sys.path.insert(0, ROOT + "/tests")
from liblightzk_b200 import _capi, batch, device, groth16, msm, synth
from oracle import Oracle, FR
from helpers import same_point
orc = Oracle()
L = _capi.lib()
assert L.lzk_debug_checks_enabled() == 1, "not the debug library"
L.lzk_debug_check_word(1)
st = np.array([7], np.uint64)
for g, n in ((1, 20000), (2, 3000)):
    s = orc.rand_field(FR, n, st); b = orc.fixed_base(g, orc.rand_field(FR, n, st))
    want = orc.msm(g, s, b)
    ds, db = device.to_device(s), device.to_device(b)
    assert same_point(orc, g, device.to_host(msm.msm(g, ds, db)), want)
    t = msm.precompute(g, db, 12, msm.windows_for(12), n)
    assert same_point(orc, g, device.to_host(msm.msm_precomputed(g, ds, t, 12, msm.windows_for(12), n)), want)
circ = synth.Circuit(9, seed=3, n_public=1, n_free=16, block=16)
z = circ.witness(4); pk = synth.ProvingKey(circ, seed=5)
h = device.to_host
keys = {"a_query": h(pk.a), "b1_query": h(pk.b1), "b2_query": h(pk.b2), "l_query": h(pk.l), "h_query": h(pk.h),
        "alpha1": h(pk.alpha1), "beta1": h(pk.beta1), "delta1": h(pk.delta1), "beta2": h(pk.beta2),
        "delta2": h(pk.delta2)}
for mode in (0, 1):
    r, s2 = orc.rand_field(FR, 2, st)
    p = groth16.Prover(circ, pk, mode=mode, window_bits=8)
    A, B, C = groth16.split_proof(p.prove(z, r, s2))
    p.close()
    eA, eB, eC = orc.groth16_prove([m.host() for m in circ.mats], circ.M, circ.n_vars, circ.n_public, circ.log_m,
                                   keys, h(z), r, s2, mode)
    assert same_point(orc, 1, A, eA) and same_point(orc, 2, B, eB) and same_point(orc, 1, C, eC)
msms = []
for i, n in enumerate((1000, 5000, 300)):
    msms.append((synth.random_fr(n, 9, i), synth.fixed_base(1, synth.random_fr(n, 10, i)), device.empty((3, 4))))
plan = batch.BatchPlan(1, msms, [])
plan.run(use_graph=False)
for s, b, o in msms:
    assert same_point(orc, 1, h(o), orc.msm(1, h(s), h(b)))
plan.close()
torch.cuda.synchronize()
word = L.lzk_debug_check_word(1)
assert word == 0, f"debug error word {word:#x}"
print("debug checks ok")
'''


def test_release_library_has_no_checks():
    from liblightzk_b200 import _capi
    L = _capi.lib()
    assert L.lzk_debug_checks_enabled() == 0 and L.lzk_debug_check_word(1) == 0


@pytest.mark.gpu
def test_debug_library_checks_pass_on_valid_work(cuda):
    if not os.path.exists(DEBUG_LIB):
        pytest.fail("liblzk_b200_debug.so is not built (python -m liblightzk_b200.build --debug)")
    env = dict(os.environ, LZK_LIBRARY=DEBUG_LIB)
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + CHILD], env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0 and "debug checks ok" in r.stdout, r.stdout[-2000:] + r.stderr[-3000:]
