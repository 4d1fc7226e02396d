"""Event tracing of device regions (trace.cu), the replacement for the
reference's synchronising Timer / CUDA_DEBUG pairs (timer.cu:3-16,
device-utils.cuh:3): per-name totals and the timeline of one proof, whose
regions run on four streams and must nest inside the proof's own region."""
import pytest

pytestmark = pytest.mark.gpu


def test_proof_timeline(cuda):
    import torch

    from liblightzk_b200 import _capi, device, groth16, synth
    circ = synth.Circuit(10, seed=3, n_public=2, n_free=32, block=32)
    z = circ.witness(4)
    pk = synth.ProvingKey(circ, seed=5)
    prover = groth16.Prover(circ, pk, mode=groth16.STANDARD, window_bits=8)
    r = device.to_host(synth.random_fr(2, 6, 1))
    prover.prove(z, r[0], r[1])
    torch.cuda.synchronize()
    _capi.trace_reset()
    _capi.trace_enable(True)
    try:
        prover.prove(z, r[0], r[1])
        torch.cuda.synchronize()
    finally:
        _capi.trace_enable(False)
    assert _capi.trace_get("groth16_prove")[1] == 1
    # G1 MSMs: A, B1, and L + H as one
    assert _capi.trace_get("msm_g1")[1] == 3 and _capi.trace_get("msm_g2")[1] == 1
    tl = _capi.trace_timeline()
    names = [t[0] for t in tl]
    for n in ("groth16_prove", "groth16_h_poly", "groth16_fixed_products", "groth16_dep_products",
              "groth16_assemble", "msm_g1_accumulate", "msm_g2_reduce", "msm_shared_sort"):
        assert n in names, n
    eps = 0.05    # ms: events recorded back to back on one stream
    assert all(b >= a - eps for _, a, b in tl)
    (p0, p1), = [(a, b) for n, a, b in tl if n == "groth16_prove"]
    assert abs(p0) < eps          # the proof is the first region begun
    assert all(p0 - eps <= a and b <= p1 + eps for _, a, b in tl)
    (a0, _), = [(a, b) for n, a, b in tl if n == "groth16_assemble"]
    assert all(b <= a0 + eps for n, _, b in tl if n in ("msm_g1", "msm_g2", "groth16_dep_products"))
    # a reset clears the timeline
    _capi.trace_reset()
    assert _capi.trace_timeline() == []
    prover.close()


def test_trace_only_filter(cuda):
    import torch

    from liblightzk_b200 import _capi, device, groth16, synth
    circ = synth.Circuit(9, seed=4, n_public=2, n_free=32, block=32)
    z = circ.witness(5)
    pk = synth.ProvingKey(circ, seed=6)
    prover = groth16.Prover(circ, pk, mode=groth16.STANDARD, window_bits=8)
    r = device.to_host(synth.random_fr(2, 7, 1))
    _capi.trace_reset()
    _capi.trace_only(["msm_g1_accumulate", "groth16_assemble"])
    _capi.trace_enable(True)
    try:
        prover.prove(z, r[0], r[1])
        torch.cuda.synchronize()
    finally:
        _capi.trace_enable(False)
        _capi.trace_only(None)
    assert _capi.trace_get("msm_g1_accumulate")[1] == 3
    assert _capi.trace_get("groth16_assemble")[1] == 1
    assert _capi.trace_get("msm_g2")[1] == 0 and _capi.trace_get("groth16_prove")[1] == 0
    assert {t[0] for t in _capi.trace_timeline()} == {"msm_g1_accumulate", "groth16_assemble"}
    _capi.trace_reset()
    prover.close()


def test_nvtx_ranges_beside_events(cuda, orc, rng_state):
    """NVTX ranges on, alone and together with the event tracer: results and
    event timings are unaffected (the ranges only mark host-side enqueues)"""
    from helpers import bases, same_point, scalars
    from liblightzk_b200 import _capi, device, msm
    n = 3000
    s, b = scalars(orc, n, rng_state), bases(orc, 1, n, rng_state)
    want = orc.msm(1, s, b)
    lib = _capi.lib()
    try:
        lib.lzk_trace_nvtx(1)
        got = device.to_host(msm.msm(1, device.to_device(s), device.to_device(b)))
        assert same_point(orc, 1, got, want)
        _capi.trace_reset()
        _capi.trace_enable(True)
        got = device.to_host(msm.msm(1, device.to_device(s), device.to_device(b)))
        _capi.trace_enable(False)
        assert same_point(orc, 1, got, want)
        ms, cnt = _capi.trace_get("msm_g1")
        assert cnt == 1 and ms > 0
    finally:
        lib.lzk_trace_nvtx(0)
        _capi.trace_enable(False)
