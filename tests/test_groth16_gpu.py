"""End-to-end Groth16 parity: the CUDA prove chain (lzk_groth16_prove through
the C ABI) against the oracle's restatement of Groth16::Prove
(groth16.cuh:154-222), on the same seeded circuit, witness, proving key and
(r, s), in both modes.  Proof points compared after affine normalisation.
Also covers the setup path the instances come from: seeded Fr streams,
fixed-base key generation (fix_base_multi_scalar_multiplication_*,
msm.cuh:5-46) and the witness solver."""
import numpy as np
import pytest

from helpers import R_MINUS_1_CANON, same_point
from oracle import FR

pytestmark = pytest.mark.gpu


def _host(t):
    from liblightzk_b200 import device
    return device.to_host(t)


def test_random_fr_deterministic_and_reduced(cuda, orc):
    from liblightzk_b200 import synth
    a = _host(synth.random_fr(5000, 11, 3))
    b = _host(synth.random_fr(5000, 11, 3))
    c = _host(synth.random_fr(100, 11, 3, offset=4900))
    d = _host(synth.random_fr(5000, 12, 3))
    assert (a == b).all() and (a[4900:] == c).all() and not (a == d).all()
    # every value is a canonical Montgomery residue (< r): from_mont(to_mont(x)) roundtrip
    back = orc.to_mont(FR, orc.from_mont(FR, a))
    assert (back == a).all()


@pytest.mark.parametrize("g", [1, 2])
def test_fixed_base_matches_oracle(cuda, orc, rng_state, g):
    from liblightzk_b200 import device, synth
    k = orc.rand_field(FR, 777, rng_state)
    edge = orc.to_mont(FR, np.array([[0, 0, 0, 0], [1, 0, 0, 0], R_MINUS_1_CANON, [255, 0, 0, 0]], np.uint64))
    k = np.concatenate([k, edge])
    got = _host(synth.fixed_base(g, device.to_device(k)))
    assert (got == orc.fixed_base(g, k)).all()


def _instance(log_m, seed=5):
    from liblightzk_b200 import synth
    circ = synth.Circuit(log_m, seed=seed, n_public=2, n_free=32, block=32)
    z = circ.witness(seed + 100)
    pk = synth.ProvingKey(circ, seed=seed + 200)
    return circ, z, pk


def _oracle_inputs(circ, pk):
    mats = [m.host() for m in circ.mats]
    keys = {"a_query": _host(pk.a), "b1_query": _host(pk.b1), "b2_query": _host(pk.b2), "l_query": _host(pk.l),
            "h_query": _host(pk.h), "alpha1": _host(pk.alpha1), "beta1": _host(pk.beta1),
            "delta1": _host(pk.delta1), "beta2": _host(pk.beta2), "delta2": _host(pk.delta2)}
    return mats, keys


@pytest.mark.parametrize("log_m", [3, 7])
def test_witness_satisfies(cuda, orc, log_m):
    circ, z, _ = _instance(log_m)
    assert circ.unsatisfied_rows(z) == 0
    zh = _host(z)
    out = [orc.spmv(v, c, rp[:-1], zh) for v, c, rp in (m.host() for m in circ.mats)]
    ab = orc.field_op(FR, 2, out[0], out[1])
    assert (ab == out[2]).all()
    zbad = z.clone()
    zbad[-1, 0] ^= 1
    assert circ.unsatisfied_rows(zbad) >= 1


@pytest.mark.parametrize("log_m", [4, 9, 12])
@pytest.mark.parametrize("mode", [0, 1])
def test_prove_matches_oracle(cuda, orc, rng_state, log_m, mode):
    from liblightzk_b200 import groth16
    circ, z, pk = _instance(log_m)
    r, s = orc.rand_field(FR, 2, rng_state)
    prover = groth16.Prover(circ, pk, mode=mode, window_bits=8 if log_m < 10 else 12)
    proof = prover.prove(z, r, s)
    A, B, C = groth16.split_proof(proof)
    mats, keys = _oracle_inputs(circ, pk)
    eA, eB, eC = orc.groth16_prove(mats, circ.M, circ.n_vars, circ.n_public, log_m, keys, _host(z), r, s, mode)
    assert same_point(orc, 1, A, eA)
    assert same_point(orc, 2, B, eB)
    assert same_point(orc, 1, C, eC)
    # a second proof with other (r, s) on the same resident prover
    r2, s2 = orc.rand_field(FR, 2, rng_state)
    A2, B2, C2 = groth16.split_proof(prover.prove(z, r2, s2))
    eA2, eB2, eC2 = orc.groth16_prove(mats, circ.M, circ.n_vars, circ.n_public, log_m, keys, _host(z), r2, s2, mode)
    assert same_point(orc, 1, A2, eA2) and same_point(orc, 2, B2, eB2) and same_point(orc, 1, C2, eC2)
    prover.close()


def test_modes_differ_only_in_h(cuda, orc, rng_state):
    """standard vs reference chain: A and B agree, C differs (H scalars
    differ: coset quotient vs the reference's 2M-point path)"""
    from liblightzk_b200 import groth16
    circ, z, pk = _instance(6)
    r, s = orc.rand_field(FR, 2, rng_state)
    p0 = groth16.split_proof(groth16.Prover(circ, pk, mode=0, window_bits=8).prove(z, r, s))
    p1 = groth16.split_proof(groth16.Prover(circ, pk, mode=1, window_bits=8).prove(z, r, s))
    assert same_point(orc, 1, p0[0], p1[0]) and same_point(orc, 2, p0[1], p1[1])
    assert not same_point(orc, 1, p0[2], p1[2])


def test_proof_wire_format(cuda, orc, rng_state):
    """the 256-byte wire form is the affine proof in canonical integers (the
    numbers Groth16::Prove prints, groth16.cuh:219-221); decoding gives the
    same points; infinity is all zeros; a coordinate >= p is flagged"""
    from oracle import FQ

    from liblightzk_b200 import groth16
    circ, z, pk = _instance(5)
    r, s = orc.rand_field(FR, 2, rng_state)
    prover = groth16.Prover(circ, pk, mode=0, window_bits=8)
    proof = prover.prove(z, r, s)
    A, B, C = groth16.split_proof(proof)
    wire = _host(groth16.to_wire(proof)).reshape(8, 4)
    expect = np.concatenate([orc.from_mont(FQ, orc.jac_to_aff(1, A[None])[0]),
                             orc.from_mont(FQ, orc.jac_to_aff(2, B[None])[0].reshape(4, 4)),
                             orc.from_mont(FQ, orc.jac_to_aff(1, C[None])[0])])
    assert (wire == expect).all()
    back, bad = groth16.from_wire(groth16.to_wire(proof))
    assert int(bad.item()) == 0
    A2, B2, C2 = groth16.split_proof(back)
    assert same_point(orc, 1, A, A2) and same_point(orc, 2, B, B2) and same_point(orc, 1, C, C2)
    # A at infinity (libff's (0, 1, 0)) encodes as zeros and decodes back
    one = orc.to_mont(FQ, np.array([[1, 0, 0, 0]], np.uint64))[0]
    pinf = proof.clone()
    pinf[0:12] = torch_tensor(np.concatenate([np.zeros(4, np.uint64), one, np.zeros(4, np.uint64)]), proof.device)
    w = groth16.to_wire(pinf)
    assert (_host(w).reshape(8, 4)[0:2] == 0).all()
    back, bad = groth16.from_wire(w)
    assert int(bad.item()) == 0 and (_host(back)[0:12].reshape(3, 4)[2] == 0).all()
    # a coordinate equal to p is not canonical: flagged, decoded as infinity
    p_limbs = np.array([0x3C208C16D87CFD47, 0x97816A916871CA8D, 0xB85045B68181585D, 0x30644E72E131A029], np.uint64)
    wb = _host(groth16.to_wire(proof)).copy()
    wb[0:4] = p_limbs
    back, bad = groth16.from_wire(torch_tensor(wb, proof.device))
    assert int(bad.item()) == 1 and (_host(back)[0:12].reshape(3, 4)[2] == 0).all()
    prover.close()


def torch_tensor(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.uint64).view(np.int64)).to(dev)
