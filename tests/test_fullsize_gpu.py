"""Parity at the benchmark's full sizes, where the oracle cannot redo the
whole computation in seconds, through properties that do not depend on size:

* MSM at 2^20 (G1 and G2, shifted-copy table and plain bases): linearity
  MSM(s) + MSM(t) = MSM(s + t), and equal scalars MSM(k,...,k) = k * sum(P),
  whose digits all land in one bucket per window (the skewed-bucket path);
* NTT at 2^24: forward/inverse and coset round trips, and the transform of
  x (e_1), whose outputs must be the successive powers of the root of unity
  (times the coset generator for the coset transform); linearity at 2^22;
* Groth16 at 2^20 constraints: the R1CS products A.z, B.z, C.z against the
  oracle's SpMV (poly.cuh:5-30), a repeated request gives the same proof, and the proof
  equals the oracle's Phase 6 (groth16.cuh:209-215) applied to the oracle's
  H polynomial (the coset quotient chain in C) and to MSMs taken through the
  separate plain-bases path at another window width.

Point results are compared after affine normalisation."""
import numpy as np
import pytest

from helpers import R_MINUS_1_CANON, same_point
from oracle import ADD, FR, G_ADD, G_NEG, MUL, NEG

pytestmark = pytest.mark.gpu

LOG_MSM = 20
LOG_NTT = 24


def _host(t):
    from liblightzk_b200 import device
    return device.to_host(t)


def _dev(a):
    from liblightzk_b200 import device
    return device.to_device(a)


def _fr_const(orc, canon, n):
    v = orc.to_mont(FR, np.array([canon], np.uint64))[0]
    return np.ascontiguousarray(np.broadcast_to(v, (n, 4)))


@pytest.fixture(scope="module")
def msm_inputs(cuda):
    from liblightzk_b200 import synth
    n = 1 << LOG_MSM
    s = synth.random_fr(n, 31, 1)
    t = synth.random_fr(n, 31, 2)
    return n, s, t


def _check_msm_properties(orc, g, run, n, s, t):
    """linearity, equal scalars, and k = r - 1 against k = 1"""
    sh, th = _host(s), _host(t)
    u = _dev(orc.field_op(FR, ADD, sh, th))
    Rs, Rt, Ru = (_host(run(x)) for x in (s, t, u))
    op = orc.g1_op if g == 1 else orc.g2_op
    assert same_point(orc, g, op(G_ADD, Rs, Rt), Ru), "MSM(s) + MSM(t) != MSM(s + t)"

    ones = _fr_const(orc, [1, 0, 0, 0], n)
    sum_p = _host(run(_dev(ones)))
    k = orc.rand_field(FR, 1, np.array([77], np.uint64))
    Rk = _host(run(_dev(np.ascontiguousarray(np.broadcast_to(k[0], (n, 4))))))
    mul = orc.g1_mul if g == 1 else orc.g2_mul
    assert same_point(orc, g, Rk, mul(k, sum_p[None])[0]), "MSM(k, ..., k) != k * sum(P)"

    minus = _host(run(_dev(_fr_const(orc, R_MINUS_1_CANON, n))))
    assert same_point(orc, g, minus, op(G_NEG, sum_p)), "MSM(r-1, ..., r-1) != -sum(P)"


@pytest.mark.parametrize("precomputed", [True, False])
def test_g1_msm_2e20_properties(orc, msm_inputs, precomputed):
    from liblightzk_b200 import msm, synth
    n, s, t = msm_inputs
    bases = synth.fixed_base(1, synth.random_fr(n, 31, 3))
    if precomputed:
        c = 16
        W = msm.windows_for(c)
        table = msm.precompute(1, bases, c, W, n)
        run = lambda x: msm.msm_precomputed(1, x, table, c, W, n)  # noqa: E731
    else:
        run = lambda x: msm.msm(1, x, bases, window_bits=13)  # noqa: E731
    _check_msm_properties(orc, 1, run, n, s, t)


def test_g2_msm_2e20_properties(orc, msm_inputs):
    from liblightzk_b200 import msm, synth
    n, s, t = msm_inputs
    bases = synth.fixed_base(2, synth.random_fr(n, 31, 4))
    c = 16
    W = msm.windows_for(c)
    table = msm.precompute(2, bases, c, W, n)
    _check_msm_properties(orc, 2, lambda x: msm.msm_precomputed(2, x, table, c, W, n), n, s, t)


def test_ntt_2e24_properties(cuda, orc):
    import torch

    from liblightzk_b200 import ntt, synth
    n = 1 << LOG_NTT
    a = synth.random_fr(n, 41, 1)
    b = synth.random_fr(n, 41, 2)
    # round trips in both domains
    for fwd, inv in ((ntt.FORWARD, ntt.INVERSE), (ntt.COSET_FORWARD, ntt.COSET_INVERSE)):
        x = a.clone()
        ntt.ntt(x, LOG_NTT, fwd)
        assert not torch.equal(x, a)
        ntt.ntt(x, LOG_NTT, inv)
        assert torch.equal(x, a), f"round trip {fwd}->{inv}"
    del a, b
    # linearity of the coset transform (2^22: 128 MB vectors, still far above L2)
    k = LOG_NTT - 2
    a = synth.random_fr(1 << k, 41, 3)
    b = synth.random_fr(1 << k, 41, 4)
    c = _dev(orc.field_op(FR, ADD, _host(a), _host(b)))
    for x in (a, b, c):
        ntt.ntt(x, k, ntt.COSET_FORWARD)
    assert (orc.field_op(FR, ADD, _host(a), _host(b)) == _host(c)).all(), "NTT(a) + NTT(b) != NTT(a + b)"
    del a, b, c
    # e_1 -> powers of the root of unity w (forward), g * w^j (coset, g = 5)
    one = _fr_const(orc, [1, 0, 0, 0], 1)[0]
    e1 = np.zeros((n, 4), np.uint64)
    e1[1] = one
    x = _dev(e1)
    ntt.ntt(x, LOG_NTT, ntt.FORWARD)
    w = _host(x)
    assert (w[0] == one).all()
    assert (w[n // 2] == orc.field_op(FR, NEG, one[None])[0]).all(), "w^(n/2) != -1"
    step = np.ascontiguousarray(np.broadcast_to(w[1], (n - 1, 4)))
    assert (orc.field_op(FR, MUL, w[:-1], step) == w[1:]).all(), "outputs are not successive powers of w"
    y = _dev(e1)
    ntt.ntt(y, LOG_NTT, ntt.COSET_FORWARD)
    g = _fr_const(orc, [5, 0, 0, 0], n)
    assert (orc.field_op(FR, MUL, w, g) == _host(y)).all(), "coset outputs are not g * w^j"


def test_groth16_2e20(cuda, orc):
    import torch

    from liblightzk_b200 import groth16, msm, ntt, synth
    log_m = 20
    circ = synth.Circuit(log_m, seed=1, n_public=1, n_free=4096, block=4096)
    z = circ.witness(11)
    assert circ.unsatisfied_rows(z) == 0
    zh = _host(z)
    mats = [m.host() for m in circ.mats]

    # R1CS products at full size, bit for bit against the oracle's SpMV
    outs = [torch.zeros((circ.M, 4), dtype=torch.int64, device=z.device) for _ in range(3)]
    ntt.spmv3(circ.A.desc(), circ.B.desc(), circ.C.desc(), z, *outs)
    for (val, col, rp), o in zip(mats, outs):
        assert (orc.spmv(val, col, rp[:-1], zh) == _host(o)).all(), "SpMV differs from the oracle"
    del outs

    pk = synth.ProvingKey(circ, seed=12)
    r, s = orc.rand_field(FR, 2, np.array([13], np.uint64))
    prover = groth16.Prover(circ, pk, mode=groth16.STANDARD, window_bits=16)
    A, B, C = groth16.split_proof(prover.prove(z, r, s))
    # the same request again: the same points (the Jacobian representation may
    # differ, as the order of additions inside a bucket follows the sort's atomics)
    A2, B2, C2 = groth16.split_proof(prover.prove(z, r, s))
    assert same_point(orc, 1, A, A2) and same_point(orc, 2, B, B2) and same_point(orc, 1, C, C2)

    # independent composition: oracle H chain + plain-bases MSMs (c = 13) + oracle Phase 6
    h = orc.groth16_h(mats, circ.M, circ.n_vars, circ.n_public, log_m, zh, 0)
    hd = _dev(h)
    npub = circ.n_public
    g1res = np.stack([_host(msm.msm(1, z, pk.a, window_bits=13)),
                      _host(msm.msm(1, z, pk.b1, window_bits=13)),
                      _host(msm.msm(1, z[npub + 1:], pk.l, window_bits=13)),
                      _host(msm.msm(1, hd, pk.h, window_bits=13))])
    g2res = _host(msm.msm(2, z, pk.b2, window_bits=13))
    jac1 = [orc.aff_to_jac(1, _host(p)[None])[0] for p in (pk.alpha1, pk.beta1, pk.delta1)]
    jac2 = [orc.aff_to_jac(2, _host(p)[None])[0] for p in (pk.beta2, pk.delta2)]
    og1, og2 = orc.groth16_assemble(*jac1, *jac2, g1res, g2res, r, s)
    assert same_point(orc, 1, A, og1[0]), "proof A"
    assert same_point(orc, 2, B, og2), "proof B"
    assert same_point(orc, 1, C, og1[1]), "proof C"
    prover.close()
