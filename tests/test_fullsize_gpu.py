"""Parity at the benchmark's full sizes, against the oracle:

* G1 MSM at 2^20 (shifted-copy table at the prover's window, and plain
  bases at the autotuned window) and G2 MSM at 2^20 (table): equal to the
  oracle's bucket-method MSM (test/msm-check.cu:45-58 checks the reference
  the same way, GPU against CPU at 2^20), and to a second, independent
  oracle route: the bases are k_i * G for known k_i, so sum_i s_i P_i =
  (sum_i s_i k_i mod r) * G, one field dot product and one scalar product
  on the CPU.  The size-independent properties (linearity, equal scalars in
  one bucket per window, r - 1 against 1) are anchored the same way, so a
  result that is wrong in a consistent way (the point at infinity for every
  input, say) cannot satisfy them;
* coset NTT and inverse coset NTT at 2^24, element for element against the
  oracle's transform (poly.cuh:32-73 restated, coset g = 5), plus round
  trips and the transform of x;
* Groth16 at 2^20 constraints in both modes: the synthetic benchmark
  circuit in standard mode and the reference's own MatMul p = 100 circuit
  in the reference-compatible mode (the 2M-domain H chain of
  groth16.cuh:159-198), each proof equal to the oracle's whole proof (its
  SpMV, H chain, five MSMs and Phase 6 of groth16.cuh:209-215); and the
  three SpMV outputs bit for bit.

Point results are compared after affine normalisation."""
import numpy as np
import pytest

from helpers import R_MINUS_1_CANON, same_point
from oracle import ADD, FR, G_ADD, G_NEG, MUL

pytestmark = pytest.mark.gpu

LOG_MSM = 20
LOG_NTT = 24
PROVER_WINDOW = 17


def _host(t):
    from liblightzk_b200 import device
    return device.to_host(t)


def _dev(a):
    from liblightzk_b200 import device
    return device.to_device(a)


def _fr_const(orc, canon, n):
    v = orc.to_mont(FR, np.array([canon], np.uint64))[0]
    return np.ascontiguousarray(np.broadcast_to(v, (n, 4)))


def _fr_sum(orc, x):
    """sum of the rows of x in Fr (pairwise tree over oracle additions)"""
    x = np.ascontiguousarray(x)
    while x.shape[0] > 1:
        if x.shape[0] & 1:
            x = np.concatenate([x, np.zeros((1, 4), np.uint64)])
        x = orc.field_op(FR, ADD, x[0::2], x[1::2])
    return x


def _dlog_msm(orc, g, s, k):
    """(sum_i s_i k_i) * G on the CPU: the MSM of s over the bases k_i * G"""
    dot = _fr_sum(orc, orc.field_op(FR, MUL, s, k))
    gen = orc.g1_one() if g == 1 else orc.g2_one()
    mul = orc.g1_mul if g == 1 else orc.g2_mul
    return mul(dot, gen[None])[0]


@pytest.fixture(scope="module")
def msm_inputs(cuda):
    from liblightzk_b200 import synth
    n = 1 << LOG_MSM
    s = synth.random_fr(n, 31, 1)
    t = synth.random_fr(n, 31, 2)
    return n, s, t


def _check_msm(orc, g, runs, n, s, t, k_dev, bases_dev):
    """every run (a callable scalars -> Jacobian result) against the oracle"""
    sh, th, kh = _host(s), _host(t), _host(k_dev)
    bh = _host(bases_dev)
    want = orc.msm(g, sh, bh)
    assert same_point(orc, g, want, _dlog_msm(orc, g, sh, kh)), "the two oracle routes disagree"
    ones = _fr_const(orc, [1, 0, 0, 0], n)
    sum_p = _dlog_msm(orc, g, ones, kh)
    op = orc.g1_op if g == 1 else orc.g2_op
    mul = orc.g1_mul if g == 1 else orc.g2_mul
    u = orc.field_op(FR, ADD, sh, th)
    k = orc.rand_field(FR, 1, np.array([77], np.uint64))
    for run in runs:
        assert same_point(orc, g, _host(run(s)), want), "MSM(s) differs from the oracle"
        Rt = _host(run(t))
        assert same_point(orc, g, op(G_ADD, want, Rt), _host(run(_dev(u)))), "MSM(s) + MSM(t) != MSM(s + t)"
        assert same_point(orc, g, _host(run(_dev(ones))), sum_p), "MSM(1, ..., 1) != sum of the bases"
        Rk = _host(run(_dev(np.ascontiguousarray(np.broadcast_to(k[0], (n, 4))))))
        assert same_point(orc, g, Rk, mul(k, sum_p[None])[0]), "MSM(k, ..., k) != k * sum(P)"
        minus = _host(run(_dev(_fr_const(orc, R_MINUS_1_CANON, n))))
        assert same_point(orc, g, minus, op(G_NEG, sum_p)), "MSM(r-1, ..., r-1) != -sum(P)"


def test_g1_msm_2e20_against_oracle(orc, msm_inputs):
    from liblightzk_b200 import msm, synth
    n, s, t = msm_inputs
    k = synth.random_fr(n, 31, 3)
    bases = synth.fixed_base(1, k)
    c = PROVER_WINDOW
    W = msm.windows_for(c)
    table = msm.precompute(1, bases, c, W, n)
    runs = [lambda x: msm.msm_precomputed(1, x, table, c, W, n),
            lambda x: msm.msm(1, x, bases)]
    _check_msm(orc, 1, runs, n, s, t, k, bases)


def test_g2_msm_2e20_against_oracle(orc, msm_inputs):
    from liblightzk_b200 import msm, synth
    n, s, t = msm_inputs
    k = synth.random_fr(n, 31, 4)
    bases = synth.fixed_base(2, k)
    c = PROVER_WINDOW
    W = msm.windows_for(c)
    table = msm.precompute(2, bases, c, W, n)
    _check_msm(orc, 2, [lambda x: msm.msm_precomputed(2, x, table, c, W, n)], n, s, t, k, bases)


def test_coset_ntt_2e24_against_oracle(cuda, orc):
    import torch

    from liblightzk_b200 import ntt, synth
    n = 1 << LOG_NTT
    a = synth.random_fr(n, 41, 1)
    ah = _host(a)
    for d, od in ((ntt.COSET_FORWARD, 2), (ntt.COSET_INVERSE, 3)):
        x = a.clone()
        ntt.ntt(x, LOG_NTT, d)
        assert (_host(x) == orc.ntt(ah, LOG_NTT, od)).all(), f"direction {d} differs from the oracle"
        del x
    # round trips in both domains
    for fwd, inv in ((ntt.FORWARD, ntt.INVERSE), (ntt.COSET_FORWARD, ntt.COSET_INVERSE)):
        x = a.clone()
        ntt.ntt(x, LOG_NTT, fwd)
        ntt.ntt(x, LOG_NTT, inv)
        assert torch.equal(x, a), f"round trip {fwd}->{inv}"
        del x
    del a
    # e_1 -> successive powers of the root of unity of the oracle's table
    one = _fr_const(orc, [1, 0, 0, 0], 1)[0]
    e1 = np.zeros((n, 4), np.uint64)
    e1[1] = one
    x = _dev(e1)
    ntt.ntt(x, LOG_NTT, ntt.FORWARD)
    w = _host(x)
    assert (w[1] == orc.ntt_table(0, LOG_NTT)).all(), "X_1 is not the table's root of unity"
    step = np.ascontiguousarray(np.broadcast_to(w[1], (n - 1, 4)))
    assert (orc.field_op(FR, MUL, w[:-1], step) == w[1:]).all(), "outputs are not successive powers of w"


def _keys(pk):
    return {"a_query": _host(pk.a), "b1_query": _host(pk.b1), "b2_query": _host(pk.b2), "l_query": _host(pk.l),
            "h_query": _host(pk.h), "alpha1": _host(pk.alpha1), "beta1": _host(pk.beta1),
            "delta1": _host(pk.delta1), "beta2": _host(pk.beta2), "delta2": _host(pk.delta2)}


def _prove_against_oracle(orc, circ, pk, z, mode, seed):
    from liblightzk_b200 import groth16
    r, s = orc.rand_field(FR, 2, np.array([seed], np.uint64))
    prover = groth16.Prover(circ, pk, mode=mode, window_bits=PROVER_WINDOW)
    A, B, C = groth16.split_proof(prover.prove(z, r, s))
    # the same request again: the same points (the Jacobian representation may
    # differ, as the order of additions inside a bucket follows the sort's atomics)
    A2, B2, C2 = groth16.split_proof(prover.prove(z, r, s))
    assert same_point(orc, 1, A, A2) and same_point(orc, 2, B, B2) and same_point(orc, 1, C, C2)
    prover.close()
    mats = [m.host() for m in circ.mats]
    eA, eB, eC = orc.groth16_prove(mats, circ.M, circ.n_vars, circ.n_public, circ.log_m, _keys(pk), _host(z),
                                   r, s, mode)
    assert same_point(orc, 1, A, eA), "proof A differs from the oracle"
    assert same_point(orc, 2, B, eB), "proof B differs from the oracle"
    assert same_point(orc, 1, C, eC), "proof C differs from the oracle"


def test_groth16_2e20_standard_against_oracle(cuda, orc):
    import torch

    from liblightzk_b200 import groth16, ntt, synth
    circ = synth.Circuit(20, seed=1)
    z = circ.witness(11)
    assert circ.unsatisfied_rows(z) == 0
    zh = _host(z)
    # R1CS products at full size, bit for bit against the oracle's SpMV
    outs = [torch.zeros((circ.M, 4), dtype=torch.int64, device=z.device) for _ in range(3)]
    ntt.spmv3(circ.A.desc(), circ.B.desc(), circ.C.desc(), z, *outs)
    for (val, col, rp), o in zip((m.host() for m in circ.mats), outs):
        assert (orc.spmv(val, col, rp[:-1], zh) == _host(o)).all(), "SpMV differs from the oracle"
    del outs
    pk = synth.ProvingKey(circ, seed=12)
    _prove_against_oracle(orc, circ, pk, z, groth16.STANDARD, 13)


def test_groth16_matmul_p100_reference_mode_against_oracle(cuda, orc):
    """the reference's benchmark circuit (test/groth16.cu: MatMul_p_100, 2^20
    constraints) proved in the reference-compatible mode"""
    from liblightzk_b200 import groth16, synth
    circ = synth.MatMulCircuit(100)
    assert circ.log_m == 20
    z = circ.witness(17)
    assert circ.unsatisfied_rows(z) == 0
    pk = synth.ProvingKey(circ, seed=18)
    _prove_against_oracle(orc, circ, pk, z, groth16.REFERENCE, 19)
