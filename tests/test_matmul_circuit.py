"""The reference's benchmark circuit, the product Z = X Y of two p x p
matrices (xpu-spmat.cuh:33-65; input scales MatMul_p_39/63/100 of
groth16.cuh:11-46), rebuilt by synth.MatMulCircuit in the reference's CSR
layout.  On the CPU: its structure, and that a witness solved with the
oracle satisfies every row.  On the GPU: the device witness solver gives the
same witness, and Groth16 proofs on the circuit equal the oracle's in both
modes."""
import numpy as np
import pytest

from helpers import same_point
from oracle import ADD, FR, MUL


def _host(t):
    from liblightzk_b200 import device
    return device.to_host(t)


def _expected_witness(orc, p, xy):
    """z = (1, X, Y, Z, t) with t_(i1 p^2 + i2 p + i3) = X[i2 p + i1] Y[i1 p + i3]
    and Z[r] = sum_k t_(k p^2 + r), from X, Y = xy (Montgomery limbs)"""
    p2, p3 = p * p, p ** 3
    X, Y = xy[:p2], xy[p2:2 * p2]
    i = np.arange(p3)
    i1, i2, i3 = i // p2, (i % p2) // p, i % p
    t = orc.field_op(FR, MUL, X[i2 * p + i1], Y[i1 * p + i3])
    Z = t[:p2].copy()
    for k in range(1, p):
        Z = orc.field_op(FR, ADD, Z, t[k * p2:(k + 1) * p2])
    one = orc.to_mont(FR, np.array([[1, 0, 0, 0]], np.uint64))
    return np.concatenate([one, X, Y, Z, t])


def test_matmul_structure_and_semantics(orc):
    from liblightzk_b200 import synth
    p = 5
    c = synth.MatMulCircuit(p, device="cpu")
    p2, p3 = p * p, p ** 3
    assert (c.M, c.log_m, c.n_public, c.n_vars) == (256, 8, 3 * p2, 1 + 3 * p2 + p3)
    (av, ac, ar), (bv, bc, br), (cv, cc, cr) = (m.host() for m in c.mats)
    # the reference's sizes: A holds 2 p^3 entries, B and C p^3 + p^2; M offsets each
    assert (ac.size, bc.size, cc.size) == (2 * p3, p3 + p2, p3 + p2)
    assert all(m.row_ptr.shape[0] == c.M and m.col.element_size() == 8 for m in c.mats)
    one = orc.to_mont(FR, np.array([[1, 0, 0, 0]], np.uint64))[0]
    assert all((v == one).all() for v in (av, bv, cv))
    # a sum row: A adds the p products of one output entry, B is the constant 1
    r = 7
    row = p3 + r
    assert list(ac[ar[row]:ar[row + 1]]) == [1 + 3 * p2 + k * p2 + r for k in range(p)]
    assert list(bc[br[row]:br[row + 1]]) == [0] and list(cc[cr[row]:cr[row + 1]]) == [1 + 2 * p2 + r]
    # padding rows are empty
    assert ar[-1] == ac.size and br[-1] == bc.size and ar[p3 + p2] == ac.size
    # semantics: (A z) (B z) = C z on every row for the solved witness
    xy = orc.rand_field(FR, 2 * p2, np.array([5], np.uint64))
    z = _expected_witness(orc, p, xy)
    az, bz, cz = (orc.spmv(v, col, rp[:-1], z) for v, col, rp in ((av, ac, ar), (bv, bc, br), (cv, cc, cr)))
    assert (orc.field_op(FR, MUL, az, bz) == cz).all()
    # and a wrong product breaks exactly its own row
    z[1 + 3 * p2 + 3] = orc.field_op(FR, ADD, z[1 + 3 * p2 + 3][None], one[None])[0]
    cz2 = orc.spmv(cv, cc, cr[:-1], z)
    assert (orc.field_op(FR, MUL, az, bz) != cz2).any(axis=1).sum() == 1


@pytest.mark.gpu
def test_matmul_witness_on_device(cuda, orc):
    from liblightzk_b200 import synth
    p = 6
    c = synth.MatMulCircuit(p)
    z = c.witness(21)
    assert c.unsatisfied_rows(z) == 0
    zh = _host(z)
    assert (zh == _expected_witness(orc, p, zh[1:1 + 2 * p * p])).all()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_matmul_prove_matches_oracle(cuda, orc, rng_state, mode):
    from liblightzk_b200 import groth16, synth
    circ = synth.MatMulCircuit(4)          # 80 rows -> M = 128
    z = circ.witness(22)
    pk = synth.ProvingKey(circ, seed=23)
    r, s = orc.rand_field(FR, 2, rng_state)
    prover = groth16.Prover(circ, pk, mode=mode, window_bits=8)
    A, B, C = groth16.split_proof(prover.prove(z, r, s))
    mats = [m.host() for m in circ.mats]
    keys = {"a_query": _host(pk.a), "b1_query": _host(pk.b1), "b2_query": _host(pk.b2), "l_query": _host(pk.l),
            "h_query": _host(pk.h), "alpha1": _host(pk.alpha1), "beta1": _host(pk.beta1),
            "delta1": _host(pk.delta1), "beta2": _host(pk.beta2), "delta2": _host(pk.delta2)}
    eA, eB, eC = orc.groth16_prove(mats, circ.M, circ.n_vars, circ.n_public, circ.log_m, keys, _host(z), r, s, mode)
    assert same_point(orc, 1, A, eA) and same_point(orc, 2, B, eB) and same_point(orc, 1, C, eC)
    prover.close()
