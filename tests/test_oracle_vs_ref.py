"""Randomized differential checks of the C restatement against the
reference's own host arithmetic, run where the reference tree was built
(oracle/_ref/libref.so).  The same comparisons on fixed inputs are frozen
in tests/golden/ for machines without it."""
import os

import numpy as np
import pytest

from oracle import FQ, FR, G_ADD, G_DBL, G_MADD, INV, MUL, SQR, SUB

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_host_arith.npz")


@pytest.mark.parametrize("kind", [FR, FQ])
def test_field_random(orc, ref, rng_state, kind):
    a = orc.rand_field(kind, 2000, rng_state)
    b = orc.rand_field(kind, 2000, rng_state)
    for op in (SUB, MUL, SQR):
        assert (orc.field_op(kind, op, a, b) == ref.field_op(kind, op, a, b)).all()
    assert (orc.field_op(kind, INV, a[:50]) == ref.field_op(kind, INV, a[:50])).all()


def test_group_random(orc, ref, rng_state):
    k = orc.rand_field(FR, 64, rng_state)
    P = ref.g1_mul(k, np.repeat(ref.g1_one()[None], 64, axis=0))
    Q = np.roll(P, 5, axis=0)
    for op in (G_ADD, G_DBL):
        assert (orc.g1_op(op, P, Q) == ref.g1_op(op, P, Q)).all()
    A = orc.g1_op(4, Q)
    assert (orc.g1_op(G_MADD, P, A) == ref.g1_op(G_MADD, P, A)).all()
    P2 = ref.g2_mul(k[:16], np.repeat(ref.g2_one()[None], 16, axis=0))
    assert (orc.g2_mul(k[:16], np.repeat(orc.g2_one()[None], 16, axis=0)) == P2).all()


def test_msm_vs_reference_naive(orc, ref, rng_state):
    n = 500
    k = orc.rand_field(FR, n, rng_state)
    aff = orc.fixed_base(1, k)
    s = orc.rand_field(FR, n, rng_state)
    jac = orc.aff_to_jac(1, aff)
    r = ref.g1_msm_naive_jac(s, jac)
    assert (orc.jac_to_aff(1, orc.msm(1, s, aff)[None]) == orc.jac_to_aff(1, r[None])).all()


@pytest.mark.parametrize("log_m", [2, 5, 8])
def test_h_reference_chain(orc, ref, rng_state, log_m):
    """oracle H scalars in reference mode == the reference chain composed
    from the reference bridge (spmv, ntt_ref, A*B-C, scaled iNTT_2M)"""
    M = 1 << log_m
    rng = np.random.default_rng(log_m)
    nv = 3 * M
    z = orc.rand_field(FR, nv, rng_state)
    mats = []
    for _ in range(3):
        per = rng.integers(0, 4, M)
        rp = np.concatenate([[0], np.cumsum(per)[:-1]]).astype(np.uint64)
        nnz = int(per.sum())
        mats.append((orc.rand_field(FR, nnz, rng_state), rng.integers(0, nv, nnz).astype(np.uint64), rp))
    h = orc.groth16_h(mats, M, nv, 1, log_m, z, 1)
    tab = ref.ntt_setup(M)
    x = []
    for val, col, rp in mats:
        v = np.zeros((2 * M, 4), np.uint64)
        v[:M] = ref.spmv(val, col, rp, z)
        v[:M] = ref.ntt_ref(v[:M], tab[M:2 * M], tab[2 * M])
        v = ref.ntt_ref(v, tab[2 * M + 1:4 * M + 1])
        x.append(v)
    ab = ref.field_op(FR, SUB, ref.field_op(FR, MUL, x[0], x[1]), x[2])
    hh = ref.ntt_ref(ab, tab[4 * M + 1:6 * M + 1], tab[6 * M + 1])
    assert (h == hh[M + 1:]).all()


def test_assemble_golden(orc):
    g = np.load(GOLD)
    og1, og2 = orc.groth16_assemble(g["asm_alpha1"], g["asm_beta1"], g["asm_delta1"], g["asm_beta2"],
                                    g["asm_delta2"], g["asm_g1res"], g["asm_g2res"], g["asm_r"], g["asm_s"])
    for a, b in zip(og1, g["asm_out_g1"]):
        assert (orc.jac_to_aff(1, a[None]) == orc.jac_to_aff(1, b[None])).all()
    assert (orc.jac_to_aff(2, og2[None]) == orc.jac_to_aff(2, g["asm_out_g2"][None])).all()
