"""Device field arithmetic (lzk_field_op) against the reference's own host
arithmetic: the golden arrays of tests/golden/reference_host_arith.npz were
computed by the reference's libff code (mont_t / fp2_t semantics,
mont_t.cuh:396-430, alt_bn128_t.cuh:122-151), so every product, sum,
inverse and conversion of the device routines that the MSM, NTT and point
formulas use must equal them bit for bit: products and squares here run
through the FP64-pipe forms of field52.cuh (Fq and Fq2 through the curve
formulas' out-of-line bodies, Fr through the NTT butterflies' product).  Edge operands beyond the golden
set (0, 1, p - 1, sums at 2p - 2, Fq2 operands whose Karatsuba sums and
cross terms sit at the reduction bounds) are compared with the C oracle,
which the golden arrays pin."""
import os

import numpy as np
import pytest

from oracle import FQ, FR

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_host_arith.npz")
P_CANON = {FR: [0x43E1F593F0000001, 0x2833E84879B97091, 0xB85045B68181585D, 0x30644E72E131A029],
           FQ: [0x3C208C16D87CFD47, 0x97816A916871CA8D, 0xB85045B68181585D, 0x30644E72E131A029]}


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _op(field, op, a, b=None):
    from liblightzk_b200 import device
    from liblightzk_b200.field import field_op
    da = device.to_device(np.ascontiguousarray(a))
    db = None if b is None else device.to_device(np.ascontiguousarray(b))
    return device.to_host(field_op(field, op, da, db))


def _lzk_field(kind):
    from liblightzk_b200 import field
    return field.FR if kind == FR else field.FQ


@pytest.mark.parametrize("kind,name", [(FR, "fr"), (FQ, "fq")])
def test_prime_field_ops_match_reference(cuda, golden, kind, name):
    from liblightzk_b200 import field as F
    f = _lzk_field(kind)
    a, b = golden[f"{name}_a"], golden[f"{name}_b"]
    for op, key in ((F.ADD, "add"), (F.SUB, "sub"), (F.MUL, "mul"), (F.SQR, "sqr"), (F.NEG, "neg"),
                    (F.FROM_MONT, "from_mont")):
        got = _op(f, op, a, b if op in (F.ADD, F.SUB, F.MUL) else None)
        assert (got == golden[f"{name}_{key}"]).all(), f"{name} {key}"
    assert (_op(f, F.INV, golden[f"{name}_inv_in"]) == golden[f"{name}_inv"]).all(), f"{name} inv"
    assert (_op(f, F.TO_MONT, golden[f"{name}_to_mont_in"]) == golden[f"{name}_to_mont"]).all(), f"{name} to_mont"


def test_fq2_ops_match_reference(cuda, golden):
    from liblightzk_b200 import field as F
    a, b = golden["fq2_a"], golden["fq2_b"]
    for op, key in ((F.ADD, "add"), (F.SUB, "sub"), (F.MUL, "mul"), (F.SQR, "sqr"), (F.NEG, "neg"),
                    (F.INV, "inv")):
        got = _op(F.FQ2, op, a, b if op in (F.ADD, F.SUB, F.MUL) else None)
        assert (got == golden[f"fq2_{key}"]).all(), f"fq2 {key}"


def _edge_values(orc, kind):
    """Montgomery forms of 0, 1, 2, p - 1, p - 2, (p - 1) / 2, (p + 1) / 2,
    2^255 mod p's neighbours and a few values with all-ones / all-zero limbs"""
    p = P_CANON[kind]
    pint = sum(v << (64 * i) for i, v in enumerate(p))
    vals = [0, 1, 2, pint - 1, pint - 2, (pint - 1) // 2, (pint + 1) // 2, (1 << 254) % pint,
            (1 << 253) - 1, (1 << 64) - 1, (1 << 128) - 1, (1 << 192) - 1, pint - (1 << 64)]
    canon = np.array([[(v >> (64 * i)) & ((1 << 64) - 1) for i in range(4)] for v in vals], np.uint64)
    return orc.to_mont(kind, canon), canon


@pytest.mark.parametrize("kind", [FR, FQ])
def test_prime_field_edges_and_random(cuda, orc, kind):
    from liblightzk_b200 import field as F
    f = _lzk_field(kind)
    em, ec = _edge_values(orc, kind)
    # every pair of edge values, plus random operands
    ia, ib = np.meshgrid(np.arange(len(em)), np.arange(len(em)), indexing="ij")
    rnd = orc.rand_field(kind, 20000, np.array([91 + kind], np.uint64))
    a = np.concatenate([em[ia.ravel()], rnd[:10000]])
    b = np.concatenate([em[ib.ravel()], rnd[10000:]])
    from oracle import ADD, FROM_MONT, INV, MUL, NEG, SQR, SUB, TO_MONT
    for op, oop in ((F.ADD, ADD), (F.SUB, SUB), (F.MUL, MUL)):
        assert (_op(f, op, a, b) == orc.field_op(kind, oop, a, b)).all(), f"field {kind} op {op}"
    for op, oop in ((F.SQR, SQR), (F.NEG, NEG), (F.INV, INV), (F.FROM_MONT, FROM_MONT)):
        assert (_op(f, op, a) == orc.field_op(kind, oop, a)).all(), f"field {kind} op {op}"
    assert (_op(f, F.TO_MONT, ec) == em).all()
    assert (_op(f, F.FROM_MONT, em) == ec).all()
    assert (_op(f, F.TO_MONT, orc.field_op(kind, FROM_MONT, rnd)) == rnd).all()


def test_fq2_edges_and_random(cuda, orc):
    """Fq2 operands built from the Fq edge values: with a0 = a1 = b0 = b1 =
    p - 1 the Karatsuba operand sums reach 2p - 2 and the cross term
    (a0 + a1)(b0 + b1) - a0 b0 - a1 b1 its maximum; with zero or equal halves
    the borrows of c0 = a0 b0 + p^2 - a1 b1 take every value"""
    from liblightzk_b200 import field as F
    em, _ = _edge_values(orc, FQ)
    k = len(em)
    idx = np.array([(i, j) for i in range(k) for j in range(k)])
    pairs = np.stack([em[idx[:, 0]], em[idx[:, 1]]], axis=1)          # (k^2, 2, 4)
    m = pairs.shape[0]
    ia, ib = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    sel = np.random.default_rng(5).choice(m * m, 6000, replace=False)
    a = pairs[ia.ravel()[sel]]
    b = pairs[ib.ravel()[sel]]
    rnd = orc.rand_field(FQ, 4 * 4000, np.array([97], np.uint64)).reshape(-1, 2, 2, 4)
    a = np.concatenate([a, pairs, rnd[:, 0]])
    b = np.concatenate([b, pairs[::-1], rnd[:, 1]])
    for op in (F.ADD, F.SUB, F.MUL):
        assert (_op(F.FQ2, op, a, b) == orc.fq2_op(op, a, b)).all(), f"fq2 op {op}"
    for op in (F.SQR, F.NEG, F.INV):
        assert (_op(F.FQ2, op, a) == orc.fq2_op(op, a)).all(), f"fq2 op {op}"
