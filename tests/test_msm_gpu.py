"""MSM parity: the CUDA Pippenger (lzk_msm_g1/_g2 through the C ABI) against
the oracle's sum_i s_i * P_i, compared after affine normalisation, in the
manner of the reference's test/msm-check.cu:45-58 (there: GPU result ==
naive CPU sum).  Seeded inputs; edge cases the reference's MSM must handle:
zero/one/-1 scalars, digits at the signed threshold, repeated bases
(doubling inside a bucket), P and -P (cancellation), points at infinity,
n = 0 and 1, every window width the autotuner can pick."""
import numpy as np
import pytest

from helpers import bases, edge_scalars, same_point, scalars

pytestmark = pytest.mark.gpu


def _run(g, s, b, c=0):
    from liblightzk_b200 import device, msm
    out = msm.msm(g, device.to_device(s), device.to_device(b), window_bits=c)
    return device.to_host(out)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 1000, 4096])
def test_g1_random(cuda, orc, rng_state, n):
    s, b = scalars(orc, n, rng_state), bases(orc, 1, n, rng_state)
    assert same_point(orc, 1, _run(1, s, b), orc.msm(1, s, b))


def test_g1_config1_2e16(cuda, orc, rng_state):
    """n = 2^16: scalars uniform Fr, bases k_i*G, k_i from the same seed"""
    n = 1 << 16
    s, b = scalars(orc, n, rng_state), bases(orc, 1, n, rng_state)
    assert same_point(orc, 1, _run(1, s, b), orc.msm(1, s, b))


@pytest.mark.parametrize("c", [2, 3, 4, 5, 6, 7, 8, 12, 13, 16, 17, 20])
def test_g1_window_widths(cuda, orc, rng_state, c):
    n = 777
    s, b = scalars(orc, n, rng_state), bases(orc, 1, n, rng_state)
    assert same_point(orc, 1, _run(1, s, b, c), orc.msm(1, s, b))


def test_g1_edge_scalars(cuda, orc, rng_state):
    e = edge_scalars(orc)
    b = bases(orc, 1, len(e), rng_state)
    assert same_point(orc, 1, _run(1, e, b), orc.msm(1, e, b, naive=True))
    for c in (4, 12, 16):
        assert same_point(orc, 1, _run(1, e, b, c), orc.msm(1, e, b, naive=True))


def test_g1_repeated_and_cancelling(cuda, orc, rng_state):
    n = 512
    one_base = np.repeat(bases(orc, 1, 1, rng_state), n, axis=0)
    s = scalars(orc, n, rng_state)
    s[: n // 2] = s[0]                     # same scalar, same base: doubling in every bucket
    assert same_point(orc, 1, _run(1, s, one_base), orc.msm(1, s, one_base))
    b = bases(orc, 1, 2, rng_state)
    negb = b.copy()
    from oracle import FQ, NEG
    negb[1, 1] = orc.field_op(FQ, NEG, b[0, 1])   # -P0
    negb[1, 0] = b[0, 0]
    s2 = np.repeat(scalars(orc, 1, rng_state), 2, axis=0)   # s*P + s*(-P) = O
    r = _run(1, s2, negb)
    assert orc.jac_to_aff(1, r[None]).sum() == 0


def test_g1_infinity_bases_and_zero_n(cuda, orc, rng_state):
    n = 300
    s, b = scalars(orc, n, rng_state), bases(orc, 1, n, rng_state)
    b[::7] = 0                              # points at infinity
    assert same_point(orc, 1, _run(1, s, b), orc.msm(1, s, b))
    s0 = np.zeros((n, 4), np.uint64)        # all-zero scalars -> infinity
    assert orc.jac_to_aff(1, _run(1, s0, b)[None]).sum() == 0


def test_g1_empty(cuda, orc):
    import torch
    from liblightzk_b200 import device, msm
    z = torch.zeros((0, 4), dtype=torch.int64, device="cuda")
    bz = torch.zeros((0, 2, 4), dtype=torch.int64, device="cuda")
    out = device.to_host(msm.msm(1, z, bz))
    assert orc.jac_to_aff(1, out[None]).sum() == 0


@pytest.mark.parametrize("c", [8, 12, 16, 17])
def test_g1_precomputed(cuda, orc, rng_state, c):
    from liblightzk_b200 import device, msm
    n = 3000
    s, b = scalars(orc, n, rng_state), bases(orc, 1, n, rng_state)
    W = msm.windows_for(c)
    stride = n + 5
    table = msm.precompute(1, device.to_device(b), c, W, stride)
    out = device.to_host(msm.msm_precomputed(1, device.to_device(s), table, c, W, stride))
    assert same_point(orc, 1, out, orc.msm(1, s, b))
    # the table itself: copy j is 2^(j c) * P_i
    t = device.to_host(table)
    from oracle import G_EQ
    j = W - 1
    two = np.zeros((1, 4), np.uint64)
    k = orc.to_mont(0, np.array([[0, 0, 0, 0]], np.uint64))
    canon = np.zeros(4, np.uint64)
    bit = j * c
    canon[bit // 64] = np.uint64(1) << np.uint64(bit % 64)
    k = orc.to_mont(0, canon[None])
    P = orc.aff_to_jac(1, b[:4])
    expect = orc.g1_mul(np.repeat(k, 4, axis=0), P)
    got = orc.aff_to_jac(1, t[j * stride: j * stride + 4])
    assert (orc.g1_op(G_EQ, expect, got) == 1).all()
    del two


@pytest.mark.parametrize("n", [1, 5, 64, 1024])
def test_g2_random(cuda, orc, rng_state, n):
    s, b = scalars(orc, n, rng_state), bases(orc, 2, n, rng_state)
    assert same_point(orc, 2, _run(2, s, b), orc.msm(2, s, b))


@pytest.mark.parametrize("c", [2, 6, 7, 11])
def test_g2_window_widths(cuda, orc, rng_state, c):
    n = 300
    s, b = scalars(orc, n, rng_state), bases(orc, 2, n, rng_state)
    assert same_point(orc, 2, _run(2, s, b, c), orc.msm(2, s, b))


def test_g2_precomputed_c17(cuda, orc, rng_state):
    """the prover's width: one bucket set of 2^16 for all 15 windows"""
    from liblightzk_b200 import device, msm
    n, c = 2000, 17
    s, b = scalars(orc, n, rng_state), bases(orc, 2, n, rng_state)
    W = msm.windows_for(c)
    table = msm.precompute(2, device.to_device(b), c, W, n)
    out = device.to_host(msm.msm_precomputed(2, device.to_device(s), table, c, W, n))
    assert same_point(orc, 2, out, orc.msm(2, s, b))


def test_g2_edges_and_precomputed(cuda, orc, rng_state):
    from liblightzk_b200 import device, msm
    e = edge_scalars(orc)
    b = bases(orc, 2, len(e), rng_state)
    assert same_point(orc, 2, _run(2, e, b), orc.msm(2, e, b, naive=True))
    n = 700
    s, b = scalars(orc, n, rng_state), bases(orc, 2, n, rng_state)
    c = 10
    W = msm.windows_for(c)
    table = msm.precompute(2, device.to_device(b), c, W, n)
    out = device.to_host(msm.msm_precomputed(2, device.to_device(s), table, c, W, n))
    assert same_point(orc, 2, out, orc.msm(2, s, b))


def test_to_affine(cuda, orc, rng_state):
    from liblightzk_b200 import device, msm
    n = 37
    k = scalars(orc, n, rng_state)
    P = orc.g1_mul(k, np.repeat(orc.g1_one()[None], n, axis=0))
    P[3] = [[0] * 4, orc.g1_one()[1], [0] * 4]   # infinity
    got = device.to_host(msm.to_affine(1, device.to_device(P)))
    assert (got == orc.jac_to_aff(1, P)).all()
    Q = orc.g2_mul(k, np.repeat(orc.g2_one()[None], n, axis=0))
    got2 = device.to_host(msm.to_affine(2, device.to_device(Q)))
    assert (got2 == orc.jac_to_aff(2, Q)).all()
