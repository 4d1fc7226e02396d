"""Shared test helpers: seeded inputs and point comparison after affine
normalisation (bit-exactness is defined on canonical affine coordinates)."""
import numpy as np

from oracle import FR

R_MINUS_1_CANON = [0x43E1F593F0000000, 0x2833E84879B97091, 0xB85045B68181585D, 0x30644E72E131A029]


def scalars(orc, n, state):
    return orc.rand_field(FR, n, state)


def bases(orc, g, n, state):
    """affine k_i * G with k_i uniform Fr from the same stream"""
    return orc.fixed_base(g, orc.rand_field(FR, n, state))


def edge_scalars(orc):
    """0, 1, 2, r-1, 2^253, a value with all window digits at the signed
    threshold, and a few small ones; returned in Montgomery form"""
    canon = [
        [0, 0, 0, 0], [1, 0, 0, 0], [2, 0, 0, 0], R_MINUS_1_CANON,
        [0, 0, 0, 1 << 61], [0x8000800080008000] * 3 + [0x0000800080008000],
        [0xFFFF, 0, 0, 0], [0x10000, 0, 0, 0], [0x7FFF, 0, 0, 0], [0x8000, 0, 0, 0],
        [0xFFFFFFFFFFFFFFFF, 0xFFFFFFFFFFFFFFFF, 0, 0],
    ]
    return orc.to_mont(FR, np.array(canon, np.uint64))


def same_point(orc, g, a, b):
    """a, b Jacobian (3,...) arrays; equal as group elements"""
    A = orc.jac_to_aff(g, np.asarray(a, np.uint64)[None])
    B = orc.jac_to_aff(g, np.asarray(b, np.uint64)[None])
    return bool((A == B).all())
