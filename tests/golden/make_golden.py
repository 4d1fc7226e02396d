"""Generate the golden fixtures under tests/golden/ by running the
reference's OWN host arithmetic (oracle/_ref/libref.so, compiled from the
reference tree by oracle/Makefile) on seeded inputs.

    make -C oracle && python tests/golden/make_golden.py

The reference ships no golden vectors or known-answer tests (all of its
tests are unseeded randomized differential checks), so these fixtures are
the pin: tests/test_oracle_golden.py checks the C restatement in oracle/
against them on machines where the reference tree is absent.

Inputs are drawn with the oracle's SplitMix64 stream and the rejection
sampling of Fp_model::random_element (fp.cuh:789-816); every output comes
from the reference library.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import (ADD, FQ, FR, G_ADD, G_AFF, G_DBL, G_MADD, G_NEG, G_WF, INV, MUL, NEG, SQR, SUB,  # noqa: E402
                    FROM_MONT, TO_MONT, Oracle, Ref)

R_CANON = [0x43E1F593F0000001, 0x2833E84879B97091, 0xB85045B68181585D, 0x30644E72E131A029]
Q_CANON = [0x3C208C16D87CFD47, 0x97816A916871CA8D, 0xB85045B68181585D, 0x30644E72E131A029]


def main():
    ref = Ref()
    orc = Oracle()   # used only as the seeded input generator
    st = np.array([20240601], np.uint64)
    out = {}

    # ---- fields: random operands + edge values (0, 1, p-1, 2) ----
    for kind, name, canon in ((FR, "fr", R_CANON), (FQ, "fq", Q_CANON)):
        a = orc.rand_field(kind, 48, st)
        b = orc.rand_field(kind, 48, st)
        pm1 = np.array([canon], np.uint64); pm1[0, 0] -= np.uint64(1)
        edge_c = np.concatenate([np.zeros((1, 4), np.uint64), np.array([[1, 0, 0, 0], [2, 0, 0, 0]], np.uint64), pm1])
        edge = ref.field_op(kind, TO_MONT, edge_c)
        a = np.concatenate([a, edge, edge]); b = np.concatenate([b, edge, edge[::-1]])
        out[f"{name}_a"], out[f"{name}_b"] = a, b
        for op, on in ((ADD, "add"), (SUB, "sub"), (MUL, "mul"), (SQR, "sqr"), (NEG, "neg"), (FROM_MONT, "from_mont")):
            out[f"{name}_{on}"] = ref.field_op(kind, op, a, b)
        nz = a[~(a == 0).all(axis=1)]
        out[f"{name}_inv_in"] = nz
        out[f"{name}_inv"] = ref.field_op(kind, INV, nz)
        out[f"{name}_to_mont_in"] = edge_c
        out[f"{name}_to_mont"] = ref.field_op(kind, TO_MONT, edge_c)
    a = orc.rand_field(FQ, 64, st).reshape(32, 2, 4)
    b = orc.rand_field(FQ, 64, st).reshape(32, 2, 4)
    out["fq2_a"], out["fq2_b"] = a, b
    for op, on in ((0, "add"), (1, "sub"), (2, "mul"), (3, "sqr"), (4, "neg"), (5, "inv")):
        out[f"fq2_{on}"] = ref.fq2_op(op, a, b)

    # ---- groups: scalar multiples of the generators, Jacobian ops ----
    for g, one, mul, op in ((1, ref.g1_one(), ref.g1_mul, ref.g1_op), (2, ref.g2_one(), ref.g2_mul, ref.g2_op)):
        k = orc.rand_field(FR, 24, st)
        edge_k = ref.field_op(FR, TO_MONT, np.array([[0, 0, 0, 0], [1, 0, 0, 0], [2, 0, 0, 0],
                                                      [R_CANON[0] - 1] + R_CANON[1:]], np.uint64))
        k = np.concatenate([k, edge_k])
        G = np.repeat(one[None], len(k), axis=0)
        P = mul(k, G)
        Q = np.roll(P, 3, axis=0)
        out[f"g{g}_one"] = one
        out[f"g{g}_k"] = k
        out[f"g{g}_kG"] = P
        out[f"g{g}_add"] = op(G_ADD, P, Q)
        out[f"g{g}_add_self"] = op(G_ADD, P, P)
        out[f"g{g}_dbl"] = op(G_DBL, P)
        out[f"g{g}_neg"] = op(G_NEG, P)
        out[f"g{g}_aff"] = op(G_AFF, P)
        out[f"g{g}_madd"] = op(G_MADD, P, out[f"g{g}_aff"][::-1].copy())
        out[f"g{g}_wf"] = op(G_WF, P)
        # scalar_mul on a non-generator base
        k2 = orc.rand_field(FR, len(k), st)
        out[f"g{g}_k2"] = k2
        out[f"g{g}_k2P"] = mul(k2, P)

    # ---- MSM: the reference's CPU check (test/msm-check.cu:45-55) ----
    for g, n_list in ((1, (1, 5, 64, 300)), (2, (1, 5, 40))):
        one = ref.g1_one() if g == 1 else ref.g2_one()
        mul = ref.g1_mul if g == 1 else ref.g2_mul
        naive = ref.g1_msm_naive_jac if g == 1 else ref.g2_msm_naive_jac
        aff = ref.g1_op if g == 1 else ref.g2_op
        for n in n_list:
            k = orc.rand_field(FR, n, st)
            P = mul(k, np.repeat(one[None], n, axis=0))
            A = aff(G_AFF, P)                     # Z = 1 Jacobian; affine x,y = A[:, :2]
            s = orc.rand_field(FR, n, st)
            if n >= 5:
                s[0] = 0
                s[1] = ref.field_op(FR, TO_MONT, np.array([[1, 0, 0, 0]], np.uint64))[0]
                A[2] = A[3]                       # repeated base
            out[f"msm_g{g}_{n}_s"] = s
            out[f"msm_g{g}_{n}_aff"] = A[:, :2].copy()
            out[f"msm_g{g}_{n}_out"] = naive(s, A)

    # ---- NTT: tables, ntt_setup, number_theory_transformation ----
    out["ntt_fwd_table"] = np.stack([ref.ntt_table(0, k) for k in range(29)])
    out["ntt_inv_table"] = np.stack([ref.ntt_table(1, k) for k in range(29)])
    out["ntt_scale_table"] = np.stack([ref.ntt_table(2, k) for k in range(29)])
    for M in (2, 16, 64):
        out[f"ntt_setup_{M}"] = ref.ntt_setup(M)
    for logn in (1, 2, 3, 5, 8):
        n = 1 << logn
        tab = ref.ntt_setup(n)
        c = orc.rand_field(FR, n, st)
        out[f"ntt_{n}_in"] = c
        out[f"ntt_{n}_fwd"] = ref.ntt_ref(c, tab[:n])
        out[f"ntt_{n}_inv"] = ref.ntt_ref(c, tab[n:2 * n], tab[2 * n])

    # ---- SpMV: reference CSR (row_ptr has `rows` entries, last row ends at nnz) ----
    rng = np.random.default_rng(7)
    rows, cols = 40, 30
    nnz_per = rng.integers(0, 4, rows)
    row_ptr = np.concatenate([[0], np.cumsum(nnz_per)[:-1]]).astype(np.uint64)
    nnz = int(nnz_per.sum())
    col_idx = rng.integers(0, cols, nnz).astype(np.uint64)
    val = orc.rand_field(FR, nnz, st)
    z = orc.rand_field(FR, cols, st)
    out.update(spmv_val=val, spmv_col=col_idx, spmv_row_ptr=row_ptr, spmv_z=z,
               spmv_out=ref.spmv(val, col_idx, row_ptr, z))

    # ---- Groth16 Phase 6 proof assembly (groth16.cuh:209-215) ----
    kk = orc.rand_field(FR, 12, st)
    g1s = ref.g1_mul(kk[:7], np.repeat(ref.g1_one()[None], 7, axis=0))
    g2s = ref.g2_mul(kk[7:10], np.repeat(ref.g2_one()[None], 3, axis=0))
    r, s = kk[10], kk[11]
    og1, og2 = ref.groth16_assemble(g1s[0], g1s[1], g1s[2], g2s[0], g2s[1], g1s[3:7], g2s[2], r, s)
    out.update(asm_alpha1=g1s[0], asm_beta1=g1s[1], asm_delta1=g1s[2], asm_beta2=g2s[0], asm_delta2=g2s[1],
               asm_g1res=g1s[3:7], asm_g2res=g2s[2], asm_r=r, asm_s=s, asm_out_g1=og1, asm_out_g2=og2)

    path = os.path.join(HERE, "reference_host_arith.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
