/* oracle/lzk_oracle.h -- CPU restatement of the reference's Groth16 hot path
 * (BN254 field/curve arithmetic, MSM, NTT, SpMV, prove chain).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The
 * product library (liblightzk_b200/) never links, loads or calls it.
 *
 * Data layout at this boundary (identical to the reference's host arith and
 * to the product's C-ABI): little-endian 64-bit limbs.
 *   Fr / Fq element : uint64_t[4], Montgomery form, R = 2^256
 *                     (reference include/host-arith/field/fp.cuh:33).
 *   Fq2             : [c0 c1], i^2 = -1 (alt_bn128_init.cu:77).
 *   G1 Jacobian     : [X Y Z] (alt_bn128_g1.cuh:27); infinity has Z = 0.
 *   G2 Jacobian     : [X.c0 X.c1 Y.c0 Y.c1 Z.c0 Z.c1] (alt_bn128_g2.cuh:28).
 *   G1/G2 affine    : [x y]; the point at infinity is x = y = 0.
 * Parity is pinned by tests/test_oracle_golden.py against fixtures that the
 * reference's own host code produced (tests/golden/make_golden.py).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* seeded generator: SplitMix64 over *state */
uint64_t orc_rand_u64(uint64_t* state);
/* n uniform field elements, Montgomery limbs drawn like Fp_model::random_element
 * (fp.cuh:789-816): random limbs, bits above the modulus' MSB cleared, reject
 * >= modulus.  kind 0 = Fr, 1 = Fq. */
void orc_rand_field(int kind, uint64_t* state, uint64_t* out, size_t n);

/* field ops, kind 0 = Fr, 1 = Fq: op 0 add, 1 sub, 2 mul, 3 sqr, 4 neg,
 * 5 inverse, 6 Montgomery -> canonical, 7 canonical -> Montgomery */
void orc_field_op(int kind, int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n);
/* Fq2 ops: 0 add, 1 sub, 2 mul, 3 sqr, 4 neg, 5 inverse */
void orc_fq2_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n);

/* group ops on Jacobian points: 0 add, 1 mixed_add (b has Z = 1), 2 dbl,
 * 3 neg, 4 to_affine (Jacobian with Z = 1, or (0,1,0)), 5 eq (out = 0/1),
 * 6 is_well_formed (out = 0/1) */
void orc_g1_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n);
void orc_g2_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n);
void orc_g1_one(uint64_t* out);
void orc_g2_one(uint64_t* out);
/* out[i] = scalar[i] * P[i], Jacobian in/out (curve_utils.cuh:28-49) */
void orc_g1_mul(const uint64_t* scalars, const uint64_t* pts, uint64_t* out, size_t n);
void orc_g2_mul(const uint64_t* scalars, const uint64_t* pts, uint64_t* out, size_t n);
/* Jacobian <-> affine [x y] (infinity <-> 0,0), batch inversion */
void orc_g1_jac_to_aff(const uint64_t* jac, uint64_t* aff, size_t n);
void orc_g2_jac_to_aff(const uint64_t* jac, uint64_t* aff, size_t n);
void orc_g1_aff_to_jac(const uint64_t* aff, uint64_t* jac, size_t n);
void orc_g2_aff_to_jac(const uint64_t* aff, uint64_t* jac, size_t n);
/* affine out[i] = k[i] * generator, k Montgomery Fr (fixed-base comb) */
void orc_g1_fixed_base(const uint64_t* k, uint64_t* aff, size_t n);
void orc_g2_fixed_base(const uint64_t* k, uint64_t* aff, size_t n);

/* MSM sum_i s_i * P_i over affine bases, Jacobian result.
 *   naive   : the reference's CPU check (test/msm-check.cu:45-55)
 *   pippenger: bucket method, same group element, for large n */
void orc_g1_msm_naive(const uint64_t* s, const uint64_t* aff, size_t n, uint64_t* out);
void orc_g2_msm_naive(const uint64_t* s, const uint64_t* aff, size_t n, uint64_t* out);
void orc_g1_msm(const uint64_t* s, const uint64_t* aff, size_t n, uint64_t* out);
void orc_g2_msm(const uint64_t* s, const uint64_t* aff, size_t n, uint64_t* out);

/* NTT.  ntt_setup: the (6M+2)-entry table of groth16-operator.cuh:6-31.
 * ntt_ref: number_theory_transformation (poly.cuh:65-73) on the host.
 * ntt: natural-order transform of size 2^log_n; dir 0 forward
 * X_k = sum a_j w^(jk) with w = 2^log_n-th root of ntt-params.cuh; 1 inverse
 * (w^-1, then * n^-1); 2 coset forward (a_j * g^j first, g = 5); 3 coset
 * inverse (inverse, then * g^-j). */
int orc_ntt_setup(size_t M, uint64_t* out);
void orc_ntt_ref(uint64_t* coeffs, size_t deg, const uint64_t* omega_powers, const uint64_t* factor);
int orc_ntt(uint64_t* data, uint32_t log_n, int dir);
/* root table entry k (0..28): which 0 forward, 1 inverse, 2 2^-k (Montgomery) */
int orc_ntt_table(int which, uint32_t k, uint64_t* out);

/* SpMV, one matrix, reference CSR semantics (poly.cuh:5-30): row i covers
 * [row_ptr[i], row_ptr[i+1]) and the last row ends at nnz. */
void orc_spmv(const uint64_t* val, const uint64_t* col_idx, const uint64_t* row_ptr,
              size_t rows, size_t nnz, const uint64_t* z, uint64_t* out);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- Groth16 (include/protocol/groth16.cuh) ---------------- */
typedef struct {
    const uint64_t *val, *col, *row_ptr;  /* row_ptr: rows entries; last row ends at nnz */
    size_t rows, nnz;
} orc_csr;

typedef struct {
    orc_csr A, B, C;           /* constraints = rows <= 2^log_m */
    size_t n_vars;             /* N + 1, z[0] = 1 */
    size_t n_public;           /* k (reference) / l: L query covers z[k+1 .. N] */
    uint32_t log_m;            /* evaluation domain M = 2^log_m */
    /* affine keys (x, y); G1 8 limbs, G2 16 limbs per point */
    const uint64_t *a_query, *b1_query, *b2_query, *l_query, *h_query;
    const uint64_t *alpha1, *beta1, *delta1, *beta2, *delta2;
} orc_groth16;

/* Phase 6 of Groth16::Prove (groth16.cuh:209-215) from the five MSM
 * results (Jacobian): out_g1 = [Ar, Krs + HZ], out_g2 = [Bs2]. */
void orc_groth16_assemble(const uint64_t* alpha1, const uint64_t* beta1, const uint64_t* delta1,
                          const uint64_t* beta2, const uint64_t* delta2,
                          const uint64_t* g1res, const uint64_t* g2res,
                          const uint64_t* r, const uint64_t* s, uint64_t* out_g1, uint64_t* out_g2);

/* H-polynomial scalars (M - 1 of them).
 * mode 1 = the reference chain (groth16.cuh:159-185): iNTT_M (scale M^-1),
 *   NTT_2M of the zero-padded coefficients, A*B - C, iNTT_2M with the
 *   table's (4M)^-1 scale; scalars = coefficients M+1 .. 2M-1 (198).
 * mode 0 = standard quotient on the coset g<w_M>, g = 5: iNTT_M, coset NTT,
 *   (A*B - C) / (g^M - 1), coset iNTT; scalars = h_0 .. h_{M-2}. */
int orc_groth16_h(const orc_groth16* g, int mode, const uint64_t* z, uint64_t* h_out);

/* Full prove: SpMV, H scalars, the five MSMs, Phase 6.  Outputs Jacobian
 * proof A (G1), B (G2), C (G1). */
int orc_groth16_prove(const orc_groth16* g, int mode, const uint64_t* z, const uint64_t* r, const uint64_t* s,
                      uint64_t* proof_a, uint64_t* proof_b, uint64_t* proof_c);

#ifdef __cplusplus
}
#endif
