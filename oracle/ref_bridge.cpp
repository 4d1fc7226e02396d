/* oracle/ref_bridge.cpp -- extern "C" entry points over the reference's OWN
 * host arithmetic (libff-derived, include/host-arith/** and
 * src/host-arith/**), compiled from the reference tree by oracle/Makefile
 * into oracle/_ref/libref.so.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (liblightzk_b200/) links,
 * loads or calls this.  It is used (a) to generate the golden fixtures under
 * tests/golden/ and (b) to pin the C restatement in oracle/lzk_oracle.c, and
 * (c) as the timed CPU baseline (`bench.py --impl reference`).
 *
 * Every value crosses this boundary as raw little-endian 64-bit limbs in the
 * reference's in-memory layout: Fr/Fq = bigint<4> Montgomery form (R=2^256,
 * fp.cuh:33); Fq2 = [c0 c1]; G1 = Jacobian [X Y Z] (alt_bn128_g1.cuh:27);
 * G2 = [X.c0 X.c1 Y.c0 Y.c1 Z.c0 Z.c1] (alt_bn128_g2.cuh:28).
 *
 * Where the reference has no CPU form of an operator (NTT, SpMV, the prove
 * chain), the functions below restate the reference's device algorithm with
 * the reference's own host field type, citing the lines they follow.
 */
#include "alt_bn128_g1.cuh"
#include "alt_bn128_g2.cuh"
#include "alt_bn128_init.cuh"
#include "ntt-params.cuh"
#include <omp.h>

using namespace libff;
typedef alt_bn128_Fr Fr;
typedef alt_bn128_Fq Fq;
typedef alt_bn128_Fq2 Fq2;
typedef alt_bn128_G1 G1;
typedef alt_bn128_G2 G2;

template <typename F> static F ldf(const uint64_t* p) { F x; memcpy(x.mont_repr.data, p, 32); return x; }
template <typename F> static void stf(uint64_t* p, const F& x) { memcpy(p, x.mont_repr.data, 32); }
static Fq2 ld2(const uint64_t* p) { return Fq2(ldf<Fq>(p), ldf<Fq>(p + 4)); }
static void st2(uint64_t* p, const Fq2& x) { stf(p, x.c0); stf(p + 4, x.c1); }
static G1 ldg1(const uint64_t* p) { return G1(ldf<Fq>(p), ldf<Fq>(p + 4), ldf<Fq>(p + 8)); }
static void stg1(uint64_t* p, const G1& g) { stf(p, g.X); stf(p + 4, g.Y); stf(p + 8, g.Z); }
static G2 ldg2(const uint64_t* p) { return G2(ld2(p), ld2(p + 8), ld2(p + 16)); }
static void stg2(uint64_t* p, const G2& g) { st2(p, g.X); st2(p + 8, g.Y); st2(p + 16, g.Z); }

template <typename F>
static void field_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        F x = ldf<F>(a + 4 * i), y = b ? ldf<F>(b + 4 * i) : F::zero(), r;
        switch (op) {
            case 0: r = x + y; break;
            case 1: r = x - y; break;
            case 2: r = x * y; break;
            case 3: r = x.squared(); break;
            case 4: r = -x; break;
            case 5: r = x.inverse(); break;
            case 6: { bigint<4> c = x.as_bigint(); memcpy(out + 4 * i, c.data, 32); continue; }
            case 7: { bigint<4> c; memcpy(c.data, a + 4 * i, 32); r = F(c, true); break; }
            default: return;
        }
        stf(out + 4 * i, r);
    }
}

extern "C" {

void ref_init(void)
{
    static bool done = false;
    if (!done) { init_alt_bn128_params(); done = true; }
}

/* kind 0 = Fr, 1 = Fq.  op: 0 add, 1 sub, 2 mul, 3 squared, 4 neg, 5 inverse,
 * 6 as_bigint (Montgomery -> canonical), 7 canonical -> Montgomery
 * (Fp_model(bigint, raw=true), fp.cuh:333-341). */
void ref_field_op(int kind, int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    if (kind == 0) field_op<Fr>(op, a, b, out, n); else field_op<Fq>(op, a, b, out, n);
}

/* Fq2 = Fq[i]/(i^2 - non_residue), non_residue = -1 (alt_bn128_init.cu:77).
 * op: 0 add, 1 sub, 2 mul (Karatsuba, fp2.cuh:171-183), 3 squared
 * (complex squaring, fp2.cuh:210-219), 4 neg, 5 inverse (fp2.cuh:221-235). */
void ref_fq2_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        Fq2 x = ld2(a + 8 * i), y = b ? ld2(b + 8 * i) : Fq2::zero(), r;
        switch (op) {
            case 0: r = x + y; break;
            case 1: r = x - y; break;
            case 2: r = x * y; break;
            case 3: r = x.squared(); break;
            case 4: r = -x; break;
            case 5: r = x.inverse(); break;
            default: return;
        }
        st2(out + 8 * i, r);
    }
}

/* Group ops, alt_bn128_g1.cu / alt_bn128_g2.cu.  op: 0 operator+ (135-191),
 * 1 mixed_add (248-312; b must have Z = 1), 2 dbl (314-347), 3 negate,
 * 4 to_affine_coordinates (56-73), 5 operator== (90-128; out[i] = 0/1),
 * 6 is_well_formed (out[i] = 0/1). */
void ref_g1_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        G1 x = ldg1(a + 12 * i), y = b ? ldg1(b + 12 * i) : G1::zero(), r;
        switch (op) {
            case 0: r = x + y; break;
            case 1: r = x.mixed_add(y); break;
            case 2: r = x.dbl(); break;
            case 3: r = -x; break;
            case 4: r = x; r.to_affine_coordinates(); break;
            case 5: out[i] = (x == y) ? 1 : 0; continue;
            case 6: out[i] = x.is_well_formed() ? 1 : 0; continue;
            default: return;
        }
        stg1(out + 12 * i, r);
    }
}

void ref_g2_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        G2 x = ldg2(a + 24 * i), y = b ? ldg2(b + 24 * i) : G2::zero(), r;
        switch (op) {
            case 0: r = x + y; break;
            case 1: r = x.mixed_add(y); break;
            case 2: r = x.dbl(); break;
            case 3: r = -x; break;
            case 4: r = x; r.to_affine_coordinates(); break;
            case 5: out[i] = (x == y) ? 1 : 0; continue;
            case 6: out[i] = x.is_well_formed() ? 1 : 0; continue;
            default: return;
        }
        stg2(out + 24 * i, r);
    }
}

void ref_g1_one(uint64_t* out) { stg1(out, G1::one()); }
void ref_g2_one(uint64_t* out) { stg2(out, G2::one()); }

/* out[i] = scalars[i] * pts[i]: operator*(Fp_model, G) = scalar_mul over
 * as_bigint() (alt_bn128_g1.cuh:70-74, curve_utils.cuh:28-49). */
void ref_g1_mul(const uint64_t* scalars, const uint64_t* pts, uint64_t* out, size_t n)
{
    #pragma omp parallel for schedule(dynamic, 16)
    for (size_t i = 0; i < n; i++) stg1(out + 12 * i, ldf<Fr>(scalars + 4 * i) * ldg1(pts + 12 * i));
}

void ref_g2_mul(const uint64_t* scalars, const uint64_t* pts, uint64_t* out, size_t n)
{
    #pragma omp parallel for schedule(dynamic, 16)
    for (size_t i = 0; i < n; i++) stg2(out + 24 * i, ldf<Fr>(scalars + 4 * i) * ldg2(pts + 24 * i));
}

/* The reference's CPU MSM check, test/msm-check.cu:45-55: per-thread
 * accumulators of scalars[i] * points[i], then a serial sum. */
void ref_g1_msm_naive(const uint64_t* scalars, const uint64_t* pts, size_t n, uint64_t* out)
{
    const int num_threads = omp_get_max_threads();
    std::vector<G1> local_acc(num_threads, G1::zero());
    #pragma omp parallel
    {
        const int tid = omp_get_thread_num();
        #pragma omp for
        for (size_t i = 0; i < n; i++) local_acc[tid] = local_acc[tid] + ldf<Fr>(scalars + 4 * i) * ldg1(pts + 12 * i);
    }
    for (int i = 1; i < num_threads; i++) local_acc[0] = local_acc[0] + local_acc[i];
    stg1(out, local_acc[0]);
}

void ref_g2_msm_naive(const uint64_t* scalars, const uint64_t* pts, size_t n, uint64_t* out)
{
    const int num_threads = omp_get_max_threads();
    std::vector<G2> local_acc(num_threads, G2::zero());
    #pragma omp parallel
    {
        const int tid = omp_get_thread_num();
        #pragma omp for
        for (size_t i = 0; i < n; i++) local_acc[tid] = local_acc[tid] + ldf<Fr>(scalars + 4 * i) * ldg2(pts + 24 * i);
    }
    for (int i = 1; i < num_threads; i++) local_acc[0] = local_acc[0] + local_acc[i];
    stg2(out, local_acc[0]);
}

/* The three root/scale tables of ntt-params.cuh, entry k, Montgomery limbs
 * read with raw=false exactly as ntt_setup does (groth16-operator.cuh:12-17).
 * which: 0 forward root, 1 inverse root, 2 domain scale inverse. */
int ref_ntt_table(int which, size_t k, uint64_t* out)
{
    if (k > alt_bn128_ntt_config.ntt_S) return -1;
    const char* base = which == 0 ? alt_bn128_ntt_config.forward_root_of_unity
                     : which == 1 ? alt_bn128_ntt_config.inverse_root_of_unity
                                  : alt_bn128_ntt_config.domain_scale_inverse;
    Fr x(bigint<4>(base + k * alt_bn128_ntt_config.str_len), false);
    stf(out, x);
    return 0;
}

/* ntt_setup (groth16-operator.cuh:6-31) without the device store: the
 * (6M+2)-entry table [w_M^i | w_M^-i | M^-1 | w_2M^i | w_2M^-i | scale],
 * where scale is table entry (log2 M + 2) of the domain-scale table. */
int ref_ntt_setup(size_t M, uint64_t* out)
{
    if (M < 2 || (M & (M - 1))) return -1;
    std::vector<Fr> p(6 * M + 2);
    size_t int_order = __builtin_ctzl(M), eval_order = int_order + 1;
    const size_t L = alt_bn128_ntt_config.str_len;
    p[0] = p[M] = p[2 * M + 1] = p[4 * M + 1] = Fr::one();
    p[2 * M] = Fr(bigint<4>(alt_bn128_ntt_config.domain_scale_inverse + int_order * L), false);
    p[6 * M + 1] = Fr(bigint<4>(alt_bn128_ntt_config.domain_scale_inverse + (eval_order + 1) * L), false);
    Fr w(bigint<4>(alt_bn128_ntt_config.forward_root_of_unity + int_order * L), false);
    Fr wi(bigint<4>(alt_bn128_ntt_config.inverse_root_of_unity + int_order * L), false);
    Fr e(bigint<4>(alt_bn128_ntt_config.forward_root_of_unity + eval_order * L), false);
    Fr ei(bigint<4>(alt_bn128_ntt_config.inverse_root_of_unity + eval_order * L), false);
    for (size_t i = 1; i < M; i++) { p[i] = p[i - 1] * w; p[M + i] = p[M + i - 1] * wi; }
    for (size_t i = 1; i < 2 * M; i++) { p[2 * M + 1 + i] = p[2 * M + i] * e; p[4 * M + 1 + i] = p[4 * M + i] * ei; }
    for (size_t i = 0; i < 6 * M + 2; i++) stf(out + 4 * i, p[i]);
    return 0;
}

/* number_theory_transformation (poly.cuh:65-73) on the host: log2(deg)
 * radix-2 DIF stages of ntt_loop (poly.cuh:32-41) with twiddle
 * omega_powers[(j & (hl-1)) << i], then ntt_bitrev_permutation (42-54), then
 * ntt_mul_by_factor (55-63) when factor != NULL. */
void ref_ntt(uint64_t* coeffs, size_t deg, const uint64_t* omega_powers, const uint64_t* factor)
{
    std::vector<Fr> c(deg);
    for (size_t j = 0; j < deg; j++) c[j] = ldf<Fr>(coeffs + 4 * j);
    size_t log_deg = __builtin_ctzl(deg);
    for (size_t hl = deg >> 1, i = 0; hl > 0; hl >>= 1, i++) {
        for (size_t j = 0; j < deg; j++) if ((j & hl) == 0) {
            Fr lo = c[j], hi = c[j ^ hl];
            size_t e = (j & (hl - 1)) << i;
            c[j] = lo + hi; c[j ^ hl] = (lo - hi) * ldf<Fr>(omega_powers + 4 * e);
        }
    }
    for (size_t j = 0; j < deg; j++) {
        size_t r = 0;
        for (size_t b = 0; b < log_deg; b++) if (j >> b & 1) r |= (size_t)1 << (log_deg - 1 - b);
        if (j < r) std::swap(c[j], c[r]);
    }
    if (factor) { Fr f = ldf<Fr>(factor); for (size_t j = 0; j < deg; j++) c[j] *= f; }
    for (size_t j = 0; j < deg; j++) stf(coeffs + 4 * j, c[j]);
}

/* batch_sparse_matrix_vector_multiplication (poly.cuh:5-30) for one matrix,
 * with the reference's CSR descriptor (xpu-spmat.cuh:20-25): row_ptr has
 * `rows` entries, the last row ends at cnt; acc += z[col] * val. */
void ref_spmv(const uint64_t* val, const uint64_t* col_idx, const uint64_t* row_ptr,
              size_t rows, size_t cnt, const uint64_t* z, uint64_t* out)
{
    for (size_t i = 0; i < rows; i++) {
        size_t e = (i + 1 < rows) ? row_ptr[i + 1] : cnt;
        Fr acc = Fr::zero();
        for (size_t j = row_ptr[i]; j < e; j++) acc += ldf<Fr>(z + 4 * col_idx[j]) * ldf<Fr>(val + 4 * j);
        stf(out + 4 * i, acc);
    }
}

/* polynomial_A_times_B_minus_C (poly.cuh:75-85): A[i] = A[i]*B[i] - C[i]. */
void ref_abc(uint64_t* A, const uint64_t* B, const uint64_t* C, size_t n)
{
    for (size_t i = 0; i < n; i++) stf(A + 4 * i, ldf<Fr>(A + 4 * i) * ldf<Fr>(B + 4 * i) - ldf<Fr>(C + 4 * i));
}

/* Groth16::Prove Phase 6 (groth16.cuh:209-215): proof assembly from the five
 * MSM results.  g1res = 4 G1, g2res = 1 G2; out_g1 = [Ar, Krs+HZ],
 * out_g2 = [Bs2]. */
void ref_groth16_assemble(const uint64_t* alpha1, const uint64_t* beta1, const uint64_t* delta1,
                          const uint64_t* beta2, const uint64_t* delta2,
                          const uint64_t* g1res, const uint64_t* g2res,
                          const uint64_t* r_mont, const uint64_t* s_mont,
                          uint64_t* out_g1, uint64_t* out_g2)
{
    Fr r = ldf<Fr>(r_mont), s = ldf<Fr>(s_mont);
    G1 a1 = ldg1(alpha1), b1 = ldg1(beta1), d1 = ldg1(delta1);
    G2 b2 = ldg2(beta2), d2 = ldg2(delta2);
    G1 g0 = ldg1(g1res), gb = ldg1(g1res + 12), gk = ldg1(g1res + 24), gh = ldg1(g1res + 36);
    G2 h0 = ldg2(g2res);
    G1 Ar = a1 + g0 + r * d1, Bs1 = b1 + gb + s * d1;
    G1 Krs = s * Ar + r * Bs1 + ((-r) * s) * d1 + gk, HZ = gh;
    G2 Bs2 = b2 + h0 + s * d2;
    stg1(out_g1, Ar); stg1(out_g1 + 12, Krs + HZ); stg2(out_g2, Bs2);
}

} /* extern "C" */
