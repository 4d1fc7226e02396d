/* oracle/lzk_oracle.c -- CPU restatement of the reference's Groth16 hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see lzk_oracle.h).  This is the checker the CUDA
 * product is compared against; it is never part of the product.
 *
 * Field arithmetic: 4x64-bit Montgomery (R = 2^256) CIOS, the same
 * representation as the reference's Fp_model (fp.cuh:30-108, mul_reduce
 * fp.cuh:166-331).  The moduli, Montgomery constants and generators are the
 * BN254 (alt_bn128) parameters of alt_bn128_init.cu:40-70,116-132,191-195.
 */
#include "lzk_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef unsigned __int128 u128;
typedef struct { uint64_t l[4]; } fe;
typedef struct { fe c0, c1; } fe2;
typedef struct { uint64_t p[4], inv, r2[4], one[4]; } fdesc;

/* Fq: p = 0x30644e72...d87cfd47 (alt_bn128_init.cu:57), inv = -p^-1 mod 2^64 */
static const fdesc FQD = {
    {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0x87d20782e4866389ULL,
    {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL},
    {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}};
/* Fr: r = 0x30644e72...f0000001 (alt_bn128_init.cu:40) */
static const fdesc FRD = {
    {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0xc2e1f593efffffffULL,
    {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL},
    {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL}};

static inline int fe_iszero(const fe* a) { return !(a->l[0] | a->l[1] | a->l[2] | a->l[3]); }
static inline int fe_eq(const fe* a, const fe* b) { return !((a->l[0] ^ b->l[0]) | (a->l[1] ^ b->l[1]) | (a->l[2] ^ b->l[2]) | (a->l[3] ^ b->l[3])); }
static inline int geq4(const uint64_t* t, const uint64_t* p)
{
    for (int i = 3; i >= 0; i--) { if (t[i] != p[i]) return t[i] > p[i]; }
    return 1;
}
static inline void sub4(uint64_t* t, const uint64_t* p)
{
    u128 b = 0;
    for (int i = 0; i < 4; i++) { u128 d = (u128)t[i] - p[i] - b; t[i] = (uint64_t)d; b = (d >> 64) & 1; }
}
static inline void f_add(const fdesc* F, fe* o, const fe* a, const fe* b)
{
    uint64_t t[4]; u128 c = 0;
    for (int i = 0; i < 4; i++) { c += (u128)a->l[i] + b->l[i]; t[i] = (uint64_t)c; c >>= 64; }
    if (geq4(t, F->p)) sub4(t, F->p);
    memcpy(o->l, t, 32);
}
static inline void f_sub(const fdesc* F, fe* o, const fe* a, const fe* b)
{
    uint64_t t[4]; u128 br = 0;
    for (int i = 0; i < 4; i++) { u128 d = (u128)a->l[i] - b->l[i] - br; t[i] = (uint64_t)d; br = (d >> 64) & 1; }
    if (br) { u128 c = 0; for (int i = 0; i < 4; i++) { c += (u128)t[i] + F->p[i]; t[i] = (uint64_t)c; c >>= 64; } }
    memcpy(o->l, t, 32);
}
static inline void f_neg(const fdesc* F, fe* o, const fe* a)
{
    if (fe_iszero(a)) { memset(o, 0, 32); return; }
    fe p; memcpy(p.l, F->p, 32); f_sub(F, o, &p, a);
}
/* CIOS Montgomery product a*b*2^-256 mod m, fully reduced */
static inline void f_mul(const fdesc* F, fe* o, const fe* a, const fe* b)
{
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) { c += (u128)a->l[j] * b->l[i] + t[j]; t[j] = (uint64_t)c; c >>= 64; }
        c += t[4]; t[4] = (uint64_t)c; t[5] = (uint64_t)(c >> 64);
        uint64_t m = t[0] * F->inv;
        c = (u128)m * F->p[0] + t[0]; c >>= 64;
        for (int j = 1; j < 4; j++) { c += (u128)m * F->p[j] + t[j]; t[j - 1] = (uint64_t)c; c >>= 64; }
        c += t[4]; t[3] = (uint64_t)c; t[4] = t[5] + (uint64_t)(c >> 64);
    }
    if (t[4] || geq4(t, F->p)) sub4(t, F->p);
    memcpy(o->l, t, 32);
}
static inline void f_one(const fdesc* F, fe* o) { memcpy(o->l, F->one, 32); }
/* Fermat a^(m-2), MSB first over 256 bits like Fp_model::invert (fp.cuh:766-781) */
static void f_inv(const fdesc* F, fe* o, const fe* a)
{
    uint64_t e[4]; memcpy(e, F->p, 32);
    u128 d = (u128)e[0] - 2; e[0] = (uint64_t)d;  /* p is odd and > 2: no borrow */
    fe r; f_one(F, &r);
    fe x = *a;
    for (int i = 255; i >= 0; i--) {
        f_mul(F, &r, &r, &r);
        if ((e[i >> 6] >> (i & 63)) & 1) f_mul(F, &r, &r, &x);
    }
    *o = r;
}
static inline void f_from_mont(const fdesc* F, fe* o, const fe* a) { fe one = {{1, 0, 0, 0}}; f_mul(F, o, a, &one); }
static inline void f_to_mont(const fdesc* F, fe* o, const fe* a) { fe r2; memcpy(r2.l, F->r2, 32); f_mul(F, o, a, &r2); }

/* ---- Fq and Fq2 wrappers used by the curve code ---- */
static inline void fq_add(fe* o, const fe* a, const fe* b) { f_add(&FQD, o, a, b); }
static inline void fq_sub(fe* o, const fe* a, const fe* b) { f_sub(&FQD, o, a, b); }
static inline void fq_mul(fe* o, const fe* a, const fe* b) { f_mul(&FQD, o, a, b); }
static inline void fq_sqr(fe* o, const fe* a) { f_mul(&FQD, o, a, a); }
static inline void fq_neg(fe* o, const fe* a) { f_neg(&FQD, o, a); }
static inline void fq_inv(fe* o, const fe* a) { f_inv(&FQD, o, a); }
static inline void fq_one(fe* o) { f_one(&FQD, o); }
static inline void fq_zero(fe* o) { memset(o, 0, 32); }

/* Fq2 = Fq[i]/(i^2+1): Karatsuba product (fp2.cuh:171-183), complex
 * squaring (fp2.cuh:210-219), inverse via the norm (fp2.cuh:221-235). */
static inline void fq2_add(fe2* o, const fe2* a, const fe2* b) { fq_add(&o->c0, &a->c0, &b->c0); fq_add(&o->c1, &a->c1, &b->c1); }
static inline void fq2_sub(fe2* o, const fe2* a, const fe2* b) { fq_sub(&o->c0, &a->c0, &b->c0); fq_sub(&o->c1, &a->c1, &b->c1); }
static inline void fq2_neg(fe2* o, const fe2* a) { fq_neg(&o->c0, &a->c0); fq_neg(&o->c1, &a->c1); }
static inline void fq2_mul(fe2* o, const fe2* a, const fe2* b)
{
    fe aA, bB, s1, s2, c1;
    fq_mul(&aA, &a->c0, &b->c0); fq_mul(&bB, &a->c1, &b->c1);
    fq_add(&s1, &a->c0, &a->c1); fq_add(&s2, &b->c0, &b->c1);
    fq_mul(&c1, &s1, &s2); fq_sub(&c1, &c1, &aA); fq_sub(&c1, &c1, &bB);
    fq_sub(&o->c0, &aA, &bB); o->c1 = c1;
}
static inline void fq2_sqr(fe2* o, const fe2* a)
{
    fe ab, s, d, c0;
    fq_mul(&ab, &a->c0, &a->c1);
    fq_add(&s, &a->c0, &a->c1); fq_sub(&d, &a->c0, &a->c1);
    fq_mul(&c0, &s, &d);
    fq_add(&o->c1, &ab, &ab); o->c0 = c0;
}
static inline void fq2_inv(fe2* o, const fe2* a)
{
    fe t0, t1, t2, t3, c0, c1;
    fq_sqr(&t0, &a->c0); fq_sqr(&t1, &a->c1); fq_add(&t2, &t0, &t1);
    fq_inv(&t3, &t2);
    fq_mul(&c0, &a->c0, &t3); fq_mul(&c1, &a->c1, &t3); fq_neg(&c1, &c1);
    o->c0 = c0; o->c1 = c1;
}
static inline int fq2_iszero(const fe2* a) { return fe_iszero(&a->c0) && fe_iszero(&a->c1); }
static inline int fq2_eq(const fe2* a, const fe2* b) { return fe_eq(&a->c0, &b->c0) && fe_eq(&a->c1, &b->c1); }
static inline void fq2_one(fe2* o) { fq_one(&o->c0); fq_zero(&o->c1); }
static inline void fq2_zero(fe2* o) { memset(o, 0, 64); }

/* ---- G1 over Fq ---- */
typedef struct { fe X, Y, Z; } g1j;
#define ET fe
#define PT g1j
#define PFX(x) g1_##x
#define F_add fq_add
#define F_sub fq_sub
#define F_mul fq_mul
#define F_sqr fq_sqr
#define F_neg fq_neg
#define F_inv fq_inv
#define F_iszero fe_iszero
#define F_eq fe_eq
#define F_one fq_one
#define F_zero fq_zero
#include "curve_impl.h"
#undef ET
#undef PT
#undef PFX
#undef F_add
#undef F_sub
#undef F_mul
#undef F_sqr
#undef F_neg
#undef F_inv
#undef F_iszero
#undef F_eq
#undef F_one
#undef F_zero

/* ---- G2 over Fq2 ---- */
typedef struct { fe2 X, Y, Z; } g2j;
#define ET fe2
#define PT g2j
#define PFX(x) g2_##x
#define F_add fq2_add
#define F_sub fq2_sub
#define F_mul fq2_mul
#define F_sqr fq2_sqr
#define F_neg fq2_neg
#define F_inv fq2_inv
#define F_iszero fq2_iszero
#define F_eq fq2_eq
#define F_one fq2_one
#define F_zero fq2_zero
#include "curve_impl.h"

/* curve coefficients, Montgomery form: b = 3 (alt_bn128_init.cu:116) and the
 * twist b' = 3 / (9 + i) (alt_bn128_init.cu:117-118) */
static const fe G1_B = {{0x7a17caa950ad28d7ULL, 0x1f6ac17ae15521b9ULL, 0x334bea4e696bd284ULL, 0x2a1f6744ce179d8eULL}};
static const fe2 G2_B = {{{0x3bf938e377b802a8ULL, 0x020b1b273633535dULL, 0x26b7edf049755260ULL, 0x2514c6324384a86dULL}},
                         {{0x38e7ecccd1dcff67ULL, 0x65f0b37d93ce0d3eULL, 0xd749d0dd22ac00aaULL, 0x0141b9ce4a688d4dULL}}};

/* generators (alt_bn128_init.cu:130-132, 191-195), Montgomery form */
static void g1_gen(g1j* o)
{
    fe one, two; fq_one(&one); fq_add(&two, &one, &one);
    o->X = one; o->Y = two; o->Z = one;
}
static void g2_gen(g2j* o)
{
    static const fe2 X = {{{0x8e83b5d102bc2026ULL, 0xdceb1935497b0172ULL, 0xfbb8264797811adfULL, 0x19573841af96503bULL}},
                          {{0xafb4737da84c6140ULL, 0x6043dd5a5802d8c4ULL, 0x09e950fc52a02f86ULL, 0x14fef0833aea7b6bULL}}};
    static const fe2 Y = {{{0x619dfa9d886be9f6ULL, 0xfe7fd297f59e9b78ULL, 0xff9e1a62231b7dfeULL, 0x28fd7eebae9e4206ULL}},
                          {{0x64095b56c71856eeULL, 0xdc57f922327d3cbbULL, 0x55f935be33351076ULL, 0x0da4a0e693fd6482ULL}}};
    o->X = X; o->Y = Y; fq2_one(&o->Z);
}

/* ======================= exported API ======================= */

uint64_t orc_rand_u64(uint64_t* s)
{
    uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

void orc_rand_field(int kind, uint64_t* state, uint64_t* out, size_t n)
{
    const fdesc* F = kind == 0 ? &FRD : &FQD;
    for (size_t i = 0; i < n; i++) {
        uint64_t t[4];
        do {
            for (int j = 0; j < 4; j++) t[j] = orc_rand_u64(state);
            t[3] &= 0x3fffffffffffffffULL;   /* modulus MSB is bit 253 */
        } while (geq4(t, F->p));
        memcpy(out + 4 * i, t, 32);
    }
}

void orc_field_op(int kind, int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    const fdesc* F = kind == 0 ? &FRD : &FQD;
    for (size_t i = 0; i < n; i++) {
        const fe* x = (const fe*)(a + 4 * i);
        const fe* y = b ? (const fe*)(b + 4 * i) : NULL;
        fe r, z = {{0, 0, 0, 0}};
        if (!y) y = &z;
        switch (op) {
            case 0: f_add(F, &r, x, y); break;
            case 1: f_sub(F, &r, x, y); break;
            case 2: f_mul(F, &r, x, y); break;
            case 3: f_mul(F, &r, x, x); break;
            case 4: f_neg(F, &r, x); break;
            case 5: f_inv(F, &r, x); break;
            case 6: f_from_mont(F, &r, x); break;
            case 7: f_to_mont(F, &r, x); break;
            default: return;
        }
        memcpy(out + 4 * i, r.l, 32);
    }
}

void orc_fq2_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        const fe2* x = (const fe2*)(a + 8 * i);
        fe2 z; fq2_zero(&z);
        const fe2* y = b ? (const fe2*)(b + 8 * i) : &z;
        fe2 r;
        switch (op) {
            case 0: fq2_add(&r, x, y); break;
            case 1: fq2_sub(&r, x, y); break;
            case 2: fq2_mul(&r, x, y); break;
            case 3: fq2_sqr(&r, x); break;
            case 4: fq2_neg(&r, x); break;
            case 5: fq2_inv(&r, x); break;
            default: return;
        }
        memcpy(out + 8 * i, &r, 64);
    }
}

void orc_g1_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        const g1j* x = (const g1j*)(a + 12 * i);
        g1j z; g1_zero(&z);
        const g1j* y = b ? (const g1j*)(b + 12 * i) : &z;
        g1j r;
        switch (op) {
            case 0: g1_add(&r, x, y); break;
            case 1: g1_madd(&r, x, y); break;
            case 2: g1_dbl(&r, x); break;
            case 3: g1_neg(&r, x); break;
            case 4: g1_to_affine(&r, x); break;
            case 5: out[i] = (uint64_t)g1_eq(x, y); continue;
            case 6: out[i] = (uint64_t)g1_well_formed(x, &G1_B); continue;
            default: return;
        }
        memcpy(out + 12 * i, &r, 96);
    }
}

void orc_g2_op(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        const g2j* x = (const g2j*)(a + 24 * i);
        g2j z; g2_zero(&z);
        const g2j* y = b ? (const g2j*)(b + 24 * i) : &z;
        g2j r;
        switch (op) {
            case 0: g2_add(&r, x, y); break;
            case 1: g2_madd(&r, x, y); break;
            case 2: g2_dbl(&r, x); break;
            case 3: g2_neg(&r, x); break;
            case 4: g2_to_affine(&r, x); break;
            case 5: out[i] = (uint64_t)g2_eq(x, y); continue;
            case 6: out[i] = (uint64_t)g2_well_formed(x, &G2_B); continue;
            default: return;
        }
        memcpy(out + 24 * i, &r, 192);
    }
}

void orc_g1_one(uint64_t* out) { g1j g; g1_gen(&g); memcpy(out, &g, 96); }
void orc_g2_one(uint64_t* out) { g2j g; g2_gen(&g); memcpy(out, &g, 192); }

static void canon_scalars(const uint64_t* s, uint64_t* c, size_t n)
{
    #pragma omp parallel for schedule(static, 4096)
    for (size_t i = 0; i < n; i++) f_from_mont(&FRD, (fe*)(c + 4 * i), (const fe*)(s + 4 * i));
}

void orc_g1_mul(const uint64_t* s, const uint64_t* pts, uint64_t* out, size_t n)
{
    #pragma omp parallel for schedule(dynamic, 16)
    for (size_t i = 0; i < n; i++) {
        fe k; f_from_mont(&FRD, &k, (const fe*)(s + 4 * i));
        g1_mul((g1j*)(out + 12 * i), (const g1j*)(pts + 12 * i), k.l);
    }
}

void orc_g2_mul(const uint64_t* s, const uint64_t* pts, uint64_t* out, size_t n)
{
    #pragma omp parallel for schedule(dynamic, 16)
    for (size_t i = 0; i < n; i++) {
        fe k; f_from_mont(&FRD, &k, (const fe*)(s + 4 * i));
        g2_mul((g2j*)(out + 24 * i), (const g2j*)(pts + 24 * i), k.l);
    }
}

void orc_g1_jac_to_aff(const uint64_t* jac, uint64_t* aff, size_t n) { g1_batch_to_aff((const g1j*)jac, (fe*)aff, n); }
void orc_g2_jac_to_aff(const uint64_t* jac, uint64_t* aff, size_t n) { g2_batch_to_aff((const g2j*)jac, (fe2*)aff, n); }
void orc_g1_aff_to_jac(const uint64_t* aff, uint64_t* jac, size_t n)
{
    for (size_t i = 0; i < n; i++) g1_from_aff((g1j*)(jac + 12 * i), (const fe*)(aff + 8 * i));
}
void orc_g2_aff_to_jac(const uint64_t* aff, uint64_t* jac, size_t n)
{
    for (size_t i = 0; i < n; i++) g2_from_aff((g2j*)(jac + 24 * i), (const fe2*)(aff + 16 * i));
}

void orc_g1_fixed_base(const uint64_t* k, uint64_t* aff, size_t n)
{
    uint64_t* c = (uint64_t*)malloc(32 * (n ? n : 1));
    canon_scalars(k, c, n);
    g1j G; g1_gen(&G);
    g1_fixed_base(&G, c, (fe*)aff, n);
    free(c);
}

void orc_g2_fixed_base(const uint64_t* k, uint64_t* aff, size_t n)
{
    uint64_t* c = (uint64_t*)malloc(32 * (n ? n : 1));
    canon_scalars(k, c, n);
    g2j G; g2_gen(&G);
    g2_fixed_base(&G, c, (fe2*)aff, n);
    free(c);
}

/* test/msm-check.cu:45-55: per-thread accumulators of s_i * P_i */
void orc_g1_msm_naive(const uint64_t* s, const uint64_t* aff, size_t n, uint64_t* out)
{
    int T = omp_get_max_threads();
    g1j* acc = (g1j*)malloc(sizeof(g1j) * T);
    for (int t = 0; t < T; t++) g1_zero(&acc[t]);
    #pragma omp parallel
    {
        int t = omp_get_thread_num();
        #pragma omp for
        for (size_t i = 0; i < n; i++) {
            fe k; f_from_mont(&FRD, &k, (const fe*)(s + 4 * i));
            g1j P, Q; g1_from_aff(&P, (const fe*)(aff + 8 * i));
            g1_mul(&Q, &P, k.l); g1_add(&acc[t], &acc[t], &Q);
        }
    }
    for (int t = 1; t < T; t++) g1_add(&acc[0], &acc[0], &acc[t]);
    memcpy(out, &acc[0], 96);
    free(acc);
}

void orc_g2_msm_naive(const uint64_t* s, const uint64_t* aff, size_t n, uint64_t* out)
{
    int T = omp_get_max_threads();
    g2j* acc = (g2j*)malloc(sizeof(g2j) * T);
    for (int t = 0; t < T; t++) g2_zero(&acc[t]);
    #pragma omp parallel
    {
        int t = omp_get_thread_num();
        #pragma omp for
        for (size_t i = 0; i < n; i++) {
            fe k; f_from_mont(&FRD, &k, (const fe*)(s + 4 * i));
            g2j P, Q; g2_from_aff(&P, (const fe2*)(aff + 16 * i));
            g2_mul(&Q, &P, k.l); g2_add(&acc[t], &acc[t], &Q);
        }
    }
    for (int t = 1; t < T; t++) g2_add(&acc[0], &acc[0], &acc[t]);
    memcpy(out, &acc[0], 192);
    free(acc);
}

void orc_g1_msm(const uint64_t* s, const uint64_t* aff, size_t n, uint64_t* out)
{
    uint64_t* c = (uint64_t*)malloc(32 * (n ? n : 1));
    canon_scalars(s, c, n);
    g1_pippenger(c, (const fe*)aff, n, (g1j*)out);
    free(c);
}

void orc_g2_msm(const uint64_t* s, const uint64_t* aff, size_t n, uint64_t* out)
{
    uint64_t* c = (uint64_t*)malloc(32 * (n ? n : 1));
    canon_scalars(s, c, n);
    g2_pippenger(c, (const fe2*)aff, n, (g2j*)out);
    free(c);
}

/* ---------------- NTT ---------------- */

static const fe ROOT28 = {{0x636e735580d13d9cULL, 0xa22bf3742445ffd6ULL, 0x56452ac01eb203d8ULL, 0x1860ef942963f9e7ULL}};

/* ntt-params.cuh tables, derived: entry k of the forward table is
 * w_k = w_28^(2^(28-k)) with w_28 = 5^((r-1)/2^28) (= Fr::root_of_unity,
 * alt_bn128_init.cu:51); the inverse table holds w_k^-1 and the scale table
 * 2^-k, all in Montgomery form. */
int orc_ntt_table(int which, uint32_t k, uint64_t* out)
{
    if (k > 28 || which < 0 || which > 2) return -1;
    fe r;
    if (which == 2) {
        fe two; fq_zero(&two); two.l[0] = 2; f_to_mont(&FRD, &two, &two);
        fe t; f_one(&FRD, &t);
        for (uint32_t i = 0; i < k; i++) f_mul(&FRD, &t, &t, &two);
        f_inv(&FRD, &r, &t);
    } else {
        r = ROOT28;
        for (uint32_t i = k; i < 28; i++) f_mul(&FRD, &r, &r, &r);
        if (which == 1) f_inv(&FRD, &r, &r);
    }
    memcpy(out, r.l, 32);
    return 0;
}

/* groth16-operator.cuh:6-31 */
int orc_ntt_setup(size_t M, uint64_t* out)
{
    if (M < 2 || (M & (M - 1))) return -1;
    uint32_t io = (uint32_t)__builtin_ctzl(M), eo = io + 1;
    fe* p = (fe*)out;
    f_one(&FRD, &p[0]); p[M] = p[2 * M + 1] = p[4 * M + 1] = p[0];
    orc_ntt_table(2, io, p[2 * M].l);
    orc_ntt_table(2, eo + 1, p[6 * M + 1].l);
    fe w, wi, e, ei;
    orc_ntt_table(0, io, w.l); orc_ntt_table(1, io, wi.l);
    orc_ntt_table(0, eo, e.l); orc_ntt_table(1, eo, ei.l);
    for (size_t i = 1; i < M; i++) { f_mul(&FRD, &p[i], &p[i - 1], &w); f_mul(&FRD, &p[M + i], &p[M + i - 1], &wi); }
    for (size_t i = 1; i < 2 * M; i++) { f_mul(&FRD, &p[2 * M + 1 + i], &p[2 * M + i], &e); f_mul(&FRD, &p[4 * M + 1 + i], &p[4 * M + i], &ei); }
    return 0;
}

/* poly.cuh:32-73: log2(deg) DIF stages, bit reversal, optional scale */
void orc_ntt_ref(uint64_t* coeffs, size_t deg, const uint64_t* omega_powers, const uint64_t* factor)
{
    fe* c = (fe*)coeffs;
    const fe* w = (const fe*)omega_powers;
    size_t log_deg = (size_t)__builtin_ctzl(deg);
    for (size_t hl = deg >> 1, i = 0; hl > 0; hl >>= 1, i++) {
        #pragma omp parallel for schedule(static, 4096) if (deg >= (1u << 14))
        for (size_t j = 0; j < deg; j++) if ((j & hl) == 0) {
            fe lo = c[j], hi = c[j ^ hl], d;
            size_t e = (j & (hl - 1)) << i;
            f_add(&FRD, &c[j], &lo, &hi);
            f_sub(&FRD, &d, &lo, &hi);
            f_mul(&FRD, &c[j ^ hl], &d, &w[e]);
        }
    }
    for (size_t j = 0; j < deg; j++) {
        size_t r = 0;
        for (size_t b = 0; b < log_deg; b++) if (j >> b & 1) r |= (size_t)1 << (log_deg - 1 - b);
        if (j < r) { fe t = c[j]; c[j] = c[r]; c[r] = t; }
    }
    if (factor) {
        fe f = *(const fe*)factor;
        for (size_t j = 0; j < deg; j++) f_mul(&FRD, &c[j], &c[j], &f);
    }
}

int orc_ntt(uint64_t* data, uint32_t log_n, int dir)
{
    if (log_n > 28 || dir < 0 || dir > 3) return -1;
    size_t n = (size_t)1 << log_n;
    if (log_n == 0) return 0;
    fe* d = (fe*)data;
    fe g; fq_zero(&g); g.l[0] = 5; f_to_mont(&FRD, &g, &g);
    if (dir == 2) {  /* a_j *= g^j */
        fe gp; f_one(&FRD, &gp);
        for (size_t j = 0; j < n; j++) { f_mul(&FRD, &d[j], &d[j], &gp); f_mul(&FRD, &gp, &gp, &g); }
    }
    fe w; orc_ntt_table((dir & 1) ? 1 : 0, log_n, w.l);
    fe* pw = (fe*)malloc(sizeof(fe) * (n / 2 + 1));
    f_one(&FRD, &pw[0]);
    for (size_t i = 1; i <= n / 2; i++) f_mul(&FRD, &pw[i], &pw[i - 1], &w);
    fe sc; orc_ntt_table(2, log_n, sc.l);
    orc_ntt_ref(data, n, (const uint64_t*)pw, (dir & 1) ? sc.l : NULL);
    free(pw);
    if (dir == 3) {  /* a_j *= g^-j */
        fe gi, gp; f_inv(&FRD, &gi, &g); f_one(&FRD, &gp);
        for (size_t j = 0; j < n; j++) { f_mul(&FRD, &d[j], &d[j], &gp); f_mul(&FRD, &gp, &gp, &gi); }
    }
    return 0;
}

/* ---------------- SpMV ---------------- */

void orc_spmv(const uint64_t* val, const uint64_t* col_idx, const uint64_t* row_ptr,
              size_t rows, size_t nnz, const uint64_t* z, uint64_t* out)
{
    #pragma omp parallel for schedule(static, 1024)
    for (size_t i = 0; i < rows; i++) {
        size_t e = (i + 1 < rows) ? row_ptr[i + 1] : nnz;
        fe acc = {{0, 0, 0, 0}}, t;
        for (size_t j = row_ptr[i]; j < e; j++) {
            f_mul(&FRD, &t, (const fe*)(z + 4 * col_idx[j]), (const fe*)(val + 4 * j));
            f_add(&FRD, &acc, &acc, &t);
        }
        memcpy(out + 4 * i, acc.l, 32);
    }
}

/* ---------------- Groth16 ---------------- */

static void jac_from_aff_g1(g1j* o, const uint64_t* aff) { g1_from_aff(o, (const fe*)aff); }
static void jac_from_aff_g2(g2j* o, const uint64_t* aff) { g2_from_aff(o, (const fe2*)aff); }

static void fr_canon(const uint64_t* m, uint64_t* c) { f_from_mont(&FRD, (fe*)c, (const fe*)m); }

/* groth16.cuh:211-215 */
void orc_groth16_assemble(const uint64_t* alpha1, const uint64_t* beta1, const uint64_t* delta1,
                          const uint64_t* beta2, const uint64_t* delta2,
                          const uint64_t* g1res, const uint64_t* g2res,
                          const uint64_t* r, const uint64_t* s, uint64_t* out_g1, uint64_t* out_g2)
{
    const g1j *a1 = (const g1j*)alpha1, *b1 = (const g1j*)beta1, *d1 = (const g1j*)delta1;
    const g2j *b2 = (const g2j*)beta2, *d2 = (const g2j*)delta2;
    const g1j* res = (const g1j*)g1res;
    uint64_t rc[4], sc[4], nrsc[4];
    fe nr, nrs;
    fr_canon(r, rc); fr_canon(s, sc);
    f_neg(&FRD, &nr, (const fe*)r); f_mul(&FRD, &nrs, &nr, (const fe*)s);
    fr_canon(nrs.l, nrsc);
    g1j t, Ar, Bs1, Krs;
    g1_add(&Ar, a1, &res[0]); g1_mul(&t, d1, rc); g1_add(&Ar, &Ar, &t);
    g1_add(&Bs1, b1, &res[1]); g1_mul(&t, d1, sc); g1_add(&Bs1, &Bs1, &t);
    g1_mul(&Krs, &Ar, sc);
    g1_mul(&t, &Bs1, rc); g1_add(&Krs, &Krs, &t);
    g1_mul(&t, d1, nrsc); g1_add(&Krs, &Krs, &t);
    g1_add(&Krs, &Krs, &res[2]);
    g1_add(&t, &Krs, &res[3]);
    memcpy(out_g1, &Ar, 96); memcpy(out_g1 + 12, &t, 96);
    g2j u, Bs2;
    g2_add(&Bs2, b2, (const g2j*)g2res); g2_mul(&u, d2, sc); g2_add(&Bs2, &Bs2, &u);
    memcpy(out_g2, &Bs2, 192);
}

static void csr_spmv(const orc_csr* m, const uint64_t* z, uint64_t* out)
{
    orc_spmv(m->val, m->col, m->row_ptr, m->rows, m->nnz, z, out);
}

int orc_groth16_h(const orc_groth16* g, int mode, const uint64_t* z, uint64_t* h_out)
{
    size_t M = (size_t)1 << g->log_m;
    if (g->A.rows > M || g->B.rows > M || g->C.rows > M || g->log_m < 1 || g->log_m > 26) return -1;
    size_t L = mode == 1 ? 2 * M : M;
    fe* x[3];
    for (int q = 0; q < 3; q++) { x[q] = (fe*)calloc(L, sizeof(fe)); }
    csr_spmv(&g->A, z, (uint64_t*)x[0]);
    csr_spmv(&g->B, z, (uint64_t*)x[1]);
    csr_spmv(&g->C, z, (uint64_t*)x[2]);
    if (mode == 1) {
        for (int q = 0; q < 3; q++) orc_ntt((uint64_t*)x[q], g->log_m, 1);          /* iNTT_M, * M^-1 */
        for (int q = 0; q < 3; q++) orc_ntt((uint64_t*)x[q], g->log_m + 1, 0);      /* NTT_2M */
        for (size_t j = 0; j < L; j++) { fe t; f_mul(&FRD, &t, &x[0][j], &x[1][j]); f_sub(&FRD, &x[0][j], &t, &x[2][j]); }
        /* iNTT_2M with the (4M)^-1 entry of ntt_setup (groth16-operator.cuh:13) */
        fe w; orc_ntt_table(1, g->log_m + 1, w.l);
        fe* pw = (fe*)malloc(sizeof(fe) * M);
        f_one(&FRD, &pw[0]);
        for (size_t i = 1; i < M; i++) f_mul(&FRD, &pw[i], &pw[i - 1], &w);
        fe sc; orc_ntt_table(2, g->log_m + 2, sc.l);
        orc_ntt_ref((uint64_t*)x[0], L, (const uint64_t*)pw, sc.l);
        free(pw);
        memcpy(h_out, &x[0][M + 1], sizeof(fe) * (M - 1));
    } else {
        for (int q = 0; q < 3; q++) { orc_ntt((uint64_t*)x[q], g->log_m, 1); orc_ntt((uint64_t*)x[q], g->log_m, 2); }
        /* Z(g w^j) = g^M - 1 for every j */
        fe gm, one, zinv; fq_zero(&gm); gm.l[0] = 5; f_to_mont(&FRD, &gm, &gm);
        for (uint32_t i = 0; i < g->log_m; i++) f_mul(&FRD, &gm, &gm, &gm);
        f_one(&FRD, &one); f_sub(&FRD, &gm, &gm, &one); f_inv(&FRD, &zinv, &gm);
        for (size_t j = 0; j < M; j++) {
            fe t; f_mul(&FRD, &t, &x[0][j], &x[1][j]); f_sub(&FRD, &t, &t, &x[2][j]); f_mul(&FRD, &x[0][j], &t, &zinv);
        }
        orc_ntt((uint64_t*)x[0], g->log_m, 3);
        memcpy(h_out, &x[0][0], sizeof(fe) * (M - 1));
    }
    for (int q = 0; q < 3; q++) free(x[q]);
    return 0;
}

int orc_groth16_prove(const orc_groth16* g, int mode, const uint64_t* z, const uint64_t* r, const uint64_t* s,
                      uint64_t* proof_a, uint64_t* proof_b, uint64_t* proof_c)
{
    size_t M = (size_t)1 << g->log_m;
    uint64_t* h = (uint64_t*)malloc(32 * M);
    if (orc_groth16_h(g, mode, z, h)) { free(h); return -1; }
    uint64_t g1res[4 * 12], g2res[24];
    size_t nl = g->n_vars - g->n_public - 1;
    orc_g1_msm(z, g->a_query, g->n_vars, g1res);
    orc_g1_msm(z, g->b1_query, g->n_vars, g1res + 12);
    orc_g1_msm(z + 4 * (g->n_public + 1), g->l_query, nl, g1res + 24);
    orc_g1_msm(h, g->h_query, M - 1, g1res + 36);
    orc_g2_msm(z, g->b2_query, g->n_vars, g2res);
    free(h);
    g1j a1, b1, d1; g2j b2, d2;
    jac_from_aff_g1(&a1, g->alpha1); jac_from_aff_g1(&b1, g->beta1); jac_from_aff_g1(&d1, g->delta1);
    jac_from_aff_g2(&b2, g->beta2); jac_from_aff_g2(&d2, g->delta2);
    uint64_t og1[24], og2[24];
    orc_groth16_assemble((uint64_t*)&a1, (uint64_t*)&b1, (uint64_t*)&d1, (uint64_t*)&b2, (uint64_t*)&d2,
                         g1res, g2res, r, s, og1, og2);
    memcpy(proof_a, og1, 96); memcpy(proof_c, og1 + 12, 96); memcpy(proof_b, og2, 192);
    return 0;
}
