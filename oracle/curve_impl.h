/* oracle/curve_impl.h -- Jacobian short-Weierstrass arithmetic, included once
 * per group by lzk_oracle.c (G1 over Fq, G2 over Fq2).  Test infrastructure.
 *
 * Formulas follow the reference's host arithmetic step by step so that even
 * Jacobian coordinates agree bit for bit with it:
 *   dbl       dbl-2009-l          alt_bn128_g1.cu:314-347
 *   add       add-2007-bl + dbl   alt_bn128_g1.cu:135-191
 *   madd      madd-2007-bl + dbl  alt_bn128_g1.cu:248-312
 *   eq        cross-multiplied    alt_bn128_g1.cu:90-128
 *   to_affine Z^-1, Z^-2, Z^-3    alt_bn128_g1.cu:56-73
 *   mul       MSB-first double-and-add over 256 bits, curve_utils.cuh:28-49
 * The G2 versions in alt_bn128_g2.cu are the same code over Fq2.
 *
 * Required macros: ET (field element type), PT (point type), PFX(x) (name
 * prefix), F_add F_sub F_mul F_sqr F_neg F_inv F_iszero F_eq F_one F_zero.
 */

static void PFX(zero)(PT* o) { F_zero(&o->X); F_one(&o->Y); F_zero(&o->Z); }
static int PFX(is_zero)(const PT* a) { return F_iszero(&a->Z); }

static void PFX(dbl)(PT* o, const PT* a)
{
    if (PFX(is_zero)(a)) { *o = *a; return; }
    ET A, B, C, D, E, Fv, X3, Y3, Z3, t, eightC, Y1Z1;
    F_sqr(&A, &a->X);
    F_sqr(&B, &a->Y);
    F_sqr(&C, &B);
    F_add(&t, &a->X, &B); F_sqr(&D, &t); F_sub(&D, &D, &A); F_sub(&D, &D, &C);
    F_add(&D, &D, &D);
    F_add(&E, &A, &A); F_add(&E, &E, &A);
    F_sqr(&Fv, &E);
    F_add(&t, &D, &D); F_sub(&X3, &Fv, &t);
    F_add(&eightC, &C, &C); F_add(&eightC, &eightC, &eightC); F_add(&eightC, &eightC, &eightC);
    F_sub(&t, &D, &X3); F_mul(&Y3, &E, &t); F_sub(&Y3, &Y3, &eightC);
    F_mul(&Y1Z1, &a->Y, &a->Z); F_add(&Z3, &Y1Z1, &Y1Z1);
    o->X = X3; o->Y = Y3; o->Z = Z3;
}

static void PFX(add)(PT* o, const PT* a, const PT* b)
{
    if (PFX(is_zero)(a)) { *o = *b; return; }
    if (PFX(is_zero)(b)) { *o = *a; return; }
    ET Z1Z1, Z2Z2, U1, U2, Z1c, Z2c, S1, S2, H, S2mS1, I, J, r, V, X3, Y3, Z3, t, S1J;
    F_sqr(&Z1Z1, &a->Z);
    F_sqr(&Z2Z2, &b->Z);
    F_mul(&U1, &a->X, &Z2Z2);
    F_mul(&U2, &b->X, &Z1Z1);
    F_mul(&Z1c, &a->Z, &Z1Z1);
    F_mul(&Z2c, &b->Z, &Z2Z2);
    F_mul(&S1, &a->Y, &Z2c);
    F_mul(&S2, &b->Y, &Z1c);
    if (F_eq(&U1, &U2) && F_eq(&S1, &S2)) { PFX(dbl)(o, a); return; }
    F_sub(&H, &U2, &U1);
    F_sub(&S2mS1, &S2, &S1);
    F_add(&t, &H, &H); F_sqr(&I, &t);
    F_mul(&J, &H, &I);
    F_add(&r, &S2mS1, &S2mS1);
    F_mul(&V, &U1, &I);
    F_sqr(&X3, &r); F_sub(&X3, &X3, &J); F_add(&t, &V, &V); F_sub(&X3, &X3, &t);
    F_mul(&S1J, &S1, &J);
    F_sub(&t, &V, &X3); F_mul(&Y3, &r, &t); F_add(&t, &S1J, &S1J); F_sub(&Y3, &Y3, &t);
    F_add(&t, &a->Z, &b->Z); F_sqr(&Z3, &t); F_sub(&Z3, &Z3, &Z1Z1); F_sub(&Z3, &Z3, &Z2Z2); F_mul(&Z3, &Z3, &H);
    o->X = X3; o->Y = Y3; o->Z = Z3;
}

static void PFX(madd)(PT* o, const PT* a, const PT* b)
{
    if (PFX(is_zero)(a)) { *o = *b; return; }
    if (PFX(is_zero)(b)) { *o = *a; return; }
    ET Z1Z1, U2, Z1c, S2, H, HH, I, J, r, V, X3, Y3, Z3, t;
    F_sqr(&Z1Z1, &a->Z);
    F_mul(&U2, &b->X, &Z1Z1);
    F_mul(&Z1c, &a->Z, &Z1Z1);
    F_mul(&S2, &b->Y, &Z1c);
    if (F_eq(&a->X, &U2) && F_eq(&a->Y, &S2)) { PFX(dbl)(o, a); return; }
    F_sub(&H, &U2, &a->X);
    F_sqr(&HH, &H);
    F_add(&I, &HH, &HH); F_add(&I, &I, &I);
    F_mul(&J, &H, &I);
    F_sub(&r, &S2, &a->Y); F_add(&r, &r, &r);
    F_mul(&V, &a->X, &I);
    F_sqr(&X3, &r); F_sub(&X3, &X3, &J); F_sub(&X3, &X3, &V); F_sub(&X3, &X3, &V);
    F_mul(&Y3, &a->Y, &J);
    F_sub(&t, &V, &X3); F_mul(&t, &r, &t); F_sub(&t, &t, &Y3); F_sub(&Y3, &t, &Y3);
    F_add(&t, &a->Z, &H); F_sqr(&Z3, &t); F_sub(&Z3, &Z3, &Z1Z1); F_sub(&Z3, &Z3, &HH);
    o->X = X3; o->Y = Y3; o->Z = Z3;
}

static void PFX(neg)(PT* o, const PT* a) { o->X = a->X; F_neg(&o->Y, &a->Y); o->Z = a->Z; }

static int PFX(eq)(const PT* a, const PT* b)
{
    if (PFX(is_zero)(a)) return PFX(is_zero)(b);
    if (PFX(is_zero)(b)) return 0;
    ET Z1s, Z2s, l, r, Z1c, Z2c;
    F_sqr(&Z1s, &a->Z); F_sqr(&Z2s, &b->Z);
    F_mul(&l, &a->X, &Z2s); F_mul(&r, &b->X, &Z1s);
    if (!F_eq(&l, &r)) return 0;
    F_mul(&Z1c, &a->Z, &Z1s); F_mul(&Z2c, &b->Z, &Z2s);
    F_mul(&l, &a->Y, &Z2c); F_mul(&r, &b->Y, &Z1c);
    return F_eq(&l, &r);
}

static void PFX(to_affine)(PT* o, const PT* a)
{
    if (PFX(is_zero)(a)) { PFX(zero)(o); return; }
    ET zi, z2, z3;
    F_inv(&zi, &a->Z); F_sqr(&z2, &zi); F_mul(&z3, &z2, &zi);
    F_mul(&o->X, &a->X, &z2); F_mul(&o->Y, &a->Y, &z3); F_one(&o->Z);
}

/* k: canonical scalar limbs (the as_bigint() of the Montgomery input) */
static void PFX(mul)(PT* o, const PT* P, const uint64_t k[4])
{
    PT res; PFX(zero)(&res);
    int found = 0;
    for (int i = 255; i >= 0; i--) {
        if (found) PFX(dbl)(&res, &res);
        if ((k[i >> 6] >> (i & 63)) & 1) { found = 1; PFX(add)(&res, &res, P); }
    }
    *o = res;
}

/* y^2 = x^3 + b Z^6 */
static int PFX(well_formed)(const PT* a, const ET* bcoef)
{
    if (PFX(is_zero)(a)) return 1;
    ET X2, Y2, Z2, X3, Z3, Z6, t;
    F_sqr(&X2, &a->X); F_sqr(&Y2, &a->Y); F_sqr(&Z2, &a->Z);
    F_mul(&X3, &a->X, &X2); F_mul(&Z3, &a->Z, &Z2); F_sqr(&Z6, &Z3);
    F_mul(&t, bcoef, &Z6); F_add(&t, &X3, &t);
    return F_eq(&Y2, &t);
}

/* Jacobian -> affine for a whole array with one inversion (Montgomery's
 * batch trick, the idea of batch_to_special_all_non_zeros,
 * alt_bn128_g1.cu:394-415); infinity maps to affine (0, 0). */
static void PFX(batch_to_aff)(const PT* in, ET* xy, size_t n)
{
    ET* pre = (ET*)malloc(sizeof(ET) * (n + 1));
    ET acc; F_one(&acc);
    for (size_t i = 0; i < n; i++) {
        pre[i] = acc;
        if (!PFX(is_zero)(&in[i])) F_mul(&acc, &acc, &in[i].Z);
    }
    ET inv; F_inv(&inv, &acc);
    for (size_t i = n; i-- > 0;) {
        if (PFX(is_zero)(&in[i])) { F_zero(&xy[2 * i]); F_zero(&xy[2 * i + 1]); continue; }
        ET zi, z2, z3;
        F_mul(&zi, &inv, &pre[i]);
        F_mul(&inv, &inv, &in[i].Z);
        F_sqr(&z2, &zi); F_mul(&z3, &z2, &zi);
        F_mul(&xy[2 * i], &in[i].X, &z2);
        F_mul(&xy[2 * i + 1], &in[i].Y, &z3);
    }
    free(pre);
}

static void PFX(from_aff)(PT* o, const ET* xy)
{
    if (F_iszero(&xy[0]) && F_iszero(&xy[1])) { PFX(zero)(o); return; }
    o->X = xy[0]; o->Y = xy[1]; F_one(&o->Z);
}

/* unsigned c-bit windows; buckets via madd; running sums; Horner over
 * windows (the group element equals sum s_i P_i, whatever the schedule) */
static void PFX(pippenger)(const uint64_t* canon, const ET* xy, size_t n, PT* out)
{
    int c = n < 64 ? 4 : n < 4096 ? 8 : n < (1u << 17) ? 12 : 15;
    int W = (256 + c - 1) / c;
    PT* win = (PT*)malloc(sizeof(PT) * W);
    #pragma omp parallel for schedule(dynamic, 1)
    for (int w = 0; w < W; w++) {
        size_t nb = ((size_t)1 << c) - 1;
        PT* bk = (PT*)malloc(sizeof(PT) * nb);
        for (size_t j = 0; j < nb; j++) PFX(zero)(&bk[j]);
        for (size_t i = 0; i < n; i++) {
            const uint64_t* k = canon + 4 * i;
            int lo = w * c;
            uint64_t d = 0;
            for (int b = 0; b < c && lo + b < 256; b++) d |= ((k[(lo + b) >> 6] >> ((lo + b) & 63)) & 1ull) << b;
            if (!d) continue;
            PT P; PFX(from_aff)(&P, xy + 2 * i);
            PFX(madd)(&bk[d - 1], &bk[d - 1], &P);
        }
        PT run, acc; PFX(zero)(&run); PFX(zero)(&acc);
        for (size_t j = nb; j-- > 0;) { PFX(add)(&run, &run, &bk[j]); PFX(add)(&acc, &acc, &run); }
        win[w] = acc;
        free(bk);
    }
    PT res; PFX(zero)(&res);
    for (int w = W - 1; w >= 0; w--) {
        for (int b = 0; b < c; b++) PFX(dbl)(&res, &res);
        PFX(add)(&res, &res, &win[w]);
    }
    *out = res;
    free(win);
}

/* comb tables T[j][d] = d * 2^(8j) * G, j < 32, 1 <= d < 256, as affine
 * Jacobian (Z = 1); k*G = sum_j T[j][byte_j(k)] by madd. */
static void PFX(fixed_base)(const PT* G, const uint64_t* canon, ET* xy, size_t n)
{
    PT* T = (PT*)malloc(sizeof(PT) * 32 * 256);
    PT base = *G;
    for (int j = 0; j < 32; j++) {
        PFX(zero)(&T[j * 256]);
        T[j * 256 + 1] = base;
        for (int d = 2; d < 256; d++) PFX(add)(&T[j * 256 + d], &T[j * 256 + d - 1], &base);
        for (int b = 0; b < 8; b++) PFX(dbl)(&base, &base);
    }
    ET* txy = (ET*)malloc(sizeof(ET) * 2 * 32 * 256);
    PFX(batch_to_aff)(T, txy, 32 * 256);
    for (int i = 0; i < 32 * 256; i++) PFX(from_aff)(&T[i], txy + 2 * i);
    free(txy);
    PT* R = (PT*)malloc(sizeof(PT) * n);
    #pragma omp parallel for schedule(static, 256)
    for (size_t i = 0; i < n; i++) {
        PT acc; PFX(zero)(&acc);
        for (int j = 0; j < 32; j++) {
            unsigned d = (canon[4 * i + (j >> 3)] >> (8 * (j & 7))) & 255u;
            if (d) PFX(madd)(&acc, &acc, &T[j * 256 + d]);
        }
        R[i] = acc;
    }
    const size_t CH = 4096;
    #pragma omp parallel for schedule(dynamic, 1)
    for (size_t s = 0; s < n; s += CH) PFX(batch_to_aff)(R + s, xy + 2 * s, (n - s < CH) ? n - s : CH);
    free(R); free(T);
}
