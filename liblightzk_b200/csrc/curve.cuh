// curve.cuh -- Fq2 and BN254 curve arithmetic for G1 (over Fq) and G2 (over
// Fq2), generic in the coordinate field.
//
// Three point forms:
//   Aff<F>  {x, y}          bases in HBM (64 B for G1, 128 B for G2); the
//                           point at infinity is x = y = 0 (not on the curve).
//   XYZZ<F> {X, Y, ZZ, ZZZ} bucket accumulators: x = X/ZZ, y = Y/ZZZ; the
//                           point at infinity is ZZ = 0.  Mixed addition costs
//                           8M+2S and needs no inversion.
//   Jac<F>  {X, Y, Z}       the reference's output form, x = X/Z^2,
//                           y = Y/Z^3 (alt_bn128_g1.cuh:27); the point at
//                           infinity is written as (0, 1, 0) like libff's
//                           G1_zero (alt_bn128_init.cu:127-129).
// The XYZZ formulas are the published "xyzz" set for short Weierstrass
// curves with a = 0 (Bernstein-Lange EFD: madd-2008-s, mdbl-2008-s-1,
// add-2008-s, dbl-2008-s-1); results are compared with the reference only
// after normalisation to affine, which is representation independent.
#pragma once
#include "field52.cuh"

namespace lzk {

// ---------------- Fq2 = Fq[i] / (i^2 + 1) ----------------
struct Fq2 {
    Fq c0, c1;
    __device__ __forceinline__ static Fq2 zero() { return {Fq::zero(), Fq::zero()}; }
    __device__ __forceinline__ static Fq2 one() { return {Fq::one(), Fq::zero()}; }
    __device__ __forceinline__ bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
    __device__ __forceinline__ bool operator==(const Fq2& o) const { return c0 == o.c0 && c1 == o.c1; }
};
__device__ __forceinline__ Fq2 add(const Fq2& a, const Fq2& b) { return {add(a.c0, b.c0), add(a.c1, b.c1)}; }
__device__ __forceinline__ Fq2 sub(const Fq2& a, const Fq2& b) { return {sub(a.c0, b.c0), sub(a.c1, b.c1)}; }
__device__ __forceinline__ Fq2 neg(const Fq2& a) { return {neg(a.c0), neg(a.c1)}; }
__device__ __forceinline__ Fq2 dbl(const Fq2& a) { return {dbl(a.c0), dbl(a.c1)}; }
// p^2 (Fq), 16 limbs
__host__ __device__ constexpr uint32_t fq_p2(int i)
{
    return i == 0 ? 0x275d69b1u : i == 1 ? 0x3b5458a2u : i == 2 ? 0x09eac101u : i == 3 ? 0xa602072du
         : i == 4 ? 0x6d96cadcu : i == 5 ? 0x4a50189cu : i == 6 ? 0x7a1242c8u : i == 7 ? 0x04689e95u
         : i == 8 ? 0x34c6b38du : i == 9 ? 0x26edfa5cu : i == 10 ? 0x16375606u : i == 11 ? 0xb00b8551u
         : i == 12 ? 0x0348d21cu : i == 13 ? 0x599a6f7cu : i == 14 ? 0x763cbf9cu : 0x0925c4b8u;
}

// Karatsuba with lazy reduction: the three 512-bit products stay unreduced,
//   c0 = a0 b0 + p^2 - a1 b1,   c1 = (a0 + a1)(b0 + b1) - a0 b0 - a1 b1,
// both in (0, 2p^2) < p 2^256, and only c0 and c1 are reduced (two
// Montgomery reductions instead of three).  The operand sums are < 2p and
// fit 8 limbs unreduced.  The reductions give (a0 b0 - a1 b1) R^-1 and
// (a0 b1 + a1 b0) R^-1 mod p below 2p, so after the final conditional
// subtraction the result is the canonical value that three separately
// reduced products give.
__host__ __device__ __forceinline__ void fq2_mul_lazy(uint32_t c0[8], uint32_t c1[8], const uint32_t a0[8],
                                                      const uint32_t a1[8], const uint32_t b0[8], const uint32_t b1[8])
{
    uint32_t t0[16], t1[16], t2[16], sa[8], sb[8];
    mul_wide(t0, a0, b0);
    mul_wide(t1, a1, b1);
    uint32_t ca = 0, cb = 0;
    _Pragma("unroll") for (int k = 0; k < 8; k++) {
        uint64_t x = (uint64_t)a0[k] + a1[k] + ca;
        sa[k] = (uint32_t)x; ca = (uint32_t)(x >> 32);
        uint64_t y = (uint64_t)b0[k] + b1[k] + cb;
        sb[k] = (uint32_t)y; cb = (uint32_t)(y >> 32);
    }
    mul_wide(t2, sa, sb);
    // t2 -= t0 + t1 ; t0 = t0 + p^2 - t1
    uint32_t b2 = 0, c = 0, b0r = 0;
    _Pragma("unroll") for (int k = 0; k < 16; k++) {
        uint64_t d = (uint64_t)t2[k] - t0[k] - t1[k] - b2;
        t2[k] = (uint32_t)d;
        b2 = (uint32_t)(0u - (uint32_t)(d >> 32));   // borrow 0, 1 or 2
        uint64_t e = (uint64_t)t0[k] + fq_p2(k) + c;
        c = (uint32_t)(e >> 32);
        uint64_t f = (uint64_t)(uint32_t)e - t1[k] - b0r;
        t0[k] = (uint32_t)f;
        b0r = (uint32_t)(f >> 63);
    }
    uint32_t r0[8], r1[8];
    redc_wide<FqP>(r0, t0);
    redc_wide<FqP>(r1, t2);
    _Pragma("unroll") for (int k = 0; k < 8; k++) { c0[k] = r0[k]; c1[k] = r1[k]; }
}

__device__ __forceinline__ Fq2 mul(const Fq2& a, const Fq2& b)
{
    uint32_t r0[8], r1[8];
    fq2_mul_lazy(r0, r1, a.c0.v, a.c1.v, b.c0.v, b.c1.v);
    return {final_sub<FqP>(r0), final_sub<FqP>(r1)};
}
// (a0 + a1 i)^2 = (a0+a1)(a0-a1) + 2 a0 a1 i: 2 Fq products
__device__ __forceinline__ Fq2 sqr(const Fq2& a)
{
    Fq ab = mul(a.c0, a.c1);
    return {mul(add(a.c0, a.c1), sub(a.c0, a.c1)), dbl(ab)};
}
static __device__ __noinline__ Fq2 inverse(const Fq2& a)
{
    Fq t = inverse(add(sqr(a.c0), sqr(a.c1)));
    return {mul(a.c0, t), neg(mul(a.c1, t))};
}

// Products used by the point formulas: out-of-line Fq products (mul_call),
// Fq2 products built from them.
__device__ __forceinline__ Fq cmul(const Fq& a, const Fq& b) { return mul52_call(a, b); }
__device__ __forceinline__ Fq csqr(const Fq& a) { return mul52_call(a, a); }
// One out-of-line body per Fq2 product (and square): its limb products are
// inlined there, so they interleave, and the call boundary moves two Fq2
// operands once instead of once per Fq product.
// Both run their Fq products on the FP64 pipe (field52.cuh).
static __device__ __noinline__ Fq2 fq2_mul_call(const Fq2 a, const Fq2 b)
{
    Fq2 r;
    fq2_mul52(r.c0.v, r.c1.v, a.c0.v, a.c1.v, b.c0.v, b.c1.v);
    return r;
}
static __device__ __noinline__ Fq2 fq2_sqr_call(const Fq2 a)
{
    Fq s = add(a.c0, a.c1), d = sub(a.c0, a.c1);
    Fq x = mul52(s, d), y = mul52(a.c0, a.c1);
    return {x, dbl(y)};
}
__device__ __forceinline__ Fq2 cmul(const Fq2& a, const Fq2& b) { return fq2_mul_call(a, b); }
__device__ __forceinline__ Fq2 csqr(const Fq2& a) { return fq2_sqr_call(a); }
// two independent products: Fq pairs share one out-of-line body
__device__ __forceinline__ void cmul2(Fq& r0, Fq& r1, const Fq& a0, const Fq& b0, const Fq& a1, const Fq& b1)
{
    FpPair<FqP> r = mul52x2_call(a0, b0, a1, b1);
    r0 = r.a;
    r1 = r.b;
}
// two independent squares: Fq squares share one body (15 limb products per
// square instead of 25: G1 accumulation 3.6 % faster)
__device__ __forceinline__ void csqr2(Fq& r0, Fq& r1, const Fq& a, const Fq& b)
{
    FpPair<FqP> r = sqr52x2_call(a, b);
    r0 = r.a;
    r1 = r.b;
}
// Fq2 pairs stay two calls: one body holding six interleaved Fq products
// needs 255 registers and ran the G2 accumulation 40 % slower.
__device__ __forceinline__ void cmul2(Fq2& r0, Fq2& r1, const Fq2& a0, const Fq2& b0, const Fq2& a1, const Fq2& b1)
{
    r0 = cmul(a0, b0);
    r1 = cmul(a1, b1);
}
__device__ __forceinline__ void csqr2(Fq2& r0, Fq2& r1, const Fq2& a, const Fq2& b)
{
    r0 = cmul(a, a);
    r1 = cmul(b, b);
}

// ---------------- point forms ----------------
template <class F> struct Aff { F x, y; };
template <class F> struct XYZZ { F X, Y, ZZ, ZZZ; };
template <class F> struct Jac { F X, Y, Z; };

template <class F> __device__ __forceinline__ bool aff_is_inf(const Aff<F>& p) { return p.x.is_zero() && p.y.is_zero(); }

template <class F> __device__ __forceinline__ XYZZ<F> xyzz_inf() { return {F::zero(), F::zero(), F::zero(), F::zero()}; }
template <class F> __device__ __forceinline__ bool xyzz_is_inf(const XYZZ<F>& p) { return p.ZZ.is_zero(); }
template <class F> __device__ __forceinline__ XYZZ<F> xyzz_from_aff(const Aff<F>& a)
{
    if (aff_is_inf(a)) return xyzz_inf<F>();
    return {a.x, a.y, F::one(), F::one()};
}

// 2*(x, y) for affine input (mdbl-2008-s-1)
template <class F> __device__ __forceinline__ XYZZ<F> xyzz_mdbl(const Aff<F>& a)
{
    F U = dbl(a.y);
    F V = csqr(U);
    F W = cmul(U, V);
    F S = cmul(a.x, V);
    F x2 = csqr(a.x);
    F M = add(dbl(x2), x2);
    F X3 = sub(csqr(M), dbl(S));
    F Y3 = sub(cmul(M, sub(S, X3)), cmul(W, a.y));
    return {X3, Y3, V, W};
}

// 2*P (dbl-2008-s-1); independent products in pairs
template <class F> __device__ __forceinline__ XYZZ<F> xyzz_dbl(const XYZZ<F>& p)
{
    if (xyzz_is_inf(p)) return p;
    F U = dbl(p.Y);
    F V, x2;
    csqr2(V, x2, U, p.X);
    F W, S;
    cmul2(W, S, U, V, p.X, V);
    F M = add(dbl(x2), x2);
    F MM, ZZ3;
    cmul2(MM, ZZ3, M, M, V, p.ZZ);
    F X3 = sub(MM, dbl(S));
    F t, u;
    cmul2(t, u, M, sub(S, X3), W, p.Y);
    F ZZZ3 = cmul(W, p.ZZZ);
    return {X3, sub(t, u), ZZ3, ZZZ3};
}

// P + Q with Q affine (madd-2008-s); handles infinity, P == Q and P == -Q.
// Independent products are issued in pairs.
template <class F> __device__ __forceinline__ XYZZ<F> xyzz_madd(const XYZZ<F>& p, const Aff<F>& q)
{
    if (aff_is_inf(q)) return p;
    if (xyzz_is_inf(p)) return xyzz_from_aff(q);
    F U2, S2;
    cmul2(U2, S2, q.x, p.ZZ, q.y, p.ZZZ);
    F P = sub(U2, p.X);
    F R = sub(S2, p.Y);
    if (P.is_zero()) {
        if (R.is_zero()) return xyzz_mdbl(q);
        return xyzz_inf<F>();
    }
    F PP, RR;
    csqr2(PP, RR, P, R);
    F PPP, Q;
    cmul2(PPP, Q, P, PP, p.X, PP);
    F X3 = sub(sub(RR, PPP), dbl(Q));
    F t, ZZ3;
    cmul2(t, ZZ3, R, sub(Q, X3), p.ZZ, PP);
    F u, ZZZ3;
    cmul2(u, ZZZ3, p.Y, PPP, p.ZZZ, PPP);
    return {X3, sub(t, u), ZZ3, ZZZ3};
}

// G2 mixed addition: the same products, one Fq2 product per call (pairs buy
// nothing there), each issued as soon as its inputs exist so that the base
// point and the old ZZ, X, ZZZ die early: fewer values live across the calls
// (spills of the 168-register accumulation 368/508 -> 176/380 bytes, 1.3 %
// faster).
template <> __device__ __forceinline__ XYZZ<Fq2> xyzz_madd<Fq2>(const XYZZ<Fq2>& p, const Aff<Fq2>& q)
{
    if (aff_is_inf(q)) return p;
    if (xyzz_is_inf(p)) return xyzz_from_aff(q);
    Fq2 P = sub(cmul(q.x, p.ZZ), p.X);
    Fq2 R = sub(cmul(q.y, p.ZZZ), p.Y);
    if (P.is_zero()) {
        if (R.is_zero()) return xyzz_mdbl(q);
        return xyzz_inf<Fq2>();
    }
    Fq2 PP = cmul(P, P);
    Fq2 ZZ3 = cmul(p.ZZ, PP);
    Fq2 PPP = cmul(P, PP);
    Fq2 Q = cmul(p.X, PP);
    Fq2 ZZZ3 = cmul(p.ZZZ, PPP);
    Fq2 RR = cmul(R, R);
    Fq2 X3 = sub(sub(RR, PPP), dbl(Q));
    Fq2 t = cmul(R, sub(Q, X3));
    Fq2 u = cmul(p.Y, PPP);
    return {X3, sub(t, u), ZZ3, ZZZ3};
}

// P + Q (add-2008-s); independent products in pairs
template <class F> __device__ __forceinline__ XYZZ<F> xyzz_add(const XYZZ<F>& p, const XYZZ<F>& q)
{
    if (xyzz_is_inf(q)) return p;
    if (xyzz_is_inf(p)) return q;
    F U1, U2, S1, S2;
    cmul2(U1, U2, p.X, q.ZZ, q.X, p.ZZ);
    cmul2(S1, S2, p.Y, q.ZZZ, q.Y, p.ZZZ);
    F P = sub(U2, U1);
    F R = sub(S2, S1);
    if (P.is_zero()) {
        if (R.is_zero()) return xyzz_dbl(p);
        return xyzz_inf<F>();
    }
    F PP, RR;
    csqr2(PP, RR, P, R);
    F PPP, Q;
    cmul2(PPP, Q, P, PP, U1, PP);
    F X3 = sub(sub(RR, PPP), dbl(Q));
    F t, u;
    cmul2(t, u, R, sub(Q, X3), S1, PPP);
    F zz, zzz;
    cmul2(zz, zzz, p.ZZ, q.ZZ, p.ZZZ, q.ZZZ);
    F ZZ3, ZZZ3;
    cmul2(ZZ3, ZZZ3, zz, PP, zzz, PPP);
    return {X3, sub(t, u), ZZ3, ZZZ3};
}

template <class F> __device__ __forceinline__ XYZZ<F> xyzz_neg(const XYZZ<F>& p) { return {p.X, neg(p.Y), p.ZZ, p.ZZZ}; }

// XYZZ -> Jacobian without inversion: Z = ZZ*ZZZ, X = X*ZZ*ZZZ^2, Y = Y*ZZ^3*ZZZ^2
template <class F> __device__ __forceinline__ Jac<F> xyzz_to_jac(const XYZZ<F>& p)
{
    if (xyzz_is_inf(p)) return {F::zero(), F::one(), F::zero()};
    F zzz2 = csqr(p.ZZZ);
    F Z = cmul(p.ZZ, p.ZZZ);
    F X = cmul(cmul(p.X, p.ZZ), zzz2);
    F zz3 = cmul(csqr(p.ZZ), p.ZZ);
    F Y = cmul(cmul(p.Y, zz3), zzz2);
    return {X, Y, Z};
}

template <class F> __device__ __forceinline__ XYZZ<F> jac_to_xyzz(const Jac<F>& p)
{
    if (p.Z.is_zero()) return xyzz_inf<F>();
    F z2 = csqr(p.Z);
    return {p.X, p.Y, z2, cmul(z2, p.Z)};
}

// Out-of-line copies for the cold kernels (fix-up, reduction levels, window
// combination, table building): one body per kernel instead of one per call
// site keeps code size and compile time down where the adds are not the
// bottleneck.
template <class F> __device__ __noinline__ XYZZ<F> xyzz_add_cold(const XYZZ<F> p, const XYZZ<F> q) { return xyzz_add(p, q); }
template <class F> __device__ __noinline__ XYZZ<F> xyzz_dbl_cold(const XYZZ<F> p) { return xyzz_dbl(p); }

// ---------------- warp-uniform point operations ----------------
// For chains of dependent operations on one point (the window combination,
// the weighting doublings of the bucket reduction, the proof assembly).  A
// lone warp running such a chain keeps its SM sub-partition's multiplier
// pipe busy, and a warp instruction costs the same for one active lane as
// for 32.  So all 32 lanes hold the same operands, each stage of the formula
// computes its independent products one per lane, and shuffles hand every
// lane all of them: a stage of up to six products takes the time of one.
// add-2008-s becomes four dependent stages (6, 2, 3, 3 products) instead of
// seven pairs, dbl-2008-s-1 three (2, 4, 3) instead of six, with the same
// products and results as xyzz_add / xyzz_dbl.  Callers: every lane of the
// warp, converged, with equal arguments; every lane gets the result.
template <class F>
__device__ __forceinline__ F shfl_elem(const F& x, int src)
{
    F r;
    const uint32_t* s = reinterpret_cast<const uint32_t*>(&x);
    uint32_t* o = reinterpret_cast<uint32_t*>(&r);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(F) / 4); i++) o[i] = __shfl_sync(0xffffffffu, s[i], src);
    return r;
}
template <int N, class F>
__device__ __forceinline__ void warp_products(F (&r)[N], const F (&a)[N], const F (&b)[N])
{
    const int lane = threadIdx.x & 31;
    F x = a[0], y = b[0];
    _Pragma("unroll") for (int k = 1; k < N; k++) {
        if (lane == k) { x = a[k]; y = b[k]; }
    }
    F z = cmul(x, y);
    _Pragma("unroll") for (int k = 0; k < N; k++) r[k] = shfl_elem(z, k);
}

template <class F> __device__ __noinline__ XYZZ<F> xyzz_dbl_warp(const XYZZ<F> p)
{
    if (xyzz_is_inf(p)) return p;
    F U = dbl(p.Y);
    F s1[2];
    { F a[2] = {U, p.X}; warp_products<2>(s1, a, a); }
    F V = s1[0], x2 = s1[1];
    F M = add(dbl(x2), x2);
    F s2[4];
    { F a[4] = {U, p.X, V, M}; F b[4] = {V, V, p.ZZ, M}; warp_products<4>(s2, a, b); }
    F W = s2[0], S = s2[1], ZZ3 = s2[2], MM = s2[3];
    F X3 = sub(MM, dbl(S));
    F s3[3];
    { F a[3] = {M, W, W}; F b[3] = {sub(S, X3), p.Y, p.ZZZ}; warp_products<3>(s3, a, b); }
    return {X3, sub(s3[0], s3[1]), ZZ3, s3[2]};
}

template <class F> __device__ __noinline__ XYZZ<F> xyzz_add_warp(const XYZZ<F> p, const XYZZ<F> q)
{
    if (xyzz_is_inf(q)) return p;
    if (xyzz_is_inf(p)) return q;
    F s1[6];
    { F a[6] = {p.X, q.X, p.Y, q.Y, p.ZZ, p.ZZZ}; F b[6] = {q.ZZ, p.ZZ, q.ZZZ, p.ZZZ, q.ZZ, q.ZZZ}; warp_products<6>(s1, a, b); }
    F U1 = s1[0], S1 = s1[2], zz = s1[4], zzz = s1[5];
    F P = sub(s1[1], U1);
    F R = sub(s1[3], S1);
    if (P.is_zero()) {
        if (R.is_zero()) return xyzz_dbl_warp(p);
        return xyzz_inf<F>();
    }
    F s2[2];
    { F a[2] = {P, R}; warp_products<2>(s2, a, a); }
    F PP = s2[0], RR = s2[1];
    F s3[3];
    { F a[3] = {P, U1, zz}; F b[3] = {PP, PP, PP}; warp_products<3>(s3, a, b); }
    F PPP = s3[0], Q = s3[1], ZZ3 = s3[2];
    F X3 = sub(sub(RR, PPP), dbl(Q));
    F s4[3];
    { F a[3] = {R, S1, zzz}; F b[3] = {sub(Q, X3), PPP, PPP}; warp_products<3>(s4, a, b); }
    return {X3, sub(s4[0], s4[1]), ZZ3, s4[2]};
}

// XYZZ -> Jacobian for a whole warp (products in two stages of two and one
// of two)
template <class F> __device__ __forceinline__ Jac<F> xyzz_to_jac_warp(const XYZZ<F>& p)
{
    if (xyzz_is_inf(p)) return {F::zero(), F::one(), F::zero()};
    F s1[3];
    { F a[3] = {p.ZZZ, p.ZZ, p.ZZ}; F b[3] = {p.ZZZ, p.ZZZ, p.ZZ}; warp_products<3>(s1, a, b); }
    F zzz2 = s1[0], Z = s1[1], zz2 = s1[2];
    F s2[2];
    { F a[2] = {p.X, zz2}; F b[2] = {p.ZZ, p.ZZ}; warp_products<2>(s2, a, b); }
    F s3[2];
    { F a[2] = {s2[0], p.Y}; F b[2] = {zzz2, s2[1]}; warp_products<2>(s3, a, b); }
    F s4[1];
    { F a[1] = {s3[1]}; F b[1] = {zzz2}; warp_products<1>(s4, a, b); }
    return {s3[0], s4[0], Z};
}

}  // namespace lzk
