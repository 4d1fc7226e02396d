// field52.cuh -- Montgomery products of BN254 field elements on the FP64 pipe.
//
// B200 keeps full-rate FP64 (measured 56 DFMA per SM per clock against 24
// 32x32->64-bit integer products), so a 254-bit product is cheaper when its
// limb products run as exact double-precision FMAs:
//
//   * operands are cut into five 52-bit limbs held exactly in doubles;
//   * a limb product a*b < 2^104 is split exactly into H*2^52 + L with three
//     FP64 operations: h = fma_rz(a, b, 2^104) = 2^104 + H*2^52 (rounding
//     toward zero at a 2^52 ulp is the floor), t = (2^104 + 2^52) - h =
//     2^52 - H*2^52 (exact), l = fma(a, b, t) = 2^52 + L (exact: L < 2^52).
//     The bit patterns of h and l are a fixed exponent field plus H and L, so
//     column sums are plain 64-bit integer additions of those bits, with the
//     exponent fields removed once per column by its starting value;
//   * Montgomery reduction word by word with 52-bit words and R' = 2^260,
//     m_i = c_i * (-p^-1) mod 2^52 on the integer multiplier; the low half of
//     m_i * p_0 is never formed: column i plus it is a multiple of 2^52, so
//     its carry is ceil(c_i / 2^52).
//
// The interface is that of the 32-bit-limb product (field.cuh): canonical
// 8x32-bit Montgomery operands with R = 2^256.  One operand enters as 16*a,
// so the R' = 2^260 product 16ab / 2^260 is ab / 2^256; with a, b < p the
// result is below (16p^2 + 2^260 p) / 2^260 < 2p and one conditional
// subtraction makes it canonical.  Results are bit-identical to mul().
//
// The split is a published technique (exact two-FMA product splitting as in
// Dekker/Veltkamp-style error-free transformations, with the biased-exponent
// integer view used for multi-precision arithmetic on GPUs by Emmart, Zheng
// and Weems, ARITH 2018); the code here is written from that description.
#pragma once
#include "field.cuh"

namespace lzk {

constexpr uint64_t kM52 = (1ull << 52) - 1;
constexpr uint64_t kHiBias = 0x4670000000000000ull;   // bit pattern of 2^104
constexpr uint64_t kLoBias = 0x4330000000000000ull;   // bit pattern of 2^52

// radix-2^52 limbs of the moduli and -p^-1 mod 2^52
template <class P> struct P52;
template <> struct P52<FqP> {
    __host__ __device__ static constexpr uint64_t p(int i)
    {
        return i == 0 ? 0x8c16d87cfd47ull : i == 1 ? 0x916871ca8d3c2ull : i == 2 ? 0x181585d97816aull
             : i == 3 ? 0xa029b85045b68ull : 0x30644e72e131ull;
    }
    static constexpr uint64_t ninv = 0x20782e4866389ull;
};
template <> struct P52<FrP> {
    __host__ __device__ static constexpr uint64_t p(int i)
    {
        return i == 0 ? 0x1f593f0000001ull : i == 1 ? 0x4879b9709143eull : i == 2 ? 0x181585d2833e8ull
             : i == 3 ? 0xa029b85045b68ull : 0x30644e72e131ull;
    }
    static constexpr uint64_t ninv = 0x1f593efffffffull;
};

// Number of biased terms each column receives: products a_i*b_j put their
// low half in column i+j and their high half in i+j+1; reduction step i puts
// m_i*p_j's high half in i+j+1 and, for j >= 1, its low half in i+j.
__host__ __device__ constexpr uint64_t col_bias52(int k)
{
    uint64_t b = 0;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            if (i + j == k) b += kLoBias;        // a_i b_j low
            if (i + j + 1 == k) b += kHiBias;    // a_i b_j high
            if (i + j + 1 == k) b += kHiBias;    // m_i p_j high
            if (j >= 1 && i + j == k) b += kLoBias;  // m_i p_j low
        }
    return b;
}

// exact double of an integer x < 2^52
__device__ __forceinline__ double u52_to_d(uint64_t x)
{
    return __dsub_rn(__longlong_as_double((long long)(x | kLoBias)), 0x1p52);
}

// a*b = H*2^52 + L for integers a, b < 2^52: hi = kHiBias + H, lo = kLoBias + L
__device__ __forceinline__ void split52(double a, double b, uint64_t& hi, uint64_t& lo)
{
    double h = __fma_rz(a, b, 0x1p104);
    double t = __dsub_rn(0x1.0000000000001p104, h);    // 2^104 + 2^52 - h
    double l = __fma_rn(a, b, t);
    hi = (uint64_t)__double_as_longlong(h);
    lo = (uint64_t)__double_as_longlong(l);
}
// high half only
__device__ __forceinline__ uint64_t split52_hi(double a, double b)
{
    return (uint64_t)__double_as_longlong(__fma_rz(a, b, 0x1p104));
}

// x (< 2^256, 8 limbs) times 2^S as five 52-bit limbs (x * 2^S < 2^260)
template <int S>
__device__ __forceinline__ void to_limbs52(uint64_t l[5], const uint32_t v[8])
{
    uint64_t w0 = (uint64_t)v[0] | (uint64_t)v[1] << 32, w1 = (uint64_t)v[2] | (uint64_t)v[3] << 32;
    uint64_t w2 = (uint64_t)v[4] | (uint64_t)v[5] << 32, w3 = (uint64_t)v[6] | (uint64_t)v[7] << 32;
    l[0] = (w0 << S) & kM52;
    l[1] = ((w0 >> (52 - S)) | (w1 << (12 + S))) & kM52;
    l[2] = ((w1 >> (40 - S)) | (w2 << (24 + S))) & kM52;
    l[3] = ((w2 >> (28 - S)) | (w3 << (36 + S))) & kM52;
    l[4] = w3 >> (16 - S);
}
template <int S>
__device__ __forceinline__ void to_d52(double d[5], const uint32_t v[8])
{
    uint64_t l[5];
    to_limbs52<S>(l, v);
    _Pragma("unroll") for (int i = 0; i < 5; i++) d[i] = u52_to_d(l[i]);
}
// five 52-bit limbs (value < 2^256) to 8 limbs
__device__ __forceinline__ void from_limbs52(uint32_t v[8], const uint64_t r[5])
{
    uint64_t w0 = r[0] | r[1] << 52, w1 = r[1] >> 12 | r[2] << 40;
    uint64_t w2 = r[2] >> 24 | r[3] << 28, w3 = r[3] >> 36 | r[4] << 16;
    v[0] = (uint32_t)w0; v[1] = (uint32_t)(w0 >> 32); v[2] = (uint32_t)w1; v[3] = (uint32_t)(w1 >> 32);
    v[4] = (uint32_t)w2; v[5] = (uint32_t)(w2 >> 32); v[6] = (uint32_t)w3; v[7] = (uint32_t)(w3 >> 32);
}

// Montgomery product in radix 2^52: r = a*b / 2^260 mod p, r < 2p, as
// normalised 52-bit limbs, for limbs a, b < 2^52 with a*b < p * 2^260.
template <class P>
__device__ __forceinline__ void mont52_core(uint64_t r[5], const double a[5], const double b[5])
{
    uint64_t c[10];
    _Pragma("unroll") for (int k = 0; k < 10; k++) c[k] = 0 - col_bias52(k);
    _Pragma("unroll") for (int i = 0; i < 5; i++)
        _Pragma("unroll") for (int j = 0; j < 5; j++) {
            uint64_t hi, lo;
            split52(a[i], b[j], hi, lo);
            c[i + j] += lo;
            c[i + j + 1] += hi;
        }
    _Pragma("unroll") for (int i = 0; i < 5; i++) {
        const double m = u52_to_d((c[i] * P52<P>::ninv) & kM52);
        c[i + 1] += split52_hi(m, (double)P52<P>::p(0));
        _Pragma("unroll") for (int j = 1; j < 5; j++) {
            uint64_t hi, lo;
            split52(m, (double)P52<P>::p(j), hi, lo);
            c[i + j] += lo;
            c[i + j + 1] += hi;
        }
        c[i + 1] += (c[i] + kM52) >> 52;     // column i plus lo(m p_0) is a multiple of 2^52
    }
    _Pragma("unroll") for (int k = 5; k < 9; k++) {
        r[k - 5] = c[k] & kM52;
        c[k + 1] += c[k] >> 52;
    }
    r[4] = c[9];
}

// Bias of the split terms a product a*b leaves in column k (prod_cols52), and
// of the terms one Montgomery reduction adds to column k (redc52).
__host__ __device__ constexpr uint64_t prod_bias52(int k)
{
    uint64_t b = 0;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            if (i + j == k) b += kLoBias;
            if (i + j + 1 == k) b += kHiBias;
        }
    return b;
}
__host__ __device__ constexpr uint64_t red_bias52(int k)
{
    uint64_t b = 0;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            if (i + j + 1 == k) b += kHiBias;
            if (j >= 1 && i + j == k) b += kLoBias;
        }
    return b;
}

// c[k] += the split terms of a*b in column k (each term carries its bias)
__device__ __forceinline__ void prod_cols52(uint64_t c[10], const double a[5], const double b[5])
{
    _Pragma("unroll") for (int i = 0; i < 5; i++)
        _Pragma("unroll") for (int j = 0; j < 5; j++) {
            uint64_t hi, lo;
            split52(a[i], b[j], hi, lo);
            c[i + j] += lo;
            c[i + j + 1] += hi;
        }
}

// Montgomery reduction of an integer given as ten signed 64-bit columns
// (true values, radix 2^52, total in [0, p * 2^260)): r = total / 2^260 mod p,
// r < 2p, as normalised limbs.  The columns may be negative individually.
template <class P>
__device__ __forceinline__ void redc52(uint64_t r[5], uint64_t c[10])
{
    _Pragma("unroll") for (int k = 1; k < 10; k++) c[k] -= red_bias52(k);
    _Pragma("unroll") for (int i = 0; i < 5; i++) {
        const double m = u52_to_d((c[i] * P52<P>::ninv) & kM52);
        c[i + 1] += split52_hi(m, (double)P52<P>::p(0));
        _Pragma("unroll") for (int j = 1; j < 5; j++) {
            uint64_t hi, lo;
            split52(m, (double)P52<P>::p(j), hi, lo);
            c[i + j] += lo;
            c[i + j + 1] += hi;
        }
        c[i + 1] += (uint64_t)((int64_t)(c[i] + kM52) >> 52);   // ceil(c_i / 2^52)
    }
    _Pragma("unroll") for (int k = 5; k < 9; k++) {
        r[k - 5] = c[k] & kM52;
        c[k + 1] += (uint64_t)((int64_t)c[k] >> 52);
    }
    r[4] = c[9];
}

// 16 p^2 (Fq) in radix 2^52: keeps a0 b0 - a1 b1 non-negative below
__host__ __device__ constexpr uint64_t fq_16p2_52(int k)
{
    return k == 0 ? 0x58a2275d69b10ull : k == 1 ? 0xd09eac1013b54ull : k == 2 ? 0x96cadca602072ull
         : k == 3 ? 0x2c84a50189c6dull : k == 4 ? 0x4689e957a124ull : k == 5 ? 0xdfa5c34c6b38dull
         : k == 6 ? 0x511637560626eull : k == 7 ? 0x348d21cb00b85ull : k == 8 ? 0xbf9c599a6f7c0ull : 0x925c4b8763cull;
}

// a + b of two 8-limb integers below 2^255 (no reduction)
__device__ __forceinline__ void add_nored(uint32_t s[8], const uint32_t a[8], const uint32_t b[8])
{
    uint32_t c = 0;
    _Pragma("unroll") for (int k = 0; k < 8; k++) {
        uint64_t x = (uint64_t)a[k] + b[k] + c;
        s[k] = (uint32_t)x;
        c = (uint32_t)(x >> 32);
    }
}

// Fq2 product (i^2 = -1) by Karatsuba with lazy reduction, on the FP64 pipe:
// with one operand scaled by 16 as in mul52,
//   c0 = 16 (a0 b0 - a1 b1) + 16 p^2  in (0, 32 p^2),
//   c1 = 16 (a0 + a1)(b0 + b1) - 16 a0 b0 - 16 a1 b1 = 16 (a0 b1 + a1 b0) in [0, 32 p^2),
// three 5x5-limb products and two reductions (each result < 2p, then one
// conditional subtraction): the canonical values of the schoolbook product.
__device__ __forceinline__ void fq2_mul52(uint32_t c0[8], uint32_t c1[8], const uint32_t a0[8], const uint32_t a1[8],
                                          const uint32_t b0[8], const uint32_t b1[8])
{
    uint64_t x[10], y[10];
    {
        double da0[5], da1[5], db0[5], db1[5];
        to_d52<4>(da0, a0);
        to_d52<4>(da1, a1);
        to_d52<0>(db0, b0);
        to_d52<0>(db1, b1);
        _Pragma("unroll") for (int k = 0; k < 10; k++) { x[k] = 0; y[k] = 0; }
        prod_cols52(x, da0, db0);
        prod_cols52(y, da1, db1);
    }
    // x = a0 b0 + bias, y = a1 b1 + bias (per column)
    uint64_t r0[10], r1[10];
    _Pragma("unroll") for (int k = 0; k < 10; k++) {
        r0[k] = x[k] - y[k] + fq_16p2_52(k);
        r1[k] = prod_bias52(k) - x[k] - y[k];
    }
    {
        uint32_t sa[8], sb[8];
        add_nored(sa, a0, a1);
        add_nored(sb, b0, b1);
        double ds[5], dt[5];
        to_d52<4>(ds, sa);
        to_d52<0>(dt, sb);
        prod_cols52(r1, ds, dt);
    }
    uint64_t q0[5], q1[5];
    redc52<FqP>(q0, r0);
    redc52<FqP>(q1, r1);
    uint32_t t[8];
    from_limbs52(t, q0);
    Fq f0 = final_sub<FqP>(t);
    from_limbs52(t, q1);
    Fq f1 = final_sub<FqP>(t);
    _Pragma("unroll") for (int k = 0; k < 8; k++) { c0[k] = f0.v[k]; c1[k] = f1.v[k]; }
}

// Montgomery square r = a^2 / 2^260 mod p (r < 2p) for limbs a < 2^52 with
// a^2 < p * 2^260: 15 limb products instead of 25, the cross products'
// halves added twice.
__host__ __device__ constexpr uint64_t sq_bias52(int k)
{
    uint64_t b = 0;
    for (int i = 0; i < 5; i++) {
        if (2 * i == k) b += kLoBias;
        if (2 * i + 1 == k) b += kHiBias;
        for (int j = i + 1; j < 5; j++) {
            if (i + j == k) b += 2 * kLoBias;
            if (i + j + 1 == k) b += 2 * kHiBias;
        }
    }
    return b;
}
template <class P>
__device__ __forceinline__ void mont52_sqr_core(uint64_t r[5], const double a[5])
{
    uint64_t c[10];
    _Pragma("unroll") for (int k = 0; k < 10; k++) c[k] = 0 - sq_bias52(k) - red_bias52(k);
    _Pragma("unroll") for (int i = 0; i < 5; i++) {
        uint64_t hi, lo;
        split52(a[i], a[i], hi, lo);
        c[2 * i] += lo;
        c[2 * i + 1] += hi;
        _Pragma("unroll") for (int j = i + 1; j < 5; j++) {
            split52(a[i], a[j], hi, lo);
            c[i + j] = c[i + j] + lo + lo;
            c[i + j + 1] = c[i + j + 1] + hi + hi;
        }
    }
    _Pragma("unroll") for (int i = 0; i < 5; i++) {
        const double m = u52_to_d((c[i] * P52<P>::ninv) & kM52);
        c[i + 1] += split52_hi(m, (double)P52<P>::p(0));
        _Pragma("unroll") for (int j = 1; j < 5; j++) {
            uint64_t hi, lo;
            split52(m, (double)P52<P>::p(j), hi, lo);
            c[i + j] += lo;
            c[i + j + 1] += hi;
        }
        c[i + 1] += (c[i] + kM52) >> 52;
    }
    _Pragma("unroll") for (int k = 5; k < 9; k++) {
        r[k - 5] = c[k] & kM52;
        c[k + 1] += c[k] >> 52;
    }
    r[4] = c[9];
}

// Drop-in for mul(): canonical 8x32-bit Montgomery operands (R = 2^256),
// canonical result, the same bits.
template <class P>
__device__ __forceinline__ Fp<P> mul52(const Fp<P>& a, const Fp<P>& b)
{
    double da[5], db[5];
    to_d52<4>(da, a.v);
    to_d52<0>(db, b.v);
    uint64_t r[5];
    mont52_core<P>(r, da, db);
    uint32_t t[8];
    from_limbs52(t, r);
    return final_sub<P>(t);
}

// a * b / 2^256 mod p (canonical) with b given already as radix-2^52
// doubles (to_d52<0>, as a twiddle table stores it), for any 8-limb a with
// 16 a b < 85 p^2 (a below 2p with b < p qualifies): the drop-in product
// without b's conversion.
template <class P>
__device__ __forceinline__ Fp<P> mul52_pre(const Fp<P>& a, const double db[5])
{
    double da[5];
    to_d52<4>(da, a.v);
    uint64_t r[5];
    mont52_core<P>(r, da, db);
    uint32_t t[8];
    from_limbs52(t, r);
    return final_sub<P>(t);
}

// a + p - b for canonical a, b: in (0, 2p), not reduced (a product operand)
template <class P>
__device__ __forceinline__ Fp<P> sub_plus_p(const Fp<P>& a, const Fp<P>& b)
{
    Fp<P> r;
    uint64_t c = 0, d = 0;
    _Pragma("unroll") for (int i = 0; i < 8; i++) {
        uint64_t x = (uint64_t)a.v[i] + P::p(i) + c;
        c = x >> 32;
        uint64_t y = (uint64_t)(uint32_t)x - b.v[i] - d;
        d = y >> 63;
        r.v[i] = (uint32_t)y;
    }
    return r;
}

// Square with the drop-in interface: the operand enters as 4a, so
// (4a)^2 / 2^260 = a^2 / 2^256, from 15 limb products instead of 25.
template <class P>
__device__ __forceinline__ Fp<P> sqr52(const Fp<P>& a)
{
    double da[5];
    to_d52<2>(da, a.v);
    uint64_t r[5];
    mont52_sqr_core<P>(r, da);
    uint32_t t[8];
    from_limbs52(t, r);
    return final_sub<P>(t);
}

// Out-of-line bodies for the curve formulas (one product, two independent
// products interleaved, or two squares), as mul_call / mul2_call in
// field.cuh.
template <class P> __device__ __noinline__ Fp<P> mul52_call(const Fp<P> a, const Fp<P> b) { return mul52(a, b); }
template <class P>
__device__ __noinline__ FpPair<P> mul52x2_call(const Fp<P> a0, const Fp<P> b0, const Fp<P> a1, const Fp<P> b1)
{
    return FpPair<P>{mul52(a0, b0), mul52(a1, b1)};
}
template <class P>
__device__ __noinline__ FpPair<P> sqr52x2_call(const Fp<P> a, const Fp<P> b)
{
    return FpPair<P>{sqr52(a), sqr52(b)};
}

}  // namespace lzk
