// field.cuh -- 254-bit prime-field arithmetic for BN254 on sm_100a.
//
// An element is 8 little-endian 32-bit limbs in Montgomery form with
// R = 2^256: exactly the bytes of the reference's host bigint<4> Montgomery
// representation (include/host-arith/field/fp.cuh:33) and of its device
// mont_t<254,...> (include/device-arith/field/mont_t.cuh:47), so host arrays
// cross the C-ABI unchanged.
//
// Multiplication is coarsely-integrated operand scanning over 32-bit limbs
// (mont_mul_core); the result ends below 2p and one conditional subtraction
// makes every result canonical (< p), which keeps equality and zero tests
// exact.  Conversion out of Montgomery form uses explicit mad.lo / mad.hi
// carry chains (red_row).
#pragma once
#include <cstdint>

namespace lzk {

// Fq: p = 0x30644e72e131a029b85045b68181585d97816a916871ca8d3c208c16d87cfd47
struct FqP {
    static constexpr uint32_t INV = 0xe4866389u;  // -p^-1 mod 2^32
    __host__ __device__ static constexpr uint32_t p(int i) {
        return i == 0 ? 0xd87cfd47u : i == 1 ? 0x3c208c16u : i == 2 ? 0x6871ca8du : i == 3 ? 0x97816a91u
             : i == 4 ? 0x8181585du : i == 5 ? 0xb85045b6u : i == 6 ? 0xe131a029u : 0x30644e72u;
    }
    // R mod p (Montgomery one)
    __host__ __device__ static constexpr uint32_t one(int i) {
        return i == 0 ? 0xc58f0d9du : i == 1 ? 0xd35d438du : i == 2 ? 0xf5c70b3du : i == 3 ? 0x0a78eb28u
             : i == 4 ? 0x7879462cu : i == 5 ? 0x666ea36fu : i == 6 ? 0x9a07df2fu : 0x0e0a77c1u;
    }
    // R^2 mod p
    __host__ __device__ static constexpr uint32_t r2(int i) {
        return i == 0 ? 0x538afa89u : i == 1 ? 0xf32cfc5bu : i == 2 ? 0xd44501fbu : i == 3 ? 0xb5e71911u
             : i == 4 ? 0x0a417ff6u : i == 5 ? 0x47ab1effu : i == 6 ? 0xcab8351fu : 0x06d89f71u;
    }
};

// Fr: r = 0x30644e72e131a029b85045b68181585d2833e84879b9709143e1f593f0000001
struct FrP {
    static constexpr uint32_t INV = 0xefffffffu;
    __host__ __device__ static constexpr uint32_t p(int i) {
        return i == 0 ? 0xf0000001u : i == 1 ? 0x43e1f593u : i == 2 ? 0x79b97091u : i == 3 ? 0x2833e848u
             : i == 4 ? 0x8181585du : i == 5 ? 0xb85045b6u : i == 6 ? 0xe131a029u : 0x30644e72u;
    }
    __host__ __device__ static constexpr uint32_t one(int i) {
        return i == 0 ? 0x4ffffffbu : i == 1 ? 0xac96341cu : i == 2 ? 0x9f60cd29u : i == 3 ? 0x36fc7695u
             : i == 4 ? 0x7879462eu : i == 5 ? 0x666ea36fu : i == 6 ? 0x9a07df2fu : 0x0e0a77c1u;
    }
    __host__ __device__ static constexpr uint32_t r2(int i) {
        return i == 0 ? 0xae216da7u : i == 1 ? 0x1bb8e645u : i == 2 ? 0xe35c59e3u : i == 3 ? 0x53fe3ab1u
             : i == 4 ? 0x53bb8085u : i == 5 ? 0x8c49833du : i == 6 ? 0x7f4e44a5u : 0x0216d0b1u;
    }
};

template <class P>
struct Fp {
    uint32_t v[8];

    __device__ __forceinline__ static Fp zero() { Fp r; _Pragma("unroll") for (int i = 0; i < 8; i++) r.v[i] = 0; return r; }
    __device__ __forceinline__ static Fp one() { Fp r; _Pragma("unroll") for (int i = 0; i < 8; i++) r.v[i] = P::one(i); return r; }
    __device__ __forceinline__ bool is_zero() const {
        uint32_t x = v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7];
        return x == 0;
    }
    __device__ __forceinline__ bool operator==(const Fp& o) const {
        uint32_t x = 0;
        _Pragma("unroll") for (int i = 0; i < 8; i++) x |= v[i] ^ o.v[i];
        return x == 0;
    }
    __device__ __forceinline__ bool operator!=(const Fp& o) const { return !(*this == o); }
};

// r = a + b mod p  (a, b < p)
template <class P>
__device__ __forceinline__ Fp<P> add(const Fp<P>& a, const Fp<P>& b)
{
    uint32_t t[8], s[8], br;
    asm("add.cc.u32  %0, %8,  %16;\n\t"
        "addc.cc.u32 %1, %9,  %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32    %7, %15, %23;"
        : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    asm("sub.cc.u32  %0, %9,  %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7]), "=r"(br)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
          "n"(P::p(0)), "n"(P::p(1)), "n"(P::p(2)), "n"(P::p(3)), "n"(P::p(4)), "n"(P::p(5)), "n"(P::p(6)), "n"(P::p(7)));
    Fp<P> r;
    _Pragma("unroll") for (int i = 0; i < 8; i++) r.v[i] = br ? t[i] : s[i];
    return r;
}

// r = a - b mod p
template <class P>
__device__ __forceinline__ Fp<P> sub(const Fp<P>& a, const Fp<P>& b)
{
    uint32_t t[8], br;
    asm("sub.cc.u32  %0, %9,  %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7]), "=r"(br)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    // br = 0xffffffff on borrow: add p back
    Fp<P> r;
    asm("add.cc.u32  %0, %8,  %16;\n\t"
        "addc.cc.u32 %1, %9,  %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32    %7, %15, %23;"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]), "=r"(r.v[7])
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
          "r"(P::p(0) & br), "r"(P::p(1) & br), "r"(P::p(2) & br), "r"(P::p(3) & br),
          "r"(P::p(4) & br), "r"(P::p(5) & br), "r"(P::p(6) & br), "r"(P::p(7) & br));
    return r;
}

template <class P>
__device__ __forceinline__ Fp<P> neg(const Fp<P>& a)
{
    Fp<P> r = sub(Fp<P>::zero(), a);
    return r;
}

template <class P> __device__ __forceinline__ Fp<P> dbl(const Fp<P>& a) { return add(a, a); }

// One reduction row: m = t0 * INV; t += m * p; t >>= 32 (limb shift done by caller)
template <class P>
__device__ __forceinline__ void red_row(uint32_t t[9])
{
    uint32_t m = t[0] * P::INV;
    asm("mad.lo.cc.u32  %0, %9,  %10, %0;\n\t"
        "madc.lo.cc.u32 %1, %9,  %11, %1;\n\t"
        "madc.lo.cc.u32 %2, %9,  %12, %2;\n\t"
        "madc.lo.cc.u32 %3, %9,  %13, %3;\n\t"
        "madc.lo.cc.u32 %4, %9,  %14, %4;\n\t"
        "madc.lo.cc.u32 %5, %9,  %15, %5;\n\t"
        "madc.lo.cc.u32 %6, %9,  %16, %6;\n\t"
        "madc.lo.cc.u32 %7, %9,  %17, %7;\n\t"
        "addc.u32       %8, %8,  0;\n\t"
        "mad.hi.cc.u32  %1, %9,  %10, %1;\n\t"
        "madc.hi.cc.u32 %2, %9,  %11, %2;\n\t"
        "madc.hi.cc.u32 %3, %9,  %12, %3;\n\t"
        "madc.hi.cc.u32 %4, %9,  %13, %4;\n\t"
        "madc.hi.cc.u32 %5, %9,  %14, %5;\n\t"
        "madc.hi.cc.u32 %6, %9,  %15, %6;\n\t"
        "madc.hi.cc.u32 %7, %9,  %16, %7;\n\t"
        "madc.hi.u32    %8, %9,  %17, %8;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8])
        : "r"(m), "n"(P::p(0)), "n"(P::p(1)), "n"(P::p(2)), "n"(P::p(3)), "n"(P::p(4)), "n"(P::p(5)), "n"(P::p(6)), "n"(P::p(7)));
}

// t < 2p  ->  t mod p
template <class P>
__device__ __forceinline__ Fp<P> final_sub(const uint32_t t[8])
{
    uint32_t s[8], br;
    asm("sub.cc.u32  %0, %9,  %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7]), "=r"(br)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
          "n"(P::p(0)), "n"(P::p(1)), "n"(P::p(2)), "n"(P::p(3)), "n"(P::p(4)), "n"(P::p(5)), "n"(P::p(6)), "n"(P::p(7)));
    Fp<P> r;
    _Pragma("unroll") for (int i = 0; i < 8; i++) r.v[i] = br ? t[i] : s[i];
    return r;
}

// a*b + t + c as a 64-bit value (it cannot overflow: (2^32-1)^2 + 2(2^32-1)
// = 2^64 - 1).  On the device the product is a plain wide multiply and the
// two additions follow: written this way the compiler neither moves t into
// an aligned register pair for a multiply-add addend nor puts the carry
// additions on the multiplier pipe as often, which measured 7 % faster for
// Fq products and 13 % for Fq2 products than the multiply-add form.
__host__ __device__ __forceinline__ uint64_t mac64(uint32_t a, uint32_t b, uint32_t t, uint32_t c)
{
#ifdef __CUDA_ARCH__
    uint64_t p;
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(p) : "r"(a), "r"(b));
    uint64_t s = p + t;
    return s + c;
#else
    return (uint64_t)a * b + t + c;
#endif
}

// Montgomery product core, t = a*b*2^-256 (t < 2p), for a, b < p.
//
// Operand scanning with the product row and the reduction row interleaved
// limb by limb (CIOS), each step a 32x32+32+32-bit multiply-add into 64 bits
// (mac64):
//   (A, t_j)     = t_j + a_j*b_i + A
//   (C, t_{j-1}) = t_j + m*p_j + C
// Because the top limb of p is below 2^31 - 1 (both BN254 moduli start
// 0x30644e72), the accumulator never needs a ninth limb: after each row
// t_7 = A + C fits in 32 bits (the "no-carry" condition of Montgomery
// multiplication for moduli with a spare top bit).  One wide product per
// step issues fewer multiplier-pipe instructions than separate mad.lo /
// mad.hi carry chains.
template <class P>
__host__ __device__ __forceinline__ void mont_mul_core(uint32_t t[8], const uint32_t a[8], const uint32_t b[8])
{
    _Pragma("unroll") for (int i = 0; i < 8; i++) t[i] = 0;
    _Pragma("unroll") for (int i = 0; i < 8; i++) {
        uint64_t s = mac64(a[0], b[i], t[0], 0);
        uint32_t A = (uint32_t)(s >> 32);
        t[0] = (uint32_t)s;
        uint32_t m = t[0] * P::INV;
        uint64_t u = mac64(m, P::p(0), t[0], 0);
        uint32_t C = (uint32_t)(u >> 32);
        _Pragma("unroll") for (int j = 1; j < 8; j++) {
            s = mac64(a[j], b[i], t[j], A);
            A = (uint32_t)(s >> 32);
            t[j] = (uint32_t)s;
            u = mac64(m, P::p(j), t[j], C);
            C = (uint32_t)(u >> 32);
            t[j - 1] = (uint32_t)u;
        }
        t[7] = C + A;
    }
}

// Full 512-bit product t = a*b of two 8-limb integers (operand scanning,
// one 32x32+32+32-bit multiply-add into 64 bits per limb pair).
__host__ __device__ __forceinline__ void mul_wide(uint32_t t[16], const uint32_t a[8], const uint32_t b[8])
{
    _Pragma("unroll") for (int i = 0; i < 16; i++) t[i] = 0;
    _Pragma("unroll") for (int i = 0; i < 8; i++) {
        uint32_t C = 0;
        _Pragma("unroll") for (int j = 0; j < 8; j++) {
            uint64_t s = mac64(a[j], b[i], t[i + j], C);
            t[i + j] = (uint32_t)s;
            C = (uint32_t)(s >> 32);
        }
        t[i + 8] = C;
    }
}

// Montgomery reduction r = t*2^-256 (r < 2p) of a 512-bit t < p*2^256,
// row by row (separated operand scanning); the carry out of each row's top
// limb is added one limb higher in the next row.  t is consumed.
template <class P>
__host__ __device__ __forceinline__ void redc_wide(uint32_t r[8], uint32_t t[16])
{
    uint32_t top = 0;
    _Pragma("unroll") for (int i = 0; i < 8; i++) {
        uint32_t m = t[i] * P::INV;
        uint64_t s = mac64(m, P::p(0), t[i], 0);
        uint32_t C = (uint32_t)(s >> 32);
        _Pragma("unroll") for (int j = 1; j < 8; j++) {
            s = mac64(m, P::p(j), t[i + j], C);
            t[i + j] = (uint32_t)s;
            C = (uint32_t)(s >> 32);
        }
        uint64_t u = (uint64_t)t[i + 8] + C + top;
        t[i + 8] = (uint32_t)u;
        top = (uint32_t)(u >> 32);
    }
    _Pragma("unroll") for (int j = 0; j < 8; j++) r[j] = t[8 + j];
}

// Montgomery product a*b*2^-256 mod p
template <class P>
__device__ __forceinline__ Fp<P> mul(const Fp<P>& a, const Fp<P>& b)
{
    uint32_t t[8];
    mont_mul_core<P>(t, a.v, b.v);
    return final_sub<P>(t);
}

template <class P> __device__ __forceinline__ Fp<P> sqr(const Fp<P>& a) { return mul(a, a); }

// Out-of-line Montgomery product for code that chains many products (the
// curve formulas): one ~300-instruction body shared by every call keeps the
// hot loops inside the instruction cache, where fully inlined mixed
// additions (ten products each) would not fit.
template <class P> __device__ __noinline__ Fp<P> mul_call(const Fp<P> a, const Fp<P> b) { return mul(a, b); }

// Two independent products in one out-of-line body, so their carry chains
// can be interleaved (instruction-level parallelism 2 per thread).
template <class P>
struct FpPair {
    Fp<P> a, b;
};
template <class P>
__device__ __noinline__ FpPair<P> mul2_call(const Fp<P> a0, const Fp<P> b0, const Fp<P> a1, const Fp<P> b1)
{
    return FpPair<P>{mul(a0, b0), mul(a1, b1)};
}

// Montgomery -> canonical integer (multiply by 1)
template <class P>
__device__ __forceinline__ Fp<P> from_mont(const Fp<P>& a)
{
    uint32_t t[9];
    _Pragma("unroll") for (int i = 0; i < 8; i++) t[i] = a.v[i];
    t[8] = 0;
    _Pragma("unroll") for (int i = 0; i < 8; i++) {
        red_row<P>(t);
        _Pragma("unroll") for (int j = 0; j < 8; j++) t[j] = t[j + 1];
        t[8] = 0;
    }
    return final_sub<P>(t);
}

template <class P>
__device__ __forceinline__ Fp<P> to_mont(const Fp<P>& a)
{
    Fp<P> r2;
    _Pragma("unroll") for (int i = 0; i < 8; i++) r2.v[i] = P::r2(i);
    return mul(a, r2);
}

// a^(p-2) by left-to-right square-and-multiply (Fermat inverse; 0 -> 0)
template <class P>
__device__ __noinline__ Fp<P> inverse(const Fp<P>& a)
{
    Fp<P> r = Fp<P>::one();
    #pragma unroll 1
    for (int i = 7; i >= 0; i--) {
        uint32_t e = P::p(i) - (i == 0 ? 2u : 0u);
        #pragma unroll 1
        for (int b = 31; b >= 0; b--) {
            r = sqr(r);
            if ((e >> b) & 1) r = mul(r, a);
        }
    }
    return r;
}

using Fq = Fp<FqP>;
using Fr = Fp<FrP>;

}  // namespace lzk
