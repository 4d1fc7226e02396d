// fieldops.cu -- element-wise field arithmetic on the device.
//
// The device counterpart of the reference's mont_t operators (operator*,
// sqr, +=, -=, cneg, reciprocal, from/to; include/device-arith/field/
// mont_t.cuh:396-430, 208-302, 465-629) and of fp2_t (alt_bn128_t.cuh:
// 97-224), applied to arrays.  Each operation runs through the same device
// routines the operators use: Fq and Fq2 products and squares through the
// out-of-line bodies of the curve formulas (mul52_call, fq2_mul_call with its
// lazily reduced Karatsuba product, fq2_sqr_call) and the square of their
// square pairs (sqr52), Fr products through the product of the NTT
// butterflies (mul52), all of them on the FP64 pipe (field52.cuh), additions
// and subtractions through the same carry chains.  Results are canonical
// (< p).
#include "common.cuh"
#include "curve.cuh"

namespace lzk {

template <class F>
__device__ __forceinline__ F fop_mul(const F& a, const F& b) { return mul52(a, b); }
template <>
__device__ __forceinline__ Fq fop_mul<Fq>(const Fq& a, const Fq& b) { return cmul(a, b); }
template <>
__device__ __forceinline__ Fq2 fop_mul<Fq2>(const Fq2& a, const Fq2& b) { return cmul(a, b); }

template <class F>
__device__ __forceinline__ F fop_sqr(const F& a) { return sqr52(a); }
template <>
__device__ __forceinline__ Fq2 fop_sqr<Fq2>(const Fq2& a) { return csqr(a); }

template <class P> __device__ __forceinline__ Fp<P> fop_from(const Fp<P>& a) { return from_mont(a); }
template <class P> __device__ __forceinline__ Fp<P> fop_to(const Fp<P>& a) { return to_mont(a); }
__device__ __forceinline__ Fq2 fop_from(const Fq2& a) { return {from_mont(a.c0), from_mont(a.c1)}; }
__device__ __forceinline__ Fq2 fop_to(const Fq2& a) { return {to_mont(a.c0), to_mont(a.c1)}; }

template <class F>
__global__ void k_field_op(int op, const F* __restrict__ a, const F* __restrict__ b, F* __restrict__ out, size_t n)
{
    for (uint64_t i = gtid(); i < n; i += gstride()) {
        F x = ld_elem(a + i), r;
        switch (op) {
            case LZK_FOP_ADD: r = add(x, ld_elem(b + i)); break;
            case LZK_FOP_SUB: r = sub(x, ld_elem(b + i)); break;
            case LZK_FOP_MUL: r = fop_mul(x, ld_elem(b + i)); break;
            case LZK_FOP_SQR: r = fop_sqr(x); break;
            case LZK_FOP_NEG: r = neg(x); break;
            case LZK_FOP_INV: r = inverse(x); break;
            case LZK_FOP_FROM_MONT: r = fop_from(x); break;
            default: r = fop_to(x); break;
        }
        st_elem(out + i, r);
    }
}

template <class F>
static int launch_field_op(int op, const void* a, const void* b, void* out, size_t n, cudaStream_t st)
{
    k_field_op<F><<<grid_for(n, 128, sm_count() * 16), 128, 0, st>>>(op, static_cast<const F*>(a),
                                                                       static_cast<const F*>(b), static_cast<F*>(out), n);
    note_launch();
    return launch_status();
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_field_op(int field, int op, const void* a, const void* b, void* out, size_t n, void* stream)
{
    if (op < LZK_FOP_ADD || op > LZK_FOP_TO_MONT) return LZK_EINVAL;
    if (n == 0) return LZK_OK;
    bool binary = op == LZK_FOP_ADD || op == LZK_FOP_SUB || op == LZK_FOP_MUL;
    if (!a || !out || (binary && !b)) return LZK_EINVAL;
    cudaStream_t st = as_stream(stream);
    switch (field) {
        case LZK_FIELD_FR: return launch_field_op<Fr>(op, a, b, out, n, st);
        case LZK_FIELD_FQ: return launch_field_op<Fq>(op, a, b, out, n, st);
        case LZK_FIELD_FQ2: return launch_field_op<Fq2>(op, a, b, out, n, st);
        default: return LZK_EINVAL;
    }
}

}  // extern "C"
