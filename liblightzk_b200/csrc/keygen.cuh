// keygen.cuh -- fixed-base comb tables shared by key generation
// (keygen.cu) and the prover's fixed-point products (groth16.cu).
#pragma once
#include "common.cuh"
#include "curve.cuh"

namespace lzk {

// T[j*256 + d] = d * 2^(8j) * P (affine, j < 32, d < 256; d = 0 unused) for
// P = *base (device), or the group generator when base is null.  Enqueued on
// st; T holds 8192 affine points.
template <class F>
int comb_build(const Aff<F>* base, Aff<F>* T, cudaStream_t st);

// k * P from P's comb table: the sum of the 32 entries selected by the bytes
// of the canonical scalar k (32 mixed additions, no doublings)
template <class F>
__device__ __forceinline__ XYZZ<F> comb_mul(const Aff<F>* __restrict__ T, const Fr& k)
{
    XYZZ<F> acc = xyzz_inf<F>();
    for (int j = 0; j < 32; j++) {
        uint32_t d = (k.v[j >> 2] >> (8 * (j & 3))) & 255u;
        if (d) acc = xyzz_madd(acc, ldg_elem(T + j * 256 + d));
    }
    return acc;
}

}  // namespace lzk
