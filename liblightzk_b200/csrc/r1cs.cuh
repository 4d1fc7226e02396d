// r1cs.cuh -- device view of a CSR matrix (lzk_csr) and the row dot
// product shared by the SpMV, the witness solver and the prover.
#pragma once
#include "common.cuh"
#include "field.cuh"

namespace lzk {

struct CsrDev {
    const Fr* val;
    const void* col;
    const void* rowp;
    uint64_t rows, nnz;
    uint32_t ib;  // index bytes
};

__device__ __forceinline__ uint64_t ld_index(const void* p, uint64_t i, uint32_t ib)
{
    return ib == 8 ? __ldg(reinterpret_cast<const unsigned long long*>(p) + i)
                   : (uint64_t)__ldg(reinterpret_cast<const unsigned int*>(p) + i);
}

__device__ __forceinline__ bool is_mont_one(const Fr& v)
{
    Fr o = Fr::one();
    return v == o;
}

// sum_j z[col_j] * val_j over row i
__device__ __forceinline__ Fr row_dot(const CsrDev& M, uint64_t i, const Fr* __restrict__ z)
{
    uint64_t s = ld_index(M.rowp, i, M.ib);
    uint64_t e = (i + 1 < M.rows) ? ld_index(M.rowp, i + 1, M.ib) : M.nnz;
    Fr acc = Fr::zero();
    for (uint64_t j = s; j < e; j++) {
        Fr v = ldg_elem(M.val + j);
        Fr x = ldg_elem(z + ld_index(M.col, j, M.ib));
        acc = add(acc, is_mont_one(v) ? x : mul(x, v));
    }
    return acc;
}

inline int csr_to_dev(const lzk_csr* c, CsrDev& d)
{
    if (!c) { d = CsrDev{nullptr, nullptr, nullptr, 0, 0, 4}; return LZK_OK; }
    if ((c->index_bytes != 4 && c->index_bytes != 8) || (c->rows && !c->row_ptr) || (c->nnz && (!c->val || !c->col_idx)))
        return LZK_EINVAL;
    d = CsrDev{reinterpret_cast<const Fr*>(c->val), c->col_idx, c->row_ptr, c->rows, c->nnz, c->index_bytes};
    return LZK_OK;
}

}  // namespace lzk
