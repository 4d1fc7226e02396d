// spmv.cu -- R1CS evaluation: A*z, B*z, C*z over Fr for CSR matrices.
//
// Replaces batch_sparse_matrix_vector_multiplication (reference
// include/operator/poly.cuh:5-30): one launch covers all three matrices
// (blockIdx.y selects the matrix), each thread owns whole rows and
// accumulates z[col] * val in Montgomery form.  Row i covers
// [row_ptr[i], row_ptr[i+1]) and the last row ends at nnz -- the reference's
// descriptor (xpu-spmat.cuh:20-25, `row` row starts plus `cnt`); a standard
// CSR with rows+1 offsets works unchanged.  Indices may be 32- or 64-bit
// (the reference uses size_t).  Entries equal to one (Montgomery R mod r)
// skip the product: z * 1 = z exactly.
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

__global__ void __launch_bounds__(256) k_spmv3(CsrDev m0, CsrDev m1, CsrDev m2, const Fr* __restrict__ z,
                                                Fr* __restrict__ o0, Fr* __restrict__ o1, Fr* __restrict__ o2)
{
    const CsrDev& M = blockIdx.y == 0 ? m0 : (blockIdx.y == 1 ? m1 : m2);
    Fr* out = blockIdx.y == 0 ? o0 : (blockIdx.y == 1 ? o1 : o2);
    if (!out) return;
    for (uint64_t i = gtid(); i < M.rows; i += gstride()) {
        uint64_t s = ld_index(M.rowp, i, M.ib);
        uint64_t e = (i + 1 < M.rows) ? ld_index(M.rowp, i + 1, M.ib) : M.nnz;
        Fr acc = Fr::zero();
        for (uint64_t j = s; j < e; j++) {
            Fr v = ldg_elem(M.val + j);
            Fr x = ldg_elem(z + ld_index(M.col, j, M.ib));
            acc = add(acc, is_mont_one(v) ? x : mul(x, v));
        }
        st_elem(out + i, acc);
    }
}

static int to_dev(const lzk_csr* c, CsrDev& d)
{
    if (!c) { d = CsrDev{nullptr, nullptr, nullptr, 0, 0, 4}; return LZK_OK; }
    if ((c->index_bytes != 4 && c->index_bytes != 8) || (c->rows && !c->row_ptr) || (c->nnz && (!c->val || !c->col_idx)))
        return LZK_EINVAL;
    d = CsrDev{reinterpret_cast<const Fr*>(c->val), c->col_idx, c->row_ptr, c->rows, c->nnz, c->index_bytes};
    return LZK_OK;
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_spmv3(const lzk_csr* A, const lzk_csr* B, const lzk_csr* C, const lzk_fr_t* z, lzk_fr_t* Az, lzk_fr_t* Bz,
              lzk_fr_t* Cz, void* stream)
{
    if (!z && ((A && A->nnz) || (B && B->nnz) || (C && C->nnz))) return LZK_EINVAL;
    if ((A && !Az) || (B && !Bz) || (C && !Cz)) return LZK_EINVAL;
    CsrDev a, b, c;
    LZK_TRY(to_dev(A, a));
    LZK_TRY(to_dev(B, b));
    LZK_TRY(to_dev(C, c));
    uint64_t rows = a.rows > b.rows ? a.rows : b.rows;
    rows = rows > c.rows ? rows : c.rows;
    if (rows == 0) return LZK_OK;
    k_spmv3<<<dim3(grid_for(rows, 256, 148 * 8), 3), 256, 0, as_stream(stream)>>>(
        a, b, c, reinterpret_cast<const Fr*>(z), A ? reinterpret_cast<Fr*>(Az) : nullptr,
        B ? reinterpret_cast<Fr*>(Bz) : nullptr, C ? reinterpret_cast<Fr*>(Cz) : nullptr);
    return launch_status();
}

int lzk_spmv(const lzk_csr* M, const lzk_fr_t* z, lzk_fr_t* out, void* stream)
{
    if (!M) return LZK_EINVAL;
    return lzk_spmv3(M, nullptr, nullptr, z, out, nullptr, nullptr, stream);
}

}  // extern "C"
