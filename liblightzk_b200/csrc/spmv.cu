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
#include "r1cs.cuh"

namespace lzk {

__global__ void __launch_bounds__(256) k_spmv3(CsrDev m0, CsrDev m1, CsrDev m2, const Fr* __restrict__ z,
                                                Fr* __restrict__ o0, Fr* __restrict__ o1, Fr* __restrict__ o2)
{
    const CsrDev& M = blockIdx.y == 0 ? m0 : (blockIdx.y == 1 ? m1 : m2);
    Fr* out = blockIdx.y == 0 ? o0 : (blockIdx.y == 1 ? o1 : o2);
    if (!out) return;
    for (uint64_t i = gtid(); i < M.rows; i += gstride()) st_elem(out + i, row_dot(M, i, z));
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
    LZK_TRY(csr_to_dev(A, a));
    LZK_TRY(csr_to_dev(B, b));
    LZK_TRY(csr_to_dev(C, c));
    uint64_t rows = a.rows > b.rows ? a.rows : b.rows;
    rows = rows > c.rows ? rows : c.rows;
    if (rows == 0) return LZK_OK;
    k_spmv3<<<dim3(grid_for(rows, 256, sm_count() * 8), 3), 256, 0, as_stream(stream)>>>(
        a, b, c, reinterpret_cast<const Fr*>(z), A ? reinterpret_cast<Fr*>(Az) : nullptr,
        B ? reinterpret_cast<Fr*>(Bz) : nullptr, C ? reinterpret_cast<Fr*>(Cz) : nullptr); note_launch();
    return launch_status();
}

int lzk_spmv(const lzk_csr* M, const lzk_fr_t* z, lzk_fr_t* out, void* stream)
{
    if (!M) return LZK_EINVAL;
    return lzk_spmv3(M, nullptr, nullptr, z, out, nullptr, nullptr, stream);
}

}  // extern "C"
