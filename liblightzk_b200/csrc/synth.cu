// synth.cu -- witness solving and constraint checking for R1CS instances.
//
// The synthetic circuits of the benchmark (multiplication gates
// w_i = x_a * x_b over earlier variables, rows of unit vectors plus a few
// random terms) are solved on the device: constraint i defines the variable
// named by the first entry of C's row i (coefficient one), and
//     z[def_i] = (A_i . z) * (B_i . z) - (C_i . z without that entry).
// The host lays out the rows so that a launch over rows [r0, r1) only reads
// variables defined by earlier launches.  This plays the role of the
// reference's instance generator (xpu::spmat MatMul circuits and the random
// witness of Groth16::Setup, xpu-spmat.cuh:33-65, groth16.cuh:128-132),
// except that the witness here satisfies the constraints.
#include "r1cs.cuh"

namespace lzk {

__global__ void k_r1cs_solve(CsrDev A, CsrDev B, CsrDev C, Fr* z, uint64_t r0, uint64_t r1)
{
    for (uint64_t i = r0 + gtid(); i < r1; i += gstride()) {
        Fr a = row_dot(A, i, z), b = row_dot(B, i, z);
        uint64_t s = ld_index(C.rowp, i, C.ib);
        uint64_t e = (i + 1 < C.rows) ? ld_index(C.rowp, i + 1, C.ib) : C.nnz;
        if (s >= e) continue;
        uint64_t def = ld_index(C.col, s, C.ib);
        Fr rest = Fr::zero();
        for (uint64_t j = s + 1; j < e; j++) {
            Fr v = ldg_elem(C.val + j);
            Fr x = ldg_elem(z + ld_index(C.col, j, C.ib));
            rest = add(rest, is_mont_one(v) ? x : mul(x, v));
        }
        st_elem(z + def, sub(mul(a, b), rest));
    }
}

// bad[0] += number of rows with (A_i z)(B_i z) != C_i z
__global__ void k_r1cs_check(CsrDev A, CsrDev B, CsrDev C, const Fr* __restrict__ z, uint64_t rows,
                             unsigned long long* bad)
{
    for (uint64_t i = gtid(); i < rows; i += gstride()) {
        Fr l = mul(row_dot(A, i, z), row_dot(B, i, z));
        Fr r = row_dot(C, i, z);
        if (l != r) atomicAdd(bad, 1ull);
    }
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_r1cs_solve(const lzk_csr* A, const lzk_csr* B, const lzk_csr* C, lzk_fr_t* z, uint64_t row_begin,
                   uint64_t row_end, void* stream)
{
    if (!A || !B || !C || !z || row_end < row_begin) return LZK_EINVAL;
    CsrDev a, b, c;
    LZK_TRY(csr_to_dev(A, a));
    LZK_TRY(csr_to_dev(B, b));
    LZK_TRY(csr_to_dev(C, c));
    if (row_end > a.rows || row_end > b.rows || row_end > c.rows) return LZK_EINVAL;
    if (row_end == row_begin) return LZK_OK;
    k_r1cs_solve<<<grid_for(row_end - row_begin, 128), 128, 0, as_stream(stream)>>>(a, b, c, reinterpret_cast<Fr*>(z),
                                                                                    row_begin, row_end); note_launch();
    return launch_status();
}

int lzk_r1cs_check(const lzk_csr* A, const lzk_csr* B, const lzk_csr* C, const lzk_fr_t* z,
                   unsigned long long* bad_rows, void* stream)
{
    if (!A || !B || !C || !z || !bad_rows) return LZK_EINVAL;
    CsrDev a, b, c;
    LZK_TRY(csr_to_dev(A, a));
    LZK_TRY(csr_to_dev(B, b));
    LZK_TRY(csr_to_dev(C, c));
    uint64_t rows = a.rows < b.rows ? a.rows : b.rows;
    rows = rows < c.rows ? rows : c.rows;
    LZK_CUDA(cudaMemsetAsync(bad_rows, 0, sizeof(unsigned long long), as_stream(stream)));
    if (!rows) return LZK_OK;
    k_r1cs_check<<<grid_for(rows, 128, sm_count() * 8), 128, 0, as_stream(stream)>>>(a, b, c, reinterpret_cast<const Fr*>(z),
                                                                             rows, bad_rows); note_launch();
    return launch_status();
}

}  // extern "C"
