/* lzk_compat.hpp -- LibLightZK's operator names and signatures on top of
 * the C ABI in lzk.h, so the reference's call sites keep compiling:
 *
 *   multi_scalar_multiplication_g1/_g2   include/operator/msm.cuh:210-247
 *   number_theory_transformation        include/operator/poly.cuh:65-73
 *   batch_sparse_matrix_vector_multiplication  poly.cuh:5-30 (a kernel
 *       there, launched <<<216,1024>>>; here a host function with the same
 *       arguments -- drop the launch configuration at the call site)
 *   polynomial_A_times_B_minus_C        poly.cuh:75-85 (likewise)
 *
 * Argument meaning is the reference's: device pointers, scalars in
 * Montgomery form, the pre_comp_g1/_g2 table (win_cnt shifted copies,
 * level_stride apart, Jacobian records with Z = 1; G2 in the device
 * lane-pair layout), dest written as one Jacobian point (G2 in host
 * layout, as bucket_reduce_g2's write_to does).  Work goes to the legacy
 * default stream like the reference's launches.  Error behaviour matches
 * too: the reference returns nothing and prints CUDA errors
 * (device-utils.cuh:3); these shims print the library status to stderr and
 * return.  bucket_cnt is accepted and ignored: the signed-digit MSM uses
 * 2^(win_siz-1) buckets.
 */
#ifndef LZK_COMPAT_HPP
#define LZK_COMPAT_HPP

#include <cstddef>
#include <cstdio>
#include "lzk.h"

namespace lzk_compat {

inline void report(int status, const char* where)
{
    if (status != LZK_OK) std::fprintf(stderr, "%s: %s (%d)\n", where, lzk_status_string(status), status);
}

template <typename devFdT, typename dG1>
void multi_scalar_multiplication_g1(size_t length, devFdT* scalars, dG1* points, dG1* dest, size_t win_siz,
                                    size_t win_cnt, size_t bucket_cnt, size_t level_stride)
{
    (void)bucket_cnt;
    lzk_msm_cfg cfg = {};
    cfg.window_bits = (uint32_t)win_siz;
    cfg.flags = LZK_MSM_PRECOMPUTED;
    cfg.precomp_windows = (uint32_t)win_cnt;
    cfg.base_layout = LZK_BASES_REF_G1_JAC;
    cfg.level_stride = level_stride;
    report(lzk_msm_g1(reinterpret_cast<const lzk_fr_t*>(scalars), points, length, reinterpret_cast<lzk_g1_t*>(dest),
                      &cfg, nullptr),
           "multi_scalar_multiplication_g1");
}

template <typename devFdT, typename dG2>
void multi_scalar_multiplication_g2(size_t length, devFdT* scalars, dG2* points, dG2* dest, size_t win_siz,
                                    size_t win_cnt, size_t bucket_cnt, size_t level_stride)
{
    (void)bucket_cnt;
    lzk_msm_cfg cfg = {};
    cfg.window_bits = (uint32_t)win_siz;
    cfg.flags = LZK_MSM_PRECOMPUTED;
    cfg.precomp_windows = (uint32_t)win_cnt;
    cfg.base_layout = LZK_BASES_REF_G2_LANES;
    cfg.level_stride = level_stride;
    report(lzk_msm_g2(reinterpret_cast<const lzk_fr_t*>(scalars), points, length, reinterpret_cast<lzk_g2_t*>(dest),
                      &cfg, nullptr),
           "multi_scalar_multiplication_g2");
}

template <typename devFdT>
void number_theory_transformation(size_t deg, size_t log_deg, devFdT* coeffs, devFdT* omega_powers, devFdT* factor)
{
    report(lzk_number_theory_transformation(deg, log_deg, reinterpret_cast<lzk_fr_t*>(coeffs),
                                            reinterpret_cast<const lzk_fr_t*>(omega_powers),
                                            reinterpret_cast<const lzk_fr_t*>(factor), nullptr),
           "number_theory_transformation");
}

/* Desc: any descriptor with the members of xpu::spmat_descript
 * (xpu-spmat.cuh:20-25): val, col_idx, row_ptr (size_t), row, col, cnt. */
template <typename Desc>
lzk_csr to_csr(const Desc& d)
{
    lzk_csr c = {};
    c.val = reinterpret_cast<const lzk_fr_t*>(d.val);
    c.col_idx = d.col_idx;
    c.row_ptr = d.row_ptr;
    c.rows = d.row;
    c.cols = d.col;
    c.nnz = d.cnt;
    c.index_bytes = (uint32_t)sizeof(*d.col_idx);
    return c;
}

template <typename Desc, typename devFdT>
void batch_sparse_matrix_vector_multiplication(Desc A, Desc B, Desc C, devFdT* z, devFdT* Az, devFdT* Bz, devFdT* Cz)
{
    lzk_csr a = to_csr(A), b = to_csr(B), c = to_csr(C);
    report(lzk_spmv3(&a, &b, &c, reinterpret_cast<const lzk_fr_t*>(z), reinterpret_cast<lzk_fr_t*>(Az),
                     reinterpret_cast<lzk_fr_t*>(Bz), reinterpret_cast<lzk_fr_t*>(Cz), nullptr),
           "batch_sparse_matrix_vector_multiplication");
}

template <typename devFdT>
void polynomial_A_times_B_minus_C(size_t deg, devFdT* A, devFdT* B, devFdT* C)
{
    report(lzk_poly_a_times_b_minus_c(reinterpret_cast<lzk_fr_t*>(A), reinterpret_cast<const lzk_fr_t*>(B),
                                      reinterpret_cast<const lzk_fr_t*>(C), deg, nullptr),
           "polynomial_A_times_B_minus_C");
}

}  // namespace lzk_compat

#endif /* LZK_COMPAT_HPP */
