/* lzk_compat.hpp -- LibLightZK's operator names and signatures on top of
 * the C ABI in lzk.h, so the reference's call sites keep compiling:
 *
 *   multi_scalar_multiplication_g1/_g2   include/operator/msm.cuh:210-247
 *   number_theory_transformation        include/operator/poly.cuh:65-73
 *   batch_sparse_matrix_vector_multiplication  poly.cuh:5-30 (a kernel
 *       there, launched <<<216,1024>>>; here a host function with the same
 *       arguments -- drop the launch configuration at the call site)
 *   polynomial_A_times_B_minus_C        poly.cuh:75-85 (likewise)
 *   Groth16_BN254 (Setup, Prove) and input_scale   protocol/groth16.cuh:11-222
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
#include <cstdint>
#include <cstdio>
#include <vector>
#include <cuda_runtime.h>
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

/* ---------------------------------------------------------------------
 * Groth16<...> (protocol/groth16.cuh:18-222) as test/groth16.cu uses it:
 *
 *     Groth16_BN254 protocol(input_scale::MatMul_p_100);
 *     protocol.Setup(12);
 *     protocol.Prove();
 *
 * Setup builds the MatMul circuit of the input scale (the product of two
 * p x p matrices, xpu-spmat.cuh:33-65: p = 39 / 63 / 100 give 2^16 / 2^18 /
 * 2^20 constraints) in the reference's CSR layout (8-byte indices, `rows`
 * offsets), a proving key of seeded Fr multiples of the generators
 * (lzk_random_fr and the fixed-base kernels, where the reference draws
 * unseeded host randomness, groth16.cuh:88-126), a witness whose gates are
 * solved (the reference's is random, groth16.cuh:128-132), and the prover
 * with shifted-copy tables of window win_siz.  Prove makes one proof (r and
 * s seeded) and prints it as the reference does, affine coordinates in hex
 * (groth16.cuh:219-221).  mode LZK_PROVE_REFERENCE (the default) follows the
 * reference's H chain.  Seeds: key `seed` (stream ids 16..22), witness
 * `seed + 100` (stream id 4), r and s `seed + 200` (stream id 99) -- the
 * liblightzk_b200.synth generators with the same seeds build the same
 * instance.  Errors print the library status, as the shims above do. */
enum class input_scale { MatMul_p_39, MatMul_p_63, MatMul_p_100 };

class Groth16_BN254 {
public:
    explicit Groth16_BN254(input_scale is, uint64_t seed = 1, int mode = LZK_PROVE_REFERENCE)
        : seed_(seed), mode_(mode)
    {
        p_ = is == input_scale::MatMul_p_39 ? 39 : is == input_scale::MatMul_p_63 ? 63 : 100;
        size_t p2 = p_ * p_, p3 = p2 * p_;
        M_ = 1;
        while (M_ < p3 + p2) M_ <<= 1;
        k_ = 3 * p2;
        n_vars_ = 1 + 3 * p2 + p3;
    }
    Groth16_BN254(const Groth16_BN254&) = delete;
    Groth16_BN254& operator=(const Groth16_BN254&) = delete;
    ~Groth16_BN254()
    {
        if (prover_) lzk_prover_destroy(prover_);
        for (void* d : dev_) cudaFree(d);
    }

    void Setup(size_t win_siz)
    {
        const size_t p2 = p_ * p_, p3 = p2 * p_;
        // the MatMul rows: products t_i = X[i2][i1] * Y[i1][i3], then sums
        std::vector<uint64_t> ac, ar, bc, br, cc, cr;
        for (size_t i = 0; i < p3; i++) {
            size_t i1 = i / p2, i2 = (i % p2) / p_, i3 = i % p_;
            ar.push_back(ac.size()); ac.push_back(1 + i2 * p_ + i1);
            br.push_back(bc.size()); bc.push_back(1 + p2 + i1 * p_ + i3);
            cr.push_back(cc.size()); cc.push_back(1 + 3 * p2 + i);
        }
        for (size_t r = 0; r < p2; r++) {
            ar.push_back(ac.size());
            for (size_t k = 0; k < p_; k++) ac.push_back(1 + 3 * p2 + k * p2 + r);
            br.push_back(bc.size()); bc.push_back(0);
            cr.push_back(cc.size()); cc.push_back(1 + 2 * p2 + r);
        }
        while (ar.size() < M_) { ar.push_back(ac.size()); br.push_back(bc.size()); cr.push_back(cc.size()); }
        const uint64_t one[4] = {0xAC96341C4FFFFFFBull, 0x36FC76959F60CD29ull, 0x666EA36F7879462Eull,
                                 0x0E0A77C19A07DF2Full};   // Fr one, Montgomery
        size_t nv = ac.size();                              // the largest matrix
        std::vector<uint64_t> ones(4 * nv);
        for (size_t i = 0; i < nv; i++) for (int w = 0; w < 4; w++) ones[4 * i + w] = one[w];
        lzk_fr_t* val = upload<lzk_fr_t>(ones.data(), nv * 32);
        lzk_csr* mats[3] = {&circuit_.A, &circuit_.B, &circuit_.C};
        std::vector<uint64_t>* cols[3] = {&ac, &bc, &cc};
        std::vector<uint64_t>* rows[3] = {&ar, &br, &cr};
        for (int m = 0; m < 3; m++) {
            lzk_csr& c = *mats[m];
            c.val = val;
            c.col_idx = upload<void>(cols[m]->data(), cols[m]->size() * 8);
            c.row_ptr = upload<void>(rows[m]->data(), rows[m]->size() * 8);
            c.rows = M_;
            c.cols = n_vars_;
            c.nnz = cols[m]->size();
            c.index_bytes = 8;
        }
        circuit_.n_vars = n_vars_;
        circuit_.n_public = k_;
        circuit_.log_domain = 0;
        while ((size_t(1) << circuit_.log_domain) < M_) circuit_.log_domain++;

        // proving key
        size_t nl = n_vars_ - k_ - 1, mx = n_vars_ > M_ ? n_vars_ : M_;
        lzk_fr_t* ks = alloc<lzk_fr_t>(mx * 32);
        auto g1q = [&](uint64_t sid, size_t n) {
            lzk_g1_affine_t* q = alloc<lzk_g1_affine_t>(n * sizeof(lzk_g1_affine_t));
            report(lzk_random_fr(seed_, sid, 0, n, ks, nullptr), "Setup: lzk_random_fr");
            report(lzk_g1_fixed_base(ks, n, q, nullptr), "Setup: lzk_g1_fixed_base");
            return q;
        };
        auto g2q = [&](uint64_t sid, size_t n) {
            lzk_g2_affine_t* q = alloc<lzk_g2_affine_t>(n * sizeof(lzk_g2_affine_t));
            report(lzk_random_fr(seed_, sid, 0, n, ks, nullptr), "Setup: lzk_random_fr");
            report(lzk_g2_fixed_base(ks, n, q, nullptr), "Setup: lzk_g2_fixed_base");
            return q;
        };
        pk_.a_query = g1q(16, n_vars_);
        pk_.b1_query = g1q(17, n_vars_);
        pk_.b2_query = g2q(18, n_vars_);
        pk_.l_query = g1q(19, nl ? nl : 1);
        pk_.h_query = g1q(20, M_ - 1);
        lzk_g1_affine_t* c1 = g1q(21, 3);
        lzk_g2_affine_t* c2 = g2q(22, 2);
        lzk_g1_affine_t h1[3];
        lzk_g2_affine_t h2[2];
        cudaMemcpy(h1, c1, sizeof(h1), cudaMemcpyDeviceToHost);
        cudaMemcpy(h2, c2, sizeof(h2), cudaMemcpyDeviceToHost);
        pk_.alpha1 = h1[0]; pk_.beta1 = h1[1]; pk_.delta1 = h1[2];
        pk_.beta2 = h2[0]; pk_.delta2 = h2[1];

        // witness: z_0 = 1, X and Y seeded, products and sums solved
        z_ = alloc<lzk_fr_t>(n_vars_ * 32);
        cudaMemcpy(z_, one, 32, cudaMemcpyHostToDevice);
        report(lzk_random_fr(seed_ + 100, 4, 0, 2 * p2, z_ + 1, nullptr), "Setup: witness");
        report(lzk_r1cs_solve(&circuit_.A, &circuit_.B, &circuit_.C, z_, 0, p3, nullptr), "Setup: lzk_r1cs_solve");
        report(lzk_r1cs_solve(&circuit_.A, &circuit_.B, &circuit_.C, z_, p3, p3 + p2, nullptr),
               "Setup: lzk_r1cs_solve");
        report(lzk_prover_create(&circuit_, &pk_, mode_, (uint32_t)win_siz, &prover_), "Setup: lzk_prover_create");
        proof_ = alloc<lzk_groth16_proof>(sizeof(lzk_groth16_proof));
        wire_dev_ = alloc<uint32_t>(LZK_PROOF_WIRE_BYTES);
        rs_ = alloc<lzk_fr_t>(64);
        cudaDeviceSynchronize();
    }

    void Prove()
    {
        if (!prover_) { std::fprintf(stderr, "Prove: Setup did not complete\n"); return; }
        lzk_fr_t rs[2];
        report(lzk_random_fr(seed_ + 200, 99, proofs_ * 2, 2, rs_, nullptr), "Prove: lzk_random_fr");
        cudaMemcpy(rs, rs_, sizeof(rs), cudaMemcpyDeviceToHost);
        report(lzk_groth16_prove(prover_, z_, &rs[0], &rs[1], proof_, nullptr), "Prove: lzk_groth16_prove");
        report(lzk_groth16_proof_to_wire(proof_, wire_dev_, nullptr), "Prove: lzk_groth16_proof_to_wire");
        wire_.assign(LZK_PROOF_WIRE_BYTES / 4, 0u);
        cudaMemcpy(wire_.data(), wire_dev_, LZK_PROOF_WIRE_BYTES, cudaMemcpyDeviceToHost);
        proofs_++;
        // A, C over Fq; B over Fq2 (c0, c1 of x, then of y), as print() shows them
        print_coords("x/y:", 0, 2);
        print_coords("x/y:", 48, 2);
        std::printf("x/y:\n");
        print_coords("c0/c1:", 16, 2);
        print_coords("c0/c1:", 32, 2);
    }

    // the last proof in the 256-byte wire form (lzk_groth16_proof_to_wire)
    const std::vector<uint32_t>& wire() const { return wire_; }

private:
    template <class T> T* alloc(size_t bytes)
    {
        void* d = nullptr;
        if (cudaMalloc(&d, bytes ? bytes : 16) != cudaSuccess) { std::fprintf(stderr, "Groth16_BN254: out of device memory\n"); return nullptr; }
        dev_.push_back(d);
        return static_cast<T*>(d);
    }
    template <class T> T* upload(const void* h, size_t bytes)
    {
        T* d = alloc<T>(bytes);
        if (d) cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice);
        return d;
    }
    // `count` 256-bit numbers from word `w0` of the wire form, most significant digit first
    void print_coords(const char* label, size_t w0, int count) const
    {
        std::printf("%s\n", label);
        for (int c = 0; c < count; c++) {
            for (int i = 7; i >= 0; i--) std::printf("%08x", wire_[w0 + 8 * c + i]);
            std::printf("\n");
        }
    }

    size_t p_ = 0, M_ = 0, k_ = 0, n_vars_ = 0;
    uint64_t seed_ = 1, proofs_ = 0;
    int mode_ = LZK_PROVE_REFERENCE;
    lzk_groth16_circuit circuit_{};
    lzk_groth16_pk pk_{};
    lzk_prover* prover_ = nullptr;
    lzk_fr_t *z_ = nullptr, *rs_ = nullptr;
    lzk_groth16_proof* proof_ = nullptr;
    uint32_t* wire_dev_ = nullptr;
    std::vector<uint32_t> wire_;
    std::vector<void*> dev_;
};

}  // namespace lzk_compat

#endif /* LZK_COMPAT_HPP */
