// The reference's test/msm-check.cu flow on the drop-in header: a
// pre_comp-layout table of Jacobian (Z = 1) records with win_cnt shifted
// copies, Montgomery scalars, multi_scalar_multiplication_g1 /
// number_theory_transformation / batch_sparse_matrix_vector_multiplication /
// polynomial_A_times_B_minus_C called with the reference's argument lists.
// Inputs and outputs are raw little-endian files in a directory given on the
// command line; tests/test_compat_gpu.py writes the inputs with the oracle
// and checks the outputs.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "lzk_compat.hpp"

struct fr_t { uint32_t v[8]; };
struct g1_t { uint32_t v[24]; };
struct g2_t { uint32_t v[24]; };   // one lane-pair half: {X.ci Y.ci Z.ci}

struct Desc {   // the members of xpu::spmat_descript (xpu-spmat.cuh:20-25)
    fr_t* val;
    size_t *col_idx, *row_ptr;
    size_t row, col, cnt;
};

static std::vector<char> slurp(const char* dir, const char* name)
{
    char path[4096];
    std::snprintf(path, sizeof path, "%s/%s", dir, name);
    FILE* f = std::fopen(path, "rb");
    if (!f) { std::fprintf(stderr, "missing %s\n", path); std::exit(2); }
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<char> b(n);
    if (n && std::fread(b.data(), 1, n, f) != (size_t)n) std::exit(2);
    std::fclose(f);
    return b;
}

static void spit(const char* dir, const char* name, const void* p, size_t n)
{
    char path[4096];
    std::snprintf(path, sizeof path, "%s/%s", dir, name);
    FILE* f = std::fopen(path, "wb");
    std::fwrite(p, 1, n, f);
    std::fclose(f);
}

template <class T>
static T* upload(const std::vector<char>& h)
{
    void* d = nullptr;
    if (cudaMalloc(&d, h.size() ? h.size() : 16) != cudaSuccess) std::exit(3);
    cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice);
    return static_cast<T*>(d);
}

int main(int argc, char** argv)
{
    if (argc < 2) return 1;
    const char* dir = argv[1];
    std::vector<char> meta = slurp(dir, "meta.bin");   // n, win_siz, win_cnt, ntt_log, spmv rows, nnz, zlen
    const uint64_t* m = reinterpret_cast<const uint64_t*>(meta.data());
    size_t n = m[0], win_siz = m[1], win_cnt = m[2], log_deg = m[3], rows = m[4], nnz = m[5];

    // MSM G1 / G2 over reference-layout tables
    fr_t* scalars = upload<fr_t>(slurp(dir, "scalars.bin"));
    g1_t* table1 = upload<g1_t>(slurp(dir, "table_g1.bin"));
    g2_t* table2 = upload<g2_t>(slurp(dir, "table_g2.bin"));
    g1_t* dest1;
    cudaMalloc(&dest1, sizeof(g1_t));
    g2_t* dest2;
    cudaMalloc(&dest2, 2 * sizeof(g2_t));
    lzk_compat::multi_scalar_multiplication_g1<fr_t, g1_t>(n, scalars, table1, dest1, win_siz, win_cnt,
                                                           size_t(1) << win_siz, n);
    lzk_compat::multi_scalar_multiplication_g2<fr_t, g2_t>(n, scalars, table2, dest2, win_siz, win_cnt,
                                                           size_t(1) << win_siz, n);

    // NTT with the caller's ntt_setup table: iNTT_M with factor M^-1
    size_t M = size_t(1) << log_deg;
    fr_t* params = upload<fr_t>(slurp(dir, "ntt_params.bin"));
    fr_t* coeffs = upload<fr_t>(slurp(dir, "ntt_in.bin"));
    lzk_compat::number_theory_transformation<fr_t>(M, log_deg, coeffs, params + M, params + 2 * M);

    // SpMV with size_t descriptors, then A*B - C
    fr_t* z = upload<fr_t>(slurp(dir, "z.bin"));
    Desc d[3];
    const char* names[3][3] = {{"a_val.bin", "a_col.bin", "a_rp.bin"}, {"b_val.bin", "b_col.bin", "b_rp.bin"},
                               {"c_val.bin", "c_col.bin", "c_rp.bin"}};
    for (int q = 0; q < 3; q++) {
        d[q].val = upload<fr_t>(slurp(dir, names[q][0]));
        d[q].col_idx = upload<size_t>(slurp(dir, names[q][1]));
        d[q].row_ptr = upload<size_t>(slurp(dir, names[q][2]));
        d[q].row = rows;
        d[q].col = 0;
        d[q].cnt = slurp(dir, names[q][0]).size() / sizeof(fr_t);
    }
    (void)nnz;
    fr_t *Az, *Bz, *Cz;
    cudaMalloc(&Az, rows * sizeof(fr_t));
    cudaMalloc(&Bz, rows * sizeof(fr_t));
    cudaMalloc(&Cz, rows * sizeof(fr_t));
    lzk_compat::batch_sparse_matrix_vector_multiplication(d[0], d[1], d[2], z, Az, Bz, Cz);
    lzk_compat::polynomial_A_times_B_minus_C<fr_t>(rows, Az, Bz, Cz);

    if (cudaDeviceSynchronize() != cudaSuccess) { std::fprintf(stderr, "CUDA error\n"); return 4; }
    std::vector<char> h1(sizeof(g1_t)), h2(2 * sizeof(g2_t)), hn(M * sizeof(fr_t)), ha(rows * sizeof(fr_t));
    cudaMemcpy(h1.data(), dest1, h1.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(h2.data(), dest2, h2.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(hn.data(), coeffs, hn.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(ha.data(), Az, ha.size(), cudaMemcpyDeviceToHost);
    spit(dir, "out_g1.bin", h1.data(), h1.size());
    spit(dir, "out_g2.bin", h2.data(), h2.size());
    spit(dir, "out_ntt.bin", hn.data(), hn.size());
    spit(dir, "out_abc.bin", ha.data(), ha.size());
    std::printf("compat ok\n");
    return 0;
}
