// ntt.cuh -- internal interface of the NTT (ntt.cu) for other operators.
#pragma once
#include "common.cuh"
#include "field.cuh"

namespace lzk {

struct NttTables {
    Fr* tw[2] = {nullptr, nullptr};  // w^e, w^-e for e < n/2
    Fr* consts = nullptr;            // see k_ntt_consts
};

struct CosetTables {
    Fr* lo[2] = {nullptr, nullptr};  // g^j, g^-j for j < 4096
    Fr* hi[2] = {nullptr, nullptr};  // g^(4096 i), g^-(4096 i) for i < 2^(26-12)
};

// cached per-device tables for size 2^k (built synchronously on first use)
int get_tables(uint32_t k, NttTables& out, CosetTables& cos);
// count transforms of size 2^k, `bstride` apart; dir as LZK_NTT_*; a non-null
// scale_override replaces the inverse's 2^-k factor (or adds a factor to a
// forward transform)
int ntt_run(Fr* data, uint32_t k, int dir, uint32_t count, size_t bstride, const Fr* scale_override, cudaStream_t st);

}  // namespace lzk
