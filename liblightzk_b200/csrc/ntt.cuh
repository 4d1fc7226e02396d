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
// count transforms of size 2^k, `bstride` apart (or at ptrs[t], a device
// table, when ptrs is non-null); dir as LZK_NTT_*; a non-null scale_override
// replaces the inverse's 2^-k factor (or adds a factor to a forward transform)
// one-time launch attributes (64 KB dynamic shared memory of the passes) on
// the current device; done by the first transform, or ahead of stream capture
int ntt_prepare_launch();
int ntt_run(Fr* data, uint32_t k, int dir, uint32_t count, size_t bstride, const Fr* scale_override, cudaStream_t st,
            Fr* const* ptrs = nullptr);

}  // namespace lzk
