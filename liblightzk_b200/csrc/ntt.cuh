// ntt.cuh -- internal interface of the NTT (ntt.cu) for other operators.
#pragma once
#include "common.cuh"
#include "field52.cuh"

namespace lzk {

struct NttTables {
    Fr* tw[2] = {nullptr, nullptr};  // w^e, w^-e for e < n/2
    // the same twiddles as radix-2^52 limbs in doubles (the FP64 product's
    // operand form, field52.cuh), kTwdStride doubles per twiddle
    double* twd[2] = {nullptr, nullptr};
    Fr* consts = nullptr;            // see k_ntt_consts
};
constexpr uint32_t kTwdStride = 6;   // 5 limbs and a pad: 48-byte records, three 16-byte loads
// Transforms up to 2^kTwdMaxLog read the radix-2^52 table (its 2^(k-1)
// records of 48 bytes stay in L2); larger ones the 32-byte table (at 2^24
// both measured the same).
constexpr uint32_t kTwdMaxLog = 21;
inline const double* twd_for(const NttTables& t, int inv, uint32_t k) { return k <= kTwdMaxLog ? t.twd[inv] : nullptr; }

struct CosetTables {
    Fr* lo[2] = {nullptr, nullptr};  // g^j, g^-j for j < 4096
    Fr* hi[2] = {nullptr, nullptr};  // g^(4096 i), g^-(4096 i) for i < 2^(26-12)
};

// Factor applied to every element as the first pass of a transform loads
// it (pre) or the last pass stores it (post): x * scale * g^e with g^e from
// the power tables lo/hi (g^j = lo[j & 4095] * hi[j >> 12]) and e the
// element's position, or the bit reversal of its position when brev is set
// (the coefficient index a bit-reversed position holds).  Null scale / null
// tables: factor 1.
struct NttEdge {
    const Fr* lo = nullptr;
    const Fr* hi = nullptr;
    const Fr* scale = nullptr;
    uint32_t brev = 0;
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
// The passes of `count` transforms of size 2^k (k >= 1) with twiddle table
// tw (w^e, e < n/2) and no bit reversal: DIF takes natural order to
// bit-reversed order, DIT bit-reversed order to natural order.  pre applies
// to the first pass's loads, post to the last pass's stores.  twd, when
// given, is the same table in radix-2^52 form (NttTables::twd), which the
// butterflies then read instead of converting tw.
int ntt_passes(Fr* data, uint32_t k, uint32_t count, size_t bstride, const Fr* tw, bool dit, NttEdge pre,
               NttEdge post, cudaStream_t st, Fr* const* ptrs = nullptr, const double* twd = nullptr);

}  // namespace lzk
