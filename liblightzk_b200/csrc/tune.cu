// tune.cu -- the tuning table: per size class, the values the operators use
// when their configuration leaves them open.
//
// The reference fixes all of them at compile time (window width 12 and 4096
// buckets, msm.cuh:216-227; one global-memory launch per NTT stage,
// poly.cuh:42-63).  Here each is looked up by knob, group (1 = G1, 2 = G2)
// and size class log_n = ceil(log2 n), and liblightzk_b200.autotune fills
// the table from timings on the device.  An unset entry (0) means the
// built-in default: the cost model's window width, 64 entries per
// accumulation thread, runs of 4 buckets per lane, 2048 elements per NTT
// block.  MSMs over shifted-copy tables (one bucket set for all windows)
// have their own window, chunk and run entries: their best values differ
// from those of plain-base MSMs of the same size.
#include "common.cuh"
#include "tune.cuh"
#include <atomic>

namespace lzk {

static std::atomic<uint32_t> g_tune[kTuneKnobs][3][33];

uint32_t log2_ceil(size_t n)
{
    uint32_t lg = 0;
    while (lg < 32 && (size_t(1) << lg) < n) lg++;
    return lg;
}

uint32_t tune_lookup(int knob, int group, size_t n)
{
    if (knob < 0 || knob >= kTuneKnobs || group < 0 || group > 2) return 0;
    return g_tune[knob][group][log2_ceil(n)].load(std::memory_order_relaxed);
}

uint32_t tune_chunk(int group, size_t n, bool shared)
{
    uint32_t v = tune_lookup(shared ? LZK_TUNE_MSM_TABLE_CHUNK : LZK_TUNE_MSM_CHUNK, group, n);
    return v ? v : kDefaultChunk;
}

uint32_t tune_run(int group, size_t n, bool shared)
{
    uint32_t v = tune_lookup(shared ? LZK_TUNE_MSM_TABLE_RUN : LZK_TUNE_MSM_REDUCE_RUN, group, n);
    return v ? v : kDefaultRun;
}

uint32_t tune_ntt_block(uint32_t log_n)
{
    uint32_t v = log_n <= 32 ? g_tune[LZK_TUNE_NTT_BLOCK][0][log_n].load(std::memory_order_relaxed) : 0;
    return v ? v : kDefaultNttBlock;
}

static bool pow2(uint32_t v) { return v && !(v & (v - 1)); }

bool tune_valid(int knob, uint32_t v)
{
    if (v == 0) return true;
    switch (knob) {
        case LZK_TUNE_MSM_WINDOW:
        case LZK_TUNE_MSM_TABLE_WINDOW: return v >= 2 && v <= 24;
        case LZK_TUNE_MSM_CHUNK:
        case LZK_TUNE_MSM_TABLE_CHUNK: return pow2(v) && v >= kMinChunk && v <= kMaxChunk;
        case LZK_TUNE_MSM_REDUCE_RUN:
        case LZK_TUNE_MSM_TABLE_RUN: return pow2(v) && v <= kMaxRun;
        case LZK_TUNE_NTT_BLOCK: return pow2(v) && v >= kMinNttBlock && v <= kMaxNttBlock;
        default: return false;
    }
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_tune_set(int knob, int group, uint32_t log_n, uint32_t value)
{
    if (knob < 0 || knob >= kTuneKnobs || log_n > 32 || !tune_valid(knob, value)) return LZK_EINVAL;
    if (knob == LZK_TUNE_NTT_BLOCK) group = 0;
    else if (group < 1 || group > 2) return LZK_EINVAL;
    g_tune[knob][group][log_n].store(value, std::memory_order_relaxed);
    return LZK_OK;
}

uint32_t lzk_tune_get(int knob, int group, uint32_t log_n)
{
    if (knob < 0 || knob >= kTuneKnobs || log_n > 32) return 0;
    if (knob == LZK_TUNE_NTT_BLOCK) return tune_ntt_block(log_n);
    if (group < 1 || group > 2) return 0;
    size_t n = size_t(1) << (log_n < 63 ? log_n : 62);
    switch (knob) {
        case LZK_TUNE_MSM_CHUNK: return tune_chunk(group, n, false);
        case LZK_TUNE_MSM_REDUCE_RUN: return tune_run(group, n, false);
        case LZK_TUNE_MSM_TABLE_CHUNK: return tune_chunk(group, n, true);
        case LZK_TUNE_MSM_TABLE_RUN: return tune_run(group, n, true);
        default: return g_tune[knob][group][log_n].load(std::memory_order_relaxed);
    }
}

int lzk_msm_set_window(int group, uint32_t log_n, uint32_t window_bits)
{
    return lzk_tune_set(LZK_TUNE_MSM_WINDOW, group, log_n, window_bits);
}

}  // extern "C"
