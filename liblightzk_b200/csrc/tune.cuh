// tune.cuh -- lookups in the tuning table (tune.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include "lzk.h"

namespace lzk {

constexpr int kTuneKnobs = 7;
constexpr uint32_t kDefaultChunk = 64, kMinChunk = 8, kMaxChunk = 512;
constexpr uint32_t kDefaultRun = 4, kMaxRun = 16;
constexpr uint32_t kDefaultNttBlock = 2048, kMinNttBlock = 256, kMaxNttBlock = 4096;

uint32_t log2_ceil(size_t n);
// the table's value (0 = unset) for the size class of n
uint32_t tune_lookup(int knob, int group, size_t n);
// accumulation chunk and reduction lane run of an MSM over plain bases or,
// with shared set, over a shifted-copy table; NTT block: table value or
// default
uint32_t tune_chunk(int group, size_t n, bool shared);
uint32_t tune_run(int group, size_t n, bool shared);
uint32_t tune_ntt_block(uint32_t log_n);
bool tune_valid(int knob, uint32_t v);

}  // namespace lzk
