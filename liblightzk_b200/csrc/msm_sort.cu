// msm_sort.cu -- Pippenger multi-scalar multiplication for BN254 G1 and G2.
//
// Replaces multi_scalar_multiplication_g1/_g2 of the reference
// (include/operator/msm.cuh:210-247) and its kernels (msm.cuh:77-208).
// Pipeline per call, all on one stream, no host synchronisation:
//   1. k_count     signed c-bit digits of every scalar; a histogram of
//                  (window, |digit|) buckets (global atomics).
//   2. k_scan_*    exclusive prefix sum -> bucket offsets; off[B] = entries.
//   3. k_scatter   counting-sort scatter of (point index, sign) entries.
//   4. k_accumulate each thread adds exactly K consecutive sorted entries
//                  (XYZZ mixed adds of affine bases), so the work is even
//                  whatever the bucket sizes; segments that cross a chunk
//                  boundary leave partial sums.
//   5. k_fixup     folds those partial sums into their buckets: one thread
//                  per bucket with at most kFixSmall partials, one block and
//                  a shared-memory tree per larger bucket (k_fixup_large),
//                  so a bucket holding most of the entries (all scalars
//                  equal, or the sparse top window of 254-bit scalars at
//                  some widths) is summed with logarithmic depth.
//   6. k_red_*     weighted bucket sums  sum_j j*B_j  per bucket set: warp
//                  tiles of 32 buckets by shuffle scans, then bit slices of
//                  the tile index, each doubled to its weight (msm.cuh).
//   7. k_finish    windows combined by Horner (c doublings per window), or
//                  nothing to combine when the bases come with precomputed
//                  2^(c*w) shifts (every window shares one bucket set, the
//                  scheme of msm.cuh:98-115 with pre_comp_g1's table).
#include "msm.cuh"

namespace lzk {

// bits [lo, lo+c) of a canonical 254-bit scalar held as 8 limbs
__device__ __forceinline__ uint32_t window_bits(const uint32_t s[8], uint32_t lo, uint32_t c)
{
    uint32_t w = lo >> 5, sh = lo & 31;
    uint64_t v = s[w < 8 ? w : 7] >> sh;
    if (w < 8 && sh) {
        uint32_t hi = (w + 1 < 8) ? s[w + 1] : 0u;
        v = ((uint64_t)s[w] | ((uint64_t)hi << 32)) >> sh;
    } else if (w >= 8) {
        v = 0;
    }
    return (uint32_t)v & ((1u << c) - 1u);
}

// Signed-digit recoding: raw = bits + carry in [0, 2^c]; raw > 2^(c-1) is
// used as raw - 2^c with a carry into the next window.  |digit| <= 2^(c-1).
struct DigitIter {
    uint32_t s[8];
    uint32_t carry = 0;
    __device__ __forceinline__ void load(const Fr* sc)
    {
        Fr m = ldg_elem(sc);
        Fr k = from_mont(m);
        _Pragma("unroll") for (int i = 0; i < 8; i++) s[i] = k.v[i];
        carry = 0;
    }
    // returns |digit| (0 = skip) and sets neg
    __device__ __forceinline__ uint32_t next(uint32_t w, uint32_t c, bool& neg)
    {
        uint32_t raw = window_bits(s, w * c, c) + carry;
        uint32_t half = 1u << (c - 1);
        if (raw > half) { carry = 1; neg = true; return (1u << c) - raw; }
        carry = 0; neg = false; return raw;
    }
};

// Scalar i of an MSM whose scalars are the concatenation of two arrays:
// lo[0..split) then hi[0..n - split) (one array: split = n, hi unused).
__device__ __forceinline__ const Fr* scalar_at(const Fr* lo, const Fr* hi, size_t split, uint64_t i)
{
    return i < split ? lo + i : hi + (i - split);
}

__global__ void k_count(const Fr* __restrict__ scalars, const Fr* __restrict__ hi, size_t split, size_t n, uint32_t c,
                        uint32_t W, uint32_t nb, bool shared, uint32_t* __restrict__ cnt)
{
    const uint32_t B = shared ? nb : W * nb;
    (void)B;
    for (uint64_t i = gtid(); i < n; i += gstride()) {
        DigitIter it; it.load(scalar_at(scalars, hi, split, i));
        for (uint32_t w = 0; w < W; w++) {
            bool neg; uint32_t d = it.next(w, c, neg);
            uint32_t b = (shared ? 0u : w * nb) + d - 1;
            if (d && LZK_CHECK(b < B, 0)) atomicAdd(cnt + b, 1u);
        }
    }
}

__global__ void k_scatter(const Fr* __restrict__ scalars, const Fr* __restrict__ hi, size_t split, size_t n,
                          uint32_t c, uint32_t W, uint32_t nb, bool shared, size_t stride,
                          const uint32_t* __restrict__ off, uint32_t* __restrict__ cnt, uint32_t* __restrict__ ent)
{
    const uint32_t B = shared ? nb : W * nb;
    (void)B;
    for (uint64_t i = gtid(); i < n; i += gstride()) {
        DigitIter it; it.load(scalar_at(scalars, hi, split, i));
        for (uint32_t w = 0; w < W; w++) {
            bool neg; uint32_t d = it.next(w, c, neg);
            if (!d) continue;
            uint32_t b = (shared ? 0u : w * nb) + d - 1;
            if (!LZK_CHECK(b < B, 0)) continue;
            uint32_t slot = off[b] + atomicSub(cnt + b, 1u) - 1u;
            if (!LZK_CHECK(slot >= off[b] && slot < off[b + 1], 1)) continue;
            uint32_t idx = (uint32_t)(shared ? (size_t)w * stride + i : i);
            ent[slot] = idx | (neg ? 0x80000000u : 0u);
        }
    }
}

// Exclusive scan of cnt[0..B) into off[0..B], off[B] = total, in three
// passes: per-block scans of 4096 counters (1024 threads x 4), a scan of the
// block totals in one block, and the add-back of each block's offset.
constexpr uint32_t kScanBlock = 4096;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t* warp_tot, uint32_t& total)
{
    uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t v = x;
    for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, v, o); if (lane >= (uint32_t)o) v += y; }
    if (lane == 31) warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < nw ? warp_tot[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xffffffffu, t, o); if (lane >= (uint32_t)o) t += y; }
        warp_tot[lane] = t;
    }
    __syncthreads();
    total = warp_tot[nw - 1];
    uint32_t r = v - x + (wid ? warp_tot[wid - 1] : 0u);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(1024) k_scan_local(const uint32_t* __restrict__ cnt, uint32_t B,
                                                     uint32_t* __restrict__ off, uint32_t* __restrict__ bsums)
{
    __shared__ uint32_t warp_tot[32];
    uint32_t base = blockIdx.x * kScanBlock + threadIdx.x * 4;
    uint32_t v[4];
    for (int i = 0; i < 4; i++) v[i] = (base + i < B) ? cnt[base + i] : 0u;
    uint32_t sum = v[0] + v[1] + v[2] + v[3], total;
    uint32_t run = block_exclusive_scan(sum, warp_tot, total);
    for (int i = 0; i < 4; i++) {
        if (base + i < B) off[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == 0) bsums[blockIdx.x] = total;
}

// in-place exclusive scan of nb block totals; off[B] = grand total
__global__ void __launch_bounds__(1024) k_scan_top(uint32_t* __restrict__ bsums, uint32_t nb, uint32_t* __restrict__ off,
                                                   uint32_t B)
{
    __shared__ uint32_t warp_tot[32];
    uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
    uint32_t beg = threadIdx.x * per, end = min(beg + per, nb);
    uint32_t sum = 0;
    for (uint32_t i = beg; i < end; i++) sum += bsums[i];
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, warp_tot, total);
    for (uint32_t i = beg; i < end; i++) { uint32_t t = bsums[i]; bsums[i] = run; run += t; }
    if (threadIdx.x == 0) off[B] = total;
}

__global__ void k_scan_add(uint32_t* __restrict__ off, uint32_t B, const uint32_t* __restrict__ bsums)
{
    for (uint64_t i = gtid(); i < B; i += gstride()) off[i] += bsums[i / kScanBlock];
}

int scan_offsets(const uint32_t* cnt, uint32_t B, uint32_t* off, uint32_t* bsums, cudaStream_t st)
{
    uint32_t nblk = (B + kScanBlock - 1) / kScanBlock;
    if (nblk == 0) nblk = 1;
    k_scan_local<<<nblk, 1024, 0, st>>>(cnt, B, off, bsums); note_launch();
    k_scan_top<<<1, 1024, 0, st>>>(bsums, nblk, off, B); note_launch();
    k_scan_add<<<grid_for(B, 256, sm_count() * 8), 256, 0, st>>>(off, B, bsums); note_launch();
    return launch_status();
}

int msm_sort(const MsmPlan& p, const Fr* scalars, uint32_t* cnt, uint32_t* off, uint32_t* ent, uint32_t* bsums,
             cudaStream_t st, const Fr* hi, size_t split)
{
    if (!hi) split = p.n;
    if (split > p.n) return LZK_EINVAL;
    LZK_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * p.B, st));
    unsigned g = grid_for(p.n, 256, sm_count() * 16);
    k_count<<<g, 256, 0, st>>>(scalars, hi, split, p.n, p.c, p.W, p.nb, p.shared, cnt); note_launch();
    uint32_t nblk = (p.B + kScanBlock - 1) / kScanBlock;
    k_scan_local<<<nblk, 1024, 0, st>>>(cnt, p.B, off, bsums); note_launch();
    k_scan_top<<<1, 1024, 0, st>>>(bsums, nblk, off, p.B); note_launch();
    k_scan_add<<<grid_for(p.B, 256, sm_count() * 8), 256, 0, st>>>(off, p.B, bsums); note_launch();
    k_scatter<<<g, 256, 0, st>>>(scalars, hi, split, p.n, p.c, p.W, p.nb, p.shared, p.stride, off, cnt, ent); note_launch();
    return launch_status();
}

// Cost model behind the default window width: mixed adds n*W(c) (8M+2S) plus
// the reduction (two XYZZ adds per bucket, 12M+2S) plus, for plain bases,
// the serial Horner doublings, weighted by their latency cost.
// measured window widths come from the tuning table (tune.cu), by group and
// ceil(log2 n); an unset entry falls back to the model
uint32_t msm_autotune(int group, size_t n, bool shared)
{
    if (n && group >= 1 && group <= 2) {
        uint32_t w = tune_lookup(shared ? LZK_TUNE_MSM_TABLE_WINDOW : LZK_TUNE_MSM_WINDOW, group, n);
        if (w) return w;
    }
    (void)group;
    if (n == 0) return 8;
    double best = 1e300; uint32_t bc = 8;
    for (uint32_t c = 4; c <= 22; c++) {
        double W = windows_for(c);
        double sets = shared ? 1.0 : W;
        double cost = (double)n * W * 10.0 + sets * (double)(1u << (c - 1)) * 2.0 * 14.0;
        if (!shared) cost += W * c * 9.0 * 2000.0;  // serial doublings are latency bound
        if (shared && (double)n * W > 1.9e9) continue;
        if (cost < best) { best = cost; bc = c; }
    }
    return bc;
}

SortWords msm_sort_words(size_t n, uint32_t c, size_t stride)
{
    MsmPlan p;
    plan_msm<G1>(p, n, c, true, stride);
    return SortWords{p.B, (size_t)p.B + 1, p.max_entries ? p.max_entries : 1, (p.B + 4095) / 4096 + 1};
}

int msm_sort_scalars(const Fr* scalars, size_t n, uint32_t c, size_t stride, uint32_t* cnt, uint32_t* off,
                     uint32_t* ent, uint32_t* bsums, cudaStream_t st)
{
    if (!n || c < 2 || c > 24 || stride < n) return LZK_EINVAL;
    MsmPlan p;
    plan_msm<G1>(p, n, c, true, stride);
    void* tr = trace_begin("msm_shared_sort", st);
    int rc = msm_sort(p, scalars, cnt, off, ent, bsums, st);
    trace_end(tr, st);
    return rc;
}

uint32_t debug_word_sort(bool clear) { return debug_word_here(clear); }

}  // namespace lzk

using namespace lzk;

extern "C" {

uint32_t lzk_msm_precomp_windows(uint32_t window_bits) { return window_bits ? windows_for(window_bits) : 0; }

uint32_t lzk_msm_autotune_window(int group, size_t n, uint32_t flags)
{
    return msm_autotune(group, n, (flags & LZK_MSM_PRECOMPUTED) != 0);
}

size_t lzk_msm_workspace_bytes(int group, size_t n, const lzk_msm_cfg* cfg)
{
    bool shared = cfg && (cfg->flags & LZK_MSM_PRECOMPUTED);
    uint32_t c = (cfg && cfg->window_bits) ? cfg->window_bits : msm_autotune(group, n, shared);
    if (c < 2 || c > 24 || n == 0) return 0;
    uint32_t chunk = msm_chunk(cfg, group, n), run = msm_run(cfg, group, n);
    if (!tune_valid(LZK_TUNE_MSM_CHUNK, chunk)) return 0;
    MsmPlan p;
    if (group == 2) plan_msm<G2>(p, n, c, shared, cfg ? cfg->level_stride : 0, chunk, run);
    else plan_msm<G1>(p, n, c, shared, cfg ? cfg->level_stride : 0, chunk, run);
    return p.bytes;
}

}  // extern "C"
