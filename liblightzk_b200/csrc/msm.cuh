// msm.cuh -- shared pieces of the Pippenger MSM (msm_sort.cu, msm_g1.cu,
// msm_g2.cu).  See msm_sort.cu for the pipeline.
#pragma once
#include "common.cuh"
#include "curve.cuh"
#include "tune.cuh"

namespace lzk {

struct G1 { using F = Fq; };
struct G2 { using F = Fq2; };

constexpr uint32_t kLevelL = 32;     // smallest warp tile of the bucket reduction (scratch bound)
constexpr uint32_t kFixSmall = 64;   // partials a single fix-up thread folds

struct MsmPlan {
    size_t n = 0;
    uint32_t c = 0;        // window bits
    uint32_t W = 0;        // digit windows
    uint32_t nb = 0;       // buckets per window = 2^(c-1)
    uint32_t wb = 0;       // bucket sets: W (plain) or 1 (shared, precomputed)
    uint32_t B = 0;        // total buckets = wb * nb
    bool shared = false;   // precomputed table: one bucket set for all windows
    size_t stride = 0;     // table level stride
    size_t max_entries = 0;
    uint32_t chunk = 0;    // sorted entries per accumulation thread
    uint32_t run = 0;      // buckets per lane run of the reduction tiles
    size_t chunks = 0;
    // workspace offsets
    size_t o_cnt, o_off, o_ent, o_bsum, o_head, o_tail, o_lr0, o_la0, o_lr1, o_la1, o_scan, o_large, bytes;
};

inline uint32_t windows_for(uint32_t c) { return (255 + c - 1) / c; }

// accumulation chunk and reduction run of an MSM of n points in group g:
// cfg's values, else the tuning table's (plain bases, or tables with
// LZK_MSM_PRECOMPUTED)
inline bool msm_shared(const lzk_msm_cfg* cfg) { return cfg && (cfg->flags & LZK_MSM_PRECOMPUTED); }
inline uint32_t msm_chunk(const lzk_msm_cfg* cfg, int group, size_t n)
{
    return cfg && cfg->acc_chunk ? cfg->acc_chunk : tune_chunk(group, n, msm_shared(cfg));
}
inline uint32_t msm_run(const lzk_msm_cfg* cfg, int group, size_t n)
{
    return cfg && cfg->reduce_run ? cfg->reduce_run : tune_run(group, n, msm_shared(cfg));
}

template <class Gp>
inline void plan_msm(MsmPlan& p, size_t n, uint32_t c, bool shared, size_t stride, uint32_t chunk = kDefaultChunk,
                     uint32_t run = kDefaultRun)
{
    using X = XYZZ<typename Gp::F>;
    p.n = n; p.c = c; p.W = windows_for(c); p.nb = 1u << (c - 1);
    p.shared = shared; p.stride = stride;
    p.wb = shared ? 1 : p.W;
    p.B = p.wb * p.nb;
    p.max_entries = n * (size_t)p.W;
    p.chunk = chunk;
    p.run = run;
    p.chunks = (p.max_entries + chunk - 1) / chunk;
    // bucket reduction scratch: wb * max(1, nb / kLevelL) points per buffer
    // (reduce_buckets)
    size_t lvl = (size_t)p.wb * (p.nb > kLevelL ? p.nb / kLevelL : 1);
    Carver cv;
    p.o_cnt = cv.take<uint32_t>(p.B);
    p.o_off = cv.take<uint32_t>(p.B + 1);
    p.o_ent = cv.take<uint32_t>(p.max_entries ? p.max_entries : 1);
    p.o_bsum = cv.take<X>(p.B);
    p.o_head = cv.take<X>(p.chunks ? p.chunks : 1);
    p.o_tail = cv.take<X>(p.chunks ? p.chunks : 1);
    p.o_lr0 = cv.take<X>(lvl);
    p.o_la0 = cv.take<X>(lvl);
    p.o_lr1 = cv.take<X>(lvl);
    p.o_la1 = cv.take<X>(lvl);
    p.o_scan = cv.take<uint32_t>((p.B + 4095) / 4096 + 1);
    p.o_large = cv.take<uint32_t>(p.chunks / kFixSmall + 2);   // count, then bucket ids
    p.bytes = cv.off;
}

// counting sort of the signed digits of all scalars into bucket lists:
// cnt/off/ent as carved by plan_msm (msm_sort.cu).  With hi given, the
// scalars are scalars[0..split) followed by hi[0..n - split).
int msm_sort(const MsmPlan& p, const Fr* scalars, uint32_t* cnt, uint32_t* off, uint32_t* ent, uint32_t* bsums,
             cudaStream_t st, const Fr* hi = nullptr, size_t split = 0);
uint32_t msm_autotune(int group, size_t n, bool shared);

// One digit sort shared by several shifted-table MSMs over the same scalars
// (the Groth16 A, B1 and B2 queries all take the witness): sizes of its
// buffers in 32-bit words, the sort itself, and the G1 / G2 MSMs that consume
// it (msm_sort.cu, msm_g1.cu, msm_g2.cu).  The consumers must use the same
// n, window width and table level stride as the sort.
struct SortWords { size_t cnt, off, ent, bsums; };
SortWords msm_sort_words(size_t n, uint32_t c, size_t stride);
int msm_sort_scalars(const Fr* scalars, size_t n, uint32_t c, size_t stride, uint32_t* cnt, uint32_t* off,
                     uint32_t* ent, uint32_t* bsums, cudaStream_t st);
int msm_g1_presorted(const Fr* scalars, const void* table, size_t n, Jac<Fq>* out, const lzk_msm_cfg* cfg,
                     cudaStream_t st, const uint32_t* off, const uint32_t* ent);
int msm_g2_presorted(const Fr* scalars, const void* table, size_t n, Jac<Fq2>* out, const lzk_msm_cfg* cfg,
                     cudaStream_t st, const uint32_t* off, const uint32_t* ent);
// A shifted-table G1 MSM whose scalars are two arrays, lo[0..n_lo) then
// hi[0..n_hi), over one table of n_lo + n_hi points per level (msm_g1.cu):
// two MSMs whose results are only ever added, done as one (one sort, one
// bucket set, one reduction).  cfg must carry a workspace.
int msm_g1_concat(const Fr* lo, size_t n_lo, const Fr* hi, size_t n_hi, const void* table, Jac<Fq>* out,
                  const lzk_msm_cfg* cfg, cudaStream_t st);
// exclusive scan of cnt[0..B) into off[0..B], off[B] = total; bsums holds
// (B + 4095) / 4096 + 1 words (msm_sort.cu)
int scan_offsets(const uint32_t* cnt, uint32_t B, uint32_t* off, uint32_t* bsums, cudaStream_t st);

// largest b in [lo, B) with off[b] <= e
__device__ __forceinline__ uint32_t bucket_of(const uint32_t* off, uint32_t lo, uint32_t B, uint32_t e)
{
    uint32_t hi = B;  // invariant: off[lo] <= e, answer in [lo, hi)
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= e) lo = mid; else hi = mid;
    }
    return lo;
}

// Base record layouts (lzk_msm_cfg.base_layout):
//   LZK_BASES_AFFINE        {x, y}, infinity = (0, 0)
//   LZK_BASES_REF_G1_JAC    the reference's G1 table records, Jacobian
//                           {X, Y, Z} (96 B) normalised by pre_comp_g1 to
//                           Z = 1 (msm.cuh:48-61); Z = 0 is infinity
//   LZK_BASES_REF_G2_LANES  the reference's device G2 records: two 96-B
//                           halves {X.c0 Y.c0 Z.c0}{X.c1 Y.c1 Z.c1}
//                           (alt_bn128_t.cuh:247-256), normalised to Z = 1
template <class F, int LAYOUT>
__device__ __forceinline__ Aff<F> load_raw(const void* bases, uint32_t idx);

template <>
__device__ __forceinline__ Aff<Fq> load_raw<Fq, LZK_BASES_AFFINE>(const void* bases, uint32_t idx)
{
    return ldg_elem(reinterpret_cast<const Aff<Fq>*>(bases) + idx);
}
template <>
__device__ __forceinline__ Aff<Fq2> load_raw<Fq2, LZK_BASES_AFFINE>(const void* bases, uint32_t idx)
{
    return ldg_elem(reinterpret_cast<const Aff<Fq2>*>(bases) + idx);
}
template <>
__device__ __forceinline__ Aff<Fq> load_raw<Fq, LZK_BASES_REF_G1_JAC>(const void* bases, uint32_t idx)
{
    Jac<Fq> j = ldg_elem(reinterpret_cast<const Jac<Fq>*>(bases) + idx);
    if (j.Z.is_zero()) return Aff<Fq>{Fq::zero(), Fq::zero()};
    return Aff<Fq>{j.X, j.Y};
}
template <>
__device__ __forceinline__ Aff<Fq2> load_raw<Fq2, LZK_BASES_REF_G2_LANES>(const void* bases, uint32_t idx)
{
    const Jac<Fq>* h = reinterpret_cast<const Jac<Fq>*>(bases) + 2 * (size_t)idx;
    Jac<Fq> h0 = ldg_elem(h), h1 = ldg_elem(h + 1);
    if (h0.Z.is_zero() && h1.Z.is_zero()) return Aff<Fq2>{Fq2::zero(), Fq2::zero()};
    return Aff<Fq2>{Fq2{h0.X, h1.X}, Fq2{h0.Y, h1.Y}};
}

template <class F, int LAYOUT>
__device__ __forceinline__ Aff<F> load_base(const void* bases, uint32_t v)
{
    Aff<F> p = load_raw<F, LAYOUT>(bases, v & 0x7fffffffu);
    if (v & 0x80000000u) { if (!aff_is_inf(p)) p.y = neg(p.y); }
    return p;
}

// The work of one accumulation thread, chunk t (k_accumulate below; the
// persistent batch kernel runs it too).
template <class F, int LAYOUT>
__device__ __forceinline__ void accumulate_chunk(uint64_t t, const void* __restrict__ bases,
                                                 const uint32_t* __restrict__ ent, const uint32_t* __restrict__ off,
                                                 uint32_t B, size_t chunks, uint32_t chunk, uint64_t nbases,
                                                 XYZZ<F>* __restrict__ bsum, XYZZ<F>* __restrict__ head,
                                                 XYZZ<F>* __restrict__ tail)
{
    (void)nbases;   // the base records behind the entries (debug checks)
    if (t >= chunks) return;
    uint32_t T = off[B];
    uint64_t cs64 = t * chunk;
    if (cs64 >= T) return;
    uint32_t cs = (uint32_t)cs64, ce = (uint32_t)min((uint64_t)cs + chunk, (uint64_t)T);
    uint32_t b = bucket_of(off, 0, B, cs);
    uint32_t bbeg = off[b], bend = off[b + 1];
    XYZZ<F> acc = xyzz_inf<F>();
    for (uint32_t e = cs; e < ce; e++) {
        if (e == bend) {
            // bucket b finished inside this chunk
            if (bbeg < cs) st_elem(head + t, acc); else st_elem(bsum + b, acc);
            // almost always the next bucket (at the prover's width a bucket
            // holds about 240 entries): one offset load instead of a binary
            // search of 16 dependent loads, which measured 0.9 % (G1) and
            // 1.3 % (G2) faster; searched only past an empty bucket.  Since
            // e < off[B], b + 1 < B and off[b + 2] exists.
            if (!LZK_CHECK(b + 2 <= B, 3)) return;
            bbeg = bend;
            bend = off[b + 2];
            b = b + 1;
            if (bend <= e) {
                b = bucket_of(off, b + 1, B, e);
                bbeg = off[b]; bend = off[b + 1];
            }
            acc = xyzz_inf<F>();
        }
        const uint32_t v = ent[e];
        if (!LZK_CHECK((v & 0x7fffffffu) < nbases, 2)) continue;
        acc = xyzz_madd(acc, load_base<F, LAYOUT>(bases, v));
    }
    bool began_before = bbeg < cs, cont_after = bend > ce;
    if (began_before) st_elem(head + t, acc);
    else if (cont_after) st_elem(tail + t, acc);
    else st_elem(bsum + b, acc);
}
// 128-thread blocks; at most 168 registers for G1 (3 blocks = 12 warps per
// SM) and 255 for G2 (2 blocks).  With the products on the FP64 pipe the
// tighter register bounds make the product calls spill: G1 at 3 blocks/SM
// measured 6 % faster than at 5 (which matched 4 and 6), G2 at 2 blocks 10 %
// faster than at 3 and 16 % faster than at 4.
template <class F, int LAYOUT>
__global__ void __launch_bounds__(128, sizeof(F) == 32 ? 3 : 2) k_accumulate(const void* __restrict__ bases, const uint32_t* __restrict__ ent,
                                                    const uint32_t* __restrict__ off, uint32_t B, size_t chunks,
                                                    uint32_t chunk, uint64_t nbases, XYZZ<F>* __restrict__ bsum,
                                                    XYZZ<F>* __restrict__ head, XYZZ<F>* __restrict__ tail)
{
    accumulate_chunk<F, LAYOUT>(gtid(), bases, ent, off, B, chunks, chunk, nbases, bsum, head, tail);
}

template <class F>
__device__ __forceinline__ void fixup_items(const uint32_t* __restrict__ off, uint32_t B, uint32_t chunk, uint64_t chunks,
                        XYZZ<F>* __restrict__ bsum, const XYZZ<F>* __restrict__ head, const XYZZ<F>* __restrict__ tail,
                        uint32_t* __restrict__ large)
{
    (void)chunks;
    for (uint64_t b = gtid(); b < B; b += gstride()) {
        uint32_t s = off[b], e = off[b + 1];
        if (s == e) continue;
        uint32_t c0 = s / chunk, c1 = (e - 1) / chunk;
        if (!LZK_CHECK(c1 < chunks, 4)) continue;
        if (c0 == c1) continue;
        if (c1 - c0 > kFixSmall) {
            large[1 + atomicAdd(large, 1u)] = (uint32_t)b;
            continue;
        }
        XYZZ<F> acc = ld_elem(tail + c0);
        for (uint32_t c = c0 + 1; c <= c1; c++) acc = xyzz_add_cold(acc, ld_elem(head + c));
        st_elem(bsum + b, acc);
    }
}
template <class F>
__global__ void k_fixup(const uint32_t* __restrict__ off, uint32_t B, uint32_t chunk, uint64_t chunks,
                        XYZZ<F>* __restrict__ bsum, const XYZZ<F>* __restrict__ head, const XYZZ<F>* __restrict__ tail,
                        uint32_t* __restrict__ large)
{
    fixup_items<F>(off, B, chunk, chunks, bsum, head, tail, large);
}

// One block per listed bucket: strided partial sums, then a tree in shared
// memory.  Partial q of bucket b is tail[c0] (q = 0) or head[c0 + q].
// (blockDim.x points of shared memory at sm; the persistent batch kernel
// runs it too)
template <class F>
__device__ __forceinline__ void fixup_large_items(const uint32_t* __restrict__ off, uint32_t chunk,
                                                  XYZZ<F>* __restrict__ bsum, const XYZZ<F>* __restrict__ head,
                                                  const XYZZ<F>* __restrict__ tail, const uint32_t* __restrict__ large,
                                                  XYZZ<F>* sm)
{
    uint32_t nl = large[0];
    for (uint32_t idx = blockIdx.x; idx < nl; idx += gridDim.x) {
        uint32_t b = large[1 + idx];
        uint32_t c0 = off[b] / chunk, c1 = (off[b + 1] - 1) / chunk;
        uint32_t np = c1 - c0 + 1;
        XYZZ<F> acc = xyzz_inf<F>();
        for (uint32_t q = threadIdx.x; q < np; q += blockDim.x)
            acc = xyzz_add_cold(acc, ld_elem(q ? head + c0 + q : tail + c0));
        st_elem(sm + threadIdx.x, acc);
        __syncthreads();
        for (uint32_t h = blockDim.x / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) st_elem(sm + threadIdx.x, xyzz_add_cold(ld_elem(sm + threadIdx.x), ld_elem(sm + threadIdx.x + h)));
            __syncthreads();
        }
        if (threadIdx.x == 0) st_elem(bsum + b, ld_elem(sm));
        __syncthreads();
    }
}
template <class F>
__global__ void k_fixup_large(const uint32_t* __restrict__ off, uint32_t chunk, XYZZ<F>* __restrict__ bsum,
                              const XYZZ<F>* __restrict__ head, const XYZZ<F>* __restrict__ tail,
                              const uint32_t* __restrict__ large)
{
    extern __shared__ uint4 fx_raw[];
    fixup_large_items<F>(off, chunk, bsum, head, tail, large, reinterpret_cast<XYZZ<F>*>(fx_raw));
}

// Warp shuffles of whole points
template <class F>
__device__ __forceinline__ XYZZ<F> shfl_down_pt(const XYZZ<F>& x, uint32_t d)
{
    XYZZ<F> r;
    const uint32_t* s = reinterpret_cast<const uint32_t*>(&x);
    uint32_t* o = reinterpret_cast<uint32_t*>(&r);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(XYZZ<F>) / 4); i++) o[i] = __shfl_down_sync(0xffffffffu, s[i], d);
    return r;
}
template <class F>
__device__ __forceinline__ XYZZ<F> shfl_xor_pt(const XYZZ<F>& x, uint32_t m)
{
    XYZZ<F> r;
    const uint32_t* s = reinterpret_cast<const uint32_t*>(&x);
    uint32_t* o = reinterpret_cast<uint32_t*>(&r);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(XYZZ<F>) / 4); i++) o[i] = __shfl_xor_sync(0xffffffffu, s[i], m);
    return r;
}
template <class F>
__device__ __forceinline__ XYZZ<F> shfl_pt(const XYZZ<F>& x, uint32_t lane)
{
    XYZZ<F> r;
    const uint32_t* s = reinterpret_cast<const uint32_t*>(&x);
    uint32_t* o = reinterpret_cast<uint32_t*>(&r);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(XYZZ<F>) / 4); i++) o[i] = __shfl_sync(0xffffffffu, s[i], lane);
    return r;
}

// ---------------------------- bucket reduction ----------------------------
// Per bucket set (one per window for plain bases, one for all windows with a
// shifted-copy table) of m = 2^(c-1) buckets B_0..B_{m-1}, bucket k holding
// digit k + 1, the weighted sum W = sum_k (k+1) B_k.  With tiles of L
// buckets and P = m / L tiles,
//   W = sum_u t_u + L sum_u u R_u = T + sum_{i < log P} 2^(i + log L) G_i,
// where R_u is the sum of tile u, t_u = sum_j (j+1) B_{uL+j} its locally
// weighted sum, T = sum_u t_u and G_i = sum of the R_u with bit i of u set
// (bit slices of the tile index).  Four launches, each over the items of
// any number of jobs (reduce_jobs):
//   k_red_tile     one warp per tile (below);
//   k_red_slices   one warp per 32 members of one of the 1 + log P sums T,
//                  G_0, G_1, ... (xor-shuffle tree);
//   k_red_scale    one warp per sum: fold its partials, double it
//                  i + log L times (warp-uniform doublings);
//   k_red_combine  one warp per set: add the scaled sums.
// For m = 2^16 the longest chain is 19 + 5 + 6 + 15 doublings + 5 dependent
// point operations; a ladder of 32-bucket levels with the weights carried by
// doublings at every level needs about twice that.  Empty buckets
// (off[k] == off[k+1]) read as the point at infinity.
//
// k_red_tile: lane j of a tile holds the run of r consecutive buckets
// jr .. jr + r - 1 (r = 4 for m >= 128, L = 32 r; smaller sets take r = 2 or
// 1 and L = m).  The lane forms the run's sum s_j and its locally weighted
// sum t_j = sum_i (i+1) B_{jr+i} by running sums (two additions per
// bucket), a shuffle suffix scan gives S_j = sum_{j'>=j} s_j', and since the
// tile-local weight of bucket jr + i is jr + i + 1,
//   R_u = S_0,   t_u = sum_j (t_j + r [j >= 1] S_j).
// About 4.75 additions per bucket for r = 4, against 10 for a warp scan over
// single buckets (r = 1).
struct RedShape {
    uint32_t r, L, lgL, P, lg;   // buckets per lane run, tile size, log2 L, tiles per set, log2 P
    uint32_t cT, cG, NP, NS;     // chunks of T, chunks of each G_i, partials and sums per set
};
// run: requested buckets per lane run (a power of two); a set too small
// for 32 lanes of such runs takes shorter runs, down to single buckets
inline RedShape red_shape(uint32_t m, uint32_t run = kDefaultRun)
{
    RedShape s;
    s.r = run ? run : 1;
    while (s.r > 1 && 32 * s.r > m) s.r >>= 1;
    s.L = m < 32 * s.r ? m : 32 * s.r;
    s.lgL = 0; while ((1u << s.lgL) < s.L) s.lgL++;
    s.P = m / s.L;
    s.lg = 0; while ((1u << s.lg) < s.P) s.lg++;
    s.cT = (s.P + 31) / 32;
    s.cG = (s.P / 2 + 31) / 32;
    s.NP = s.cT + s.lg * s.cG;
    s.NS = 1 + s.lg;
    return s;
}

// member v of slice i: the v-th tile index with bit i set
__device__ __forceinline__ uint32_t slice_member(uint32_t v, uint32_t i)
{
    return ((v >> i) << (i + 1)) | (1u << i) | (v & ((1u << i) - 1));
}

// One reduction job: wb sets of m buckets (bsum / off indexed w m + k) into
// win[0..wb), with scratch R, T, part, scaled of its own (at least wb * P
// points each; NP, NS <= P), so that the jobs of several window widths (a
// batch plan's width groups) run in the same launches.  s_* is the job's
// first item in each launch's item space (the items of all jobs laid end to
// end: tiles wb P, slice partials wb NP, sums wb NS, sets wb).
template <class F>
struct RedJob {
    const XYZZ<F>* bsum;
    const uint32_t* off;
    XYZZ<F> *R, *T, *part, *scaled, *win;
    uint32_t wb, m;
    RedShape sh;
    uint64_t s_tile, s_np, s_ns, s_w;
};
constexpr uint32_t kMaxRedJobs = 20;   // a kernel parameter of about 3 KB
template <class F>
struct RedJobs {
    uint32_t count;
    RedJob<F> g[kMaxRedJobs];
};

// the job whose items include `item` (jobs in item order)
template <class F>
__device__ __forceinline__ uint32_t red_job_of(const RedJobs<F>& jobs, uint64_t item, uint64_t RedJob<F>::*start)
{
    uint32_t j = 0;
    while (j + 1 < jobs.count && item >= jobs.g[j + 1].*start) j++;
    return j;
}

template <class F>
__device__ __forceinline__ void red_tile_items(const RedJobs<F>& jobs, uint64_t total)
{
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t item = gtid() >> 5; item < total; item += gstride() >> 5) {
        const RedJob<F>& J = jobs.g[red_job_of(jobs, item, &RedJob<F>::s_tile)];
        const uint64_t tile = item - J.s_tile;
        const uint32_t L = J.sh.L, r = J.sh.r;
        const uint32_t nl = L / r;   // active lanes
        XYZZ<F> s = xyzz_inf<F>(), t = xyzz_inf<F>();
        if (lane < nl) {
            const size_t k0 = (size_t)tile * L + (size_t)lane * r;   // = w m + u L + j r
            for (int i = (int)r - 1; i >= 0; i--) {
                size_t k = k0 + (uint32_t)i;
                if (J.off[k] != J.off[k + 1]) s = xyzz_add_cold(s, ld_elem(J.bsum + k));
                t = xyzz_add_cold(t, s);
            }
        }
        XYZZ<F> S = s;
        for (uint32_t d = 1; d < nl; d <<= 1) {
            XYZZ<F> o = shfl_down_pt(S, d);
            if (lane + d < nl) S = xyzz_add_cold(S, o);
        }
        XYZZ<F> U = (lane >= 1 && lane < nl) ? S : xyzz_inf<F>();
        for (uint32_t q = r; q > 1; q >>= 1) U = xyzz_dbl_cold(U);
        XYZZ<F> V = xyzz_add_cold(t, U);
        for (uint32_t d = nl >> 1; d > 0; d >>= 1) V = xyzz_add_cold(V, shfl_xor_pt(V, d));
        if (lane == 0) {
            st_elem(J.R + tile, S);
            st_elem(J.T + tile, V);
        }
    }
}
template <class F>
__global__ void __launch_bounds__(128) k_red_tile(const __grid_constant__ RedJobs<F> jobs, uint64_t total)
{
    red_tile_items<F>(jobs, total);
}


template <class F>
__device__ __forceinline__ void red_slices_items(const RedJobs<F>& jobs, uint64_t total)
{
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t item = gtid() >> 5; item < total; item += gstride() >> 5) {
        const RedJob<F>& J = jobs.g[red_job_of(jobs, item, &RedJob<F>::s_np)];
        const RedShape& sh = J.sh;
        const uint64_t g = item - J.s_np;
        uint32_t w = (uint32_t)(g / sh.NP), q = (uint32_t)(g % sh.NP);
        const size_t base = (size_t)w * sh.P;
        XYZZ<F> x = xyzz_inf<F>();
        if (q < sh.cT) {
            uint32_t v = q * 32 + lane;
            if (v < sh.P) x = ld_elem(J.T + base + v);
        } else {
            uint32_t i = (q - sh.cT) / sh.cG, v = ((q - sh.cT) % sh.cG) * 32 + lane;
            if (v < sh.P / 2) x = ld_elem(J.R + base + slice_member(v, i));
        }
        for (uint32_t d = 16; d > 0; d >>= 1) x = xyzz_add_cold(x, shfl_xor_pt(x, d));
        if (lane == 0) st_elem(J.part + g, x);
    }
}
template <class F>
__global__ void __launch_bounds__(128) k_red_slices(const __grid_constant__ RedJobs<F> jobs, uint64_t total)
{
    red_slices_items<F>(jobs, total);
}

template <class F>
__device__ __forceinline__ void red_scale_items(const RedJobs<F>& jobs, uint64_t total)
{
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t item = gtid() >> 5; item < total; item += gstride() >> 5) {
        const RedJob<F>& J = jobs.g[red_job_of(jobs, item, &RedJob<F>::s_ns)];
        const RedShape& sh = J.sh;
        const uint64_t g = item - J.s_ns;
        uint32_t w = (uint32_t)(g / sh.NS), s = (uint32_t)(g % sh.NS);
        uint32_t first = s == 0 ? 0 : sh.cT + (s - 1) * sh.cG, cnt = s == 0 ? sh.cT : sh.cG;
        const XYZZ<F>* src = J.part + (size_t)w * sh.NP + first;
        XYZZ<F> x = xyzz_inf<F>();
        for (uint32_t c = lane; c < cnt; c += 32) x = xyzz_add_cold(x, ld_elem(src + c));
        for (uint32_t d = 16; d > 0; d >>= 1) x = xyzz_add_cold(x, shfl_xor_pt(x, d));
        // lanes may hold different representations of the sum (an addition
        // with swapped operands negates Y and ZZZ); the warp-uniform
        // doublings need one
        x = shfl_pt(x, 0);
        uint32_t dbls = s == 0 ? 0 : s - 1 + sh.lgL;
        for (uint32_t d = 0; d < dbls; d++) x = xyzz_dbl_warp(x);
        if (lane == 0) st_elem(J.scaled + g, x);
    }
}
template <class F>
__global__ void __launch_bounds__(128) k_red_scale(const __grid_constant__ RedJobs<F> jobs, uint64_t total)
{
    red_scale_items<F>(jobs, total);
}

template <class F>
__device__ __forceinline__ void red_combine_items(const RedJobs<F>& jobs, uint64_t total)
{
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t item = gtid() >> 5; item < total; item += gstride() >> 5) {
        const RedJob<F>& J = jobs.g[red_job_of(jobs, item, &RedJob<F>::s_w)];
        const uint64_t w = item - J.s_w;
        const uint32_t NS = J.sh.NS;
        XYZZ<F> x = lane < NS ? ld_elem(J.scaled + w * NS + lane) : xyzz_inf<F>();
        for (uint32_t d = 16; d > 0; d >>= 1) x = xyzz_add_cold(x, shfl_xor_pt(x, d));
        if (lane == 0) st_elem(J.win + w, x);
    }
}
template <class F>
__global__ void __launch_bounds__(128) k_red_combine(const __grid_constant__ RedJobs<F> jobs, uint64_t total)
{
    red_combine_items<F>(jobs, total);
}

// Scratch points each of R, T, part and scaled needs for wb sets of m
// buckets (any run: P <= max(1, m / kLevelL), NP, NS <= P).
inline size_t red_scratch_points(uint32_t wb, uint32_t m) { return (size_t)wb * (m > kLevelL ? m / kLevelL : 1); }

template <class F>
RedJob<F> red_job(const XYZZ<F>* bsum, const uint32_t* off, uint32_t wb, uint32_t m, uint32_t run, XYZZ<F>* R,
                  XYZZ<F>* T, XYZZ<F>* part, XYZZ<F>* scaled, XYZZ<F>* win)
{
    RedJob<F> j{};
    j.bsum = bsum; j.off = off; j.R = R; j.T = T; j.part = part; j.scaled = scaled; j.win = win;
    j.wb = wb; j.m = m;
    j.sh = red_shape(m, run);
    return j;
}

// The weighted sums of every job, four launches for all of them (in rounds
// of kMaxRedJobs jobs).  A job's win may alias its R.
template <class F>
int reduce_jobs(RedJob<F>* jv, size_t n, cudaStream_t st)
{
    for (size_t b = 0; b < n; b += kMaxRedJobs) {
        RedJobs<F> jobs{};
        jobs.count = (uint32_t)(n - b < kMaxRedJobs ? n - b : kMaxRedJobs);
        uint64_t tiles = 0, nps = 0, nss = 0, sets = 0;
        for (uint32_t i = 0; i < jobs.count; i++) {
            RedJob<F> j = jv[b + i];
            j.s_tile = tiles; j.s_np = nps; j.s_ns = nss; j.s_w = sets;
            tiles += (uint64_t)j.wb * j.sh.P;
            nps += (uint64_t)j.wb * j.sh.NP;
            nss += (uint64_t)j.wb * j.sh.NS;
            sets += j.wb;
            jobs.g[i] = j;
        }
        k_red_tile<F><<<grid_for(tiles * 32, 128), 128, 0, st>>>(jobs, tiles); note_launch();
        k_red_slices<F><<<grid_for(nps * 32, 128), 128, 0, st>>>(jobs, nps); note_launch();
        k_red_scale<F><<<grid_for(nss * 32, 128), 128, 0, st>>>(jobs, nss); note_launch();
        k_red_combine<F><<<grid_for(sets * 32, 128), 128, 0, st>>>(jobs, sets); note_launch();
        LZK_TRY(launch_status());
    }
    return LZK_OK;
}

// W_w of wb sets of m buckets (bsum / off indexed w m + k) into win[0..wb).
// Scratch: R, T, part, scaled of red_scratch_points(wb, m) points each.  win
// may alias R.
template <class F>
int reduce_buckets(const XYZZ<F>* bsum, const uint32_t* off, uint32_t wb, uint32_t m, XYZZ<F>* R, XYZZ<F>* T,
                   XYZZ<F>* part, XYZZ<F>* scaled, XYZZ<F>* win, cudaStream_t st, uint32_t run = kDefaultRun)
{
    RedJob<F> j = red_job<F>(bsum, off, wb, m, run, R, T, part, scaled, win);
    return reduce_jobs<F>(&j, 1, st);
}

// Horner over the bucket sets' weighted sums (plain bases), or the
// conversion of the one set's sum (shifted-copy table): one warp, with
// warp-uniform point operations.  Launched as <<<1, 32>>>.
template <class F>
__global__ void k_finish(const XYZZ<F>* __restrict__ win, uint32_t windows, uint32_t c, Jac<F>* out)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    XYZZ<F> r = xyzz_inf<F>();
    for (int w = (int)windows - 1; w >= 0; w--) {
        if (w != (int)windows - 1)
            for (uint32_t d = 0; d < c; d++) r = xyzz_dbl_warp(r);
        r = xyzz_add_warp(r, ld_elem(win + w));
    }
    Jac<F> j = xyzz_to_jac_warp(r);
    if (threadIdx.x == 0) st_elem(out, j);
}

template <class F>
__global__ void k_write_inf(Jac<F>* out)
{
    if (gtid() == 0) st_elem(out, Jac<F>{F::zero(), F::one(), F::zero()});
}

// pre_off / pre_ent: bucket offsets and sorted entries of these scalars made
// earlier by msm_sort for the same n, window width and table stride (MSMs
// over the same scalars share one sort); null = sort here.
template <class Gp>
int run_msm(const Fr* scalars, const void* bases, size_t n, Jac<typename Gp::F>* out,
                   const lzk_msm_cfg* cfg, cudaStream_t st, uint32_t c_auto,
                   const uint32_t* pre_off = nullptr, const uint32_t* pre_ent = nullptr)
{
    using F = typename Gp::F;
    using X = XYZZ<F>;
    if (!out || (n && (!scalars || !bases))) return LZK_EINVAL;
    if (n >= (1ull << 31)) return LZK_EINVAL;
    uint32_t flags = cfg ? cfg->flags : 0u;
    uint32_t layout = cfg ? cfg->base_layout : (uint32_t)LZK_BASES_AFFINE;
    uint32_t ref_layout = sizeof(F) == 32 ? LZK_BASES_REF_G1_JAC : LZK_BASES_REF_G2_LANES;
    if (layout != LZK_BASES_AFFINE && layout != ref_layout) return LZK_EINVAL;
    bool shared = (flags & LZK_MSM_PRECOMPUTED) != 0;
    uint32_t c = (cfg && cfg->window_bits) ? cfg->window_bits : c_auto;
    if (c < 2 || c > 24) return LZK_EINVAL;
    size_t stride = shared ? cfg->level_stride : 0;
    if (shared) {
        if (!cfg->window_bits) return LZK_EINVAL;
        if (cfg->precomp_windows < windows_for(c) || stride < n) return LZK_EINVAL;
        if ((size_t)windows_for(c) * stride >= (1ull << 31)) return LZK_EINVAL;
    }
    if (n == 0) {
        k_write_inf<F><<<1, 32, 0, st>>>(out); note_launch();
        return launch_status();
    }
    const int group = sizeof(F) == 32 ? 1 : 2;
    uint32_t chunk = msm_chunk(cfg, group, n), run = msm_run(cfg, group, n);
    if (!tune_valid(LZK_TUNE_MSM_CHUNK, chunk) || !tune_valid(LZK_TUNE_MSM_REDUCE_RUN, run)) return LZK_EINVAL;
    MsmPlan p;
    plan_msm<Gp>(p, n, c, shared, stride, chunk, run);
    void* tr_all = trace_begin(sizeof(F) == 32 ? "msm_g1" : "msm_g2", st);
    Scratch ws;
    LZK_TRY(ws.acquire(p.bytes, cfg ? cfg->workspace : nullptr, cfg ? cfg->workspace_bytes : 0, st));
    char* base = ws.base;
    uint32_t* cnt = reinterpret_cast<uint32_t*>(base + p.o_cnt);
    uint32_t* off_ws = reinterpret_cast<uint32_t*>(base + p.o_off);
    uint32_t* ent_ws = reinterpret_cast<uint32_t*>(base + p.o_ent);
    const uint32_t* off = pre_off ? pre_off : off_ws;
    const uint32_t* ent = pre_ent ? pre_ent : ent_ws;
    X* bsum = reinterpret_cast<X*>(base + p.o_bsum);
    X* head = reinterpret_cast<X*>(base + p.o_head);
    X* tail = reinterpret_cast<X*>(base + p.o_tail);
    X* lr[2] = {reinterpret_cast<X*>(base + p.o_lr0), reinterpret_cast<X*>(base + p.o_lr1)};
    X* la[2] = {reinterpret_cast<X*>(base + p.o_la0), reinterpret_cast<X*>(base + p.o_la1)};

    uint32_t* bsums = reinterpret_cast<uint32_t*>(base + p.o_scan);
    uint32_t* large = reinterpret_cast<uint32_t*>(base + p.o_large);
    if (!pre_off) {
        void* tr_sort = trace_begin(sizeof(F) == 32 ? "msm_g1_sort" : "msm_g2_sort", st);
        LZK_TRY(msm_sort(p, scalars, cnt, off_ws, ent_ws, bsums, st));
        trace_end(tr_sort, st);
    }
    void* tr = trace_begin(sizeof(F) == 32 ? "msm_g1_accumulate" : "msm_g2_accumulate", st);
    {
        unsigned g = grid_for(p.chunks, 128);
        // base records the entries may name: the whole table, or the n bases
        const uint64_t nbases = shared ? (uint64_t)cfg->precomp_windows * stride : (uint64_t)n;
        constexpr int REF = sizeof(F) == 32 ? (int)LZK_BASES_REF_G1_JAC : (int)LZK_BASES_REF_G2_LANES;
        if (layout == LZK_BASES_AFFINE) {
            k_accumulate<F, LZK_BASES_AFFINE><<<g, 128, 0, st>>>(bases, ent, off, p.B, p.chunks, p.chunk, nbases, bsum, head, tail); note_launch();
        } else {
            k_accumulate<F, REF><<<g, 128, 0, st>>>(bases, ent, off, p.B, p.chunks, p.chunk, nbases, bsum, head, tail); note_launch();
        }
    }
    trace_end(tr, st);
    void* tr_fix = trace_begin(sizeof(F) == 32 ? "msm_g1_fixup" : "msm_g2_fixup", st);
    LZK_CUDA(cudaMemsetAsync(large, 0, sizeof(uint32_t), st));
    k_fixup<F><<<grid_for(p.B, 256, sm_count() * 8), 256, 0, st>>>(off, p.B, p.chunk, p.chunks, bsum, head, tail, large); note_launch();
    {
        constexpr unsigned fx_threads = 32768 / sizeof(X);   // 32 KB of shared memory
        k_fixup_large<F><<<sm_count() * 2, fx_threads, fx_threads * sizeof(X), st>>>(off, p.chunk, bsum, head, tail, large); note_launch();
    }
    trace_end(tr_fix, st);
    LZK_TRY(launch_status());

    // weighted sums per bucket set
    void* tr_red = trace_begin(sizeof(F) == 32 ? "msm_g1_reduce" : "msm_g2_reduce", st);
    X* win = lr[0];
    LZK_TRY(reduce_buckets<F>(bsum, off, p.wb, p.nb, lr[0], la[0], lr[1], la[1], win, st, p.run));
    void* tr_fin = trace_begin(sizeof(F) == 32 ? "msm_g1_finish" : "msm_g2_finish", st);
    k_finish<F><<<1, 32, 0, st>>>(win, p.wb, c, out); note_launch();
    trace_end(tr_fin, st);
    trace_end(tr_red, st);
    trace_end(tr_all, st);
    return launch_status();
}

// ------------------------- precomputed shifted bases -------------------------
template <class F>
__global__ void k_precompute(const Aff<F>* __restrict__ bases, size_t n, uint32_t c, uint32_t windows,
                             Aff<F>* __restrict__ table, size_t stride)
{
    // windows are normalised in groups of G with one inversion per group
    constexpr int G = 8;
    for (uint64_t i = gtid(); i < n; i += gstride()) {
        Aff<F> P = ldg_elem(bases + i);
        st_elem(table + i, P);
        if (aff_is_inf(P)) {
            Aff<F> z{F::zero(), F::zero()};
            for (uint32_t j = 1; j < windows; j++) st_elem(table + (size_t)j * stride + i, z);
            continue;
        }
        XYZZ<F> cur = xyzz_from_aff(P);
        for (uint32_t j0 = 1; j0 < windows; j0 += G) {
            int cntg = (int)min((uint32_t)G, windows - j0);
            XYZZ<F> pts[G];
            F pre[G];
            F acc = F::one();
            for (int k = 0; k < cntg; k++) {
                for (uint32_t d = 0; d < c; d++) cur = xyzz_dbl_cold(cur);
                pts[k] = cur;
                acc = mul(acc, mul(cur.ZZ, cur.ZZZ));
                pre[k] = acc;
            }
            F inv = inverse(acc);
            for (int k = cntg - 1; k >= 0; k--) {
                F dinv = k ? mul(inv, pre[k - 1]) : inv;  // (ZZ_k ZZZ_k)^-1
                inv = mul(inv, mul(pts[k].ZZ, pts[k].ZZZ));
                // x = X / ZZ = X * ZZZ * dinv,  y = Y / ZZZ = Y * ZZ * dinv
                Aff<F> a{mul(mul(pts[k].X, dinv), pts[k].ZZZ), mul(mul(pts[k].Y, dinv), pts[k].ZZ)};
                st_elem(table + (size_t)(j0 + k) * stride + i, a);
            }
        }
    }
}

// Jacobian -> affine, 8 points per thread with one inversion
template <class F>
__global__ void k_jac_to_aff(const Jac<F>* __restrict__ in, Aff<F>* __restrict__ out, size_t n)
{
    constexpr int G = 8;
    for (uint64_t t = gtid(); t * G < n; t += gstride()) {
        size_t b = t * G;
        int cntp = (int)((n - b) < G ? (n - b) : G);
        F pre[G];
        F acc = F::one();
        for (int k = 0; k < cntp; k++) {
            Jac<F> J = ld_elem(in + b + k);
            if (!J.Z.is_zero()) acc = mul(acc, J.Z);
            pre[k] = acc;
        }
        F inv = inverse(acc);
        for (int k = cntp - 1; k >= 0; k--) {
            Jac<F> J = ld_elem(in + b + k);
            if (J.Z.is_zero()) { st_elem(out + b + k, Aff<F>{F::zero(), F::zero()}); continue; }
            F zi = k ? mul(inv, pre[k - 1]) : inv;
            inv = mul(inv, J.Z);
            F z2 = sqr(zi);
            st_elem(out + b + k, Aff<F>{mul(J.X, z2), mul(J.Y, mul(z2, zi))});
        }
    }
}

template <class F>
int run_precompute(const Aff<F>* bases, size_t n, uint32_t c, uint32_t windows, Aff<F>* table,
                          size_t stride, cudaStream_t st)
{
    if (!bases || !table || c < 2 || c > 24 || windows == 0 || windows > 256 || stride < n) return LZK_EINVAL;
    if (n == 0) return LZK_OK;
    k_precompute<F><<<grid_for(n, 64), 64, 0, st>>>(bases, n, c, windows, table, stride); note_launch();
    return launch_status();
}

}  // namespace lzk
