// batch.cu -- many MSMs and NTTs of uneven sizes as one plan.
//
// The reference runs one operator per call, each with its own allocations
// and launches (msm.cuh:210-247, poly.cuh:65-73).  A batch plan lays every
// MSM of the batch into one global bucket space and runs each MSM phase
// once for the whole batch:
//   gather bases -> digit count -> offset scan -> scatter -> accumulate
//   -> fix-up -> bucket reduction (one level chain per window width) ->
//   window combination (one warp per MSM)
// so 64 MSMs cost about the launches of one; with LZK_BATCH_PERSISTENT
// everything after the scatter is one persistent launch (below).  MSMs are ordered by window
// width so that the windows of equal width are contiguous and reduce
// together.  NTTs are grouped by (size, direction) and each group is one
// set of pass launches over a device table of pointers, on a second stream
// that overlaps the MSM phases.  Every buffer is allocated when the plan is
// made, so running a plan is launches only; the plan captures them into a
// CUDA graph on first use and replays the graph afterwards.
#include "msm.cuh"
#include "ntt.cuh"
#include <algorithm>
#include <atomic>
#include <map>
#include <vector>

struct BDesc {                 // per MSM, device side
    const lzk::Fr* scalars;
    const void* bases;
    uint64_t pts_off;          // first point in the gathered base array
    uint64_t n;
    uint64_t bucket_base;      // first bucket in the global bucket space
    uint64_t win_base;         // first window result in the window-result array
    void* out;
    uint64_t tab_off;          // fixed bases: first entry of this MSM's shifted-copy table
    uint32_t c, W, nb;
    uint32_t hw;               // window results the finish combines: W (plain bases) or 1 (table)
};

struct lzk_batch_plan {
    int group = 1;
    uint32_t flags = 0;                // LZK_BATCH_*
    bool fixed = false;                // LZK_BATCH_FIXED_BASES: shifted-copy tables built at creation
    bool persistent = false;           // LZK_BATCH_PERSISTENT: the MSM phases after the sort in one launch
    void* table = nullptr;             // their entries, all MSMs, table_pts points
    uint64_t table_pts = 0;
    size_t table_bytes = 0;
    std::vector<BDesc> msm;            // sorted by window width
    struct WGroup { uint32_t c; uint64_t bucket_base, windows; size_t largest; uint32_t run; uint64_t scratch_off; };
    std::vector<WGroup> wgroups;
    struct NGroup { uint32_t k; int dir; uint32_t count; lzk::Fr** ptrs; };
    std::vector<NGroup> ngroups;
    uint64_t total_pts = 0, total_buckets = 0, total_windows = 0, max_entries = 0, chunks = 0, lvl = 0;
    uint32_t chunk = 0, run = 0;       // accumulation chunk, reduction run (tuning table, at creation; the
                                       // width groups take their own runs)
    char* ws = nullptr;
    size_t ws_bytes = 0;
    BDesc* d_desc = nullptr;
    uint64_t* d_ptsoff = nullptr;
    uint32_t *cnt = nullptr, *off = nullptr, *ent = nullptr, *bsums = nullptr, *large = nullptr;
    uint32_t* bar = nullptr;           // persistent launch: barrier count, error word
    void *bases = nullptr, *bsum = nullptr, *head = nullptr, *tail = nullptr, *lr[2] = {nullptr, nullptr},
         *la[2] = {nullptr, nullptr}, *wres = nullptr;
    cudaStream_t s_ntt = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
};

namespace lzk {

__device__ __forceinline__ uint32_t find_msm(const uint64_t* ptsoff, uint32_t count, uint64_t i)
{
    uint32_t lo = 0, hi = count;   // largest k with ptsoff[k] <= i
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (ptsoff[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

template <class F>
__global__ void k_bgather(const BDesc* __restrict__ d, const uint64_t* __restrict__ ptsoff, uint32_t count,
                          uint64_t total, Aff<F>* __restrict__ dst)
{
    for (uint64_t i = gtid(); i < total; i += gstride()) {
        uint32_t k = find_msm(ptsoff, count, i);
        st_elem(dst + i, ldg_elem(reinterpret_cast<const Aff<F>*>(d[k].bases) + (i - d[k].pts_off)));
    }
}

// signed digits of every scalar of the batch (the recoding of msm_sort.cu)
__device__ __forceinline__ uint32_t bwindow_bits(const uint32_t s[8], uint32_t lo, uint32_t c)
{
    uint32_t w = lo >> 5, sh = lo & 31;
    if (w >= 8) return 0;
    uint64_t v = ((uint64_t)s[w] | ((uint64_t)(w + 1 < 8 ? s[w + 1] : 0u) << 32)) >> sh;
    return (uint32_t)v & ((1u << c) - 1u);
}

// With tables (shared = true) every window of an MSM lands in its one
// bucket set and an entry names the table copy of its window:
// tab_off + w n + i; with plain bases each window has its own set and an
// entry names the gathered base i.
template <bool SCATTER>
__global__ void k_bdigits(const BDesc* __restrict__ d, const uint64_t* __restrict__ ptsoff, uint32_t count,
                          uint64_t total, bool shared, const uint32_t* __restrict__ off, uint32_t* __restrict__ cnt,
                          uint32_t* __restrict__ ent)
{
    for (uint64_t i = gtid(); i < total; i += gstride()) {
        uint32_t k = find_msm(ptsoff, count, i);
        const BDesc& m = d[k];
        Fr sc = from_mont(ldg_elem(m.scalars + (i - m.pts_off)));
        uint32_t carry = 0, half = m.nb;
        for (uint32_t w = 0; w < m.W; w++) {
            uint32_t raw = bwindow_bits(sc.v, w * m.c, m.c) + carry;
            uint32_t a;
            bool neg;
            if (raw > half) { carry = 1; neg = true; a = (1u << m.c) - raw; }
            else { carry = 0; neg = false; a = raw; }
            if (!a) continue;
            uint32_t b = (uint32_t)(m.bucket_base + (shared ? 0 : (uint64_t)w * m.nb) + a - 1);
            if (SCATTER) {
                uint32_t slot = off[b] + atomicSub(cnt + b, 1u) - 1u;
                uint32_t idx = shared ? (uint32_t)(m.tab_off + (uint64_t)w * m.n + (i - m.pts_off)) : (uint32_t)i;
                ent[slot] = idx | (neg ? 0x80000000u : 0u);
            } else {
                atomicAdd(cnt + b, 1u);
            }
        }
    }
}

// Horner over each MSM's windows: one warp per MSM (<<<count, 32>>>) with
// warp-uniform point operations, so the chain of about W * c doublings costs
// one product per stage instead of a whole serial formula
template <class F>
__device__ __forceinline__ void bfinish_one(const BDesc* __restrict__ d, uint32_t k, const XYZZ<F>* __restrict__ wres)
{
    const BDesc& m = d[k];
    XYZZ<F> r = xyzz_inf<F>();
    if (m.n) {
        for (int w = (int)m.hw - 1; w >= 0; w--) {
            if (w != (int)m.hw - 1)
                for (uint32_t b = 0; b < m.c; b++) r = xyzz_dbl_warp(r);
            r = xyzz_add_warp(r, ld_elem(wres + m.win_base + w));
        }
    }
    Jac<F> j = xyzz_to_jac_warp(r);
    if ((threadIdx.x & 31) == 0) st_elem(reinterpret_cast<Jac<F>*>(m.out), j);
}
template <class F>
__global__ void k_bfinish(const BDesc* __restrict__ d, uint32_t count, const XYZZ<F>* __restrict__ wres)
{
    const uint32_t k = blockIdx.x;
    if (k >= count || threadIdx.x >= 32) return;
    bfinish_one<F>(d, k, wres);
}

// ---------------- persistent form (LZK_BATCH_PERSISTENT) ----------------
// The MSM phases after the digit sort -- accumulation, fix-up, the large
// buckets' fix-up, the four bucket-reduction steps and the window
// combination -- as one cooperative launch of exactly the blocks the device
// holds at once, each phase a grid-stride loop over its items (the bodies of
// the separate kernels), a grid-wide barrier between phases.  Barrier k
// waits for k * gridDim.x arrivals on bar[0]; a wait gives up after
// kBarPolls polls (about 2 s), sets bar[1] and returns false, and every
// block then leaves at its next barrier, so the kernel always ends; the
// host reads bar[1] after the run (LZK_ETIMEOUT).
constexpr uint32_t kBarPolls = 1u << 23;
// lzk_debug_persistent_barrier: extra arrivals every barrier waits for (so
// that, when nonzero, none is ever reached) and the poll limit
static std::atomic<uint32_t> g_persist_extra{0}, g_persist_polls{kBarPolls};

__device__ __forceinline__ bool persist_barrier(uint32_t* bar, uint32_t phase, uint32_t extra, uint32_t max_polls)
{
    __shared__ uint32_t ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        const uint32_t target = phase * gridDim.x + extra;
        uint32_t good = 1;
        for (uint32_t polls = 0;; polls++) {
            uint32_t v;
            asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if (v >= target) break;
            if (*(volatile uint32_t*)(bar + 1)) { good = 0; break; }
            if (polls >= max_polls) { atomicOr(bar + 1, 1u); good = 0; break; }
            __nanosleep(256);
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

template <class F>
struct PersistArgs {
    const void* bases;
    const uint32_t* ent;
    const uint32_t* off;
    uint32_t B, chunk;
    uint64_t chunks, nbases;
    XYZZ<F> *bsum, *head, *tail;
    uint32_t* large;
    uint32_t* bar;
    uint64_t tiles, nps, nss, sets;    // reduction items (as reduce_jobs counts them)
    const BDesc* desc;
    uint32_t count;                    // MSMs
    const XYZZ<F>* wres;
    uint32_t extra, polls;             // barrier arrivals beyond the grid (0; tests only) and poll limit
};

template <class F>
__global__ void __launch_bounds__(128, sizeof(F) == 32 ? 3 : 2)
k_bpersist(const __grid_constant__ PersistArgs<F> a, const __grid_constant__ RedJobs<F> jobs)
{
    __shared__ uint4 fx_raw[128 * sizeof(XYZZ<F>) / 16];
    for (uint64_t t = gtid(); t < a.chunks; t += gstride())
        accumulate_chunk<F, LZK_BASES_AFFINE>(t, a.bases, a.ent, a.off, a.B, a.chunks, a.chunk, a.nbases, a.bsum,
                                             a.head, a.tail);
    if (!persist_barrier(a.bar, 1, a.extra, a.polls)) return;
    fixup_items<F>(a.off, a.B, a.chunk, a.chunks, a.bsum, a.head, a.tail, a.large);
    if (!persist_barrier(a.bar, 2, a.extra, a.polls)) return;
    fixup_large_items<F>(a.off, a.chunk, a.bsum, a.head, a.tail, a.large, reinterpret_cast<XYZZ<F>*>(fx_raw));
    if (!persist_barrier(a.bar, 3, a.extra, a.polls)) return;
    red_tile_items<F>(jobs, a.tiles);
    if (!persist_barrier(a.bar, 4, a.extra, a.polls)) return;
    red_slices_items<F>(jobs, a.nps);
    if (!persist_barrier(a.bar, 5, a.extra, a.polls)) return;
    red_scale_items<F>(jobs, a.nss);
    if (!persist_barrier(a.bar, 6, a.extra, a.polls)) return;
    red_combine_items<F>(jobs, a.sets);
    if (!persist_barrier(a.bar, 7, a.extra, a.polls)) return;
    for (uint64_t k = gtid() >> 5; k < a.count; k += gstride() >> 5) bfinish_one<F>(a.desc, (uint32_t)k, a.wres);
}

// the reduction jobs of a plan, one per window width, laid out as
// reduce_jobs lays them (at most kMaxRedJobs: checked at creation)
template <class F>
static RedJobs<F> plan_jobs(lzk_batch_plan* p, uint64_t& tiles, uint64_t& nps, uint64_t& nss, uint64_t& sets)
{
    using X = XYZZ<F>;
    RedJobs<F> jobs{};
    tiles = nps = nss = sets = 0;
    uint64_t wdone = 0;
    X* bsum = static_cast<X*>(p->bsum);
    for (auto& wg : p->wgroups) {
        const uint64_t o = wg.scratch_off;
        RedJob<F> j = red_job<F>(bsum + wg.bucket_base, p->off + wg.bucket_base, (uint32_t)wg.windows,
                                 1u << (wg.c - 1), wg.run, static_cast<X*>(p->lr[0]) + o,
                                 static_cast<X*>(p->la[0]) + o, static_cast<X*>(p->lr[1]) + o,
                                 static_cast<X*>(p->la[1]) + o, static_cast<X*>(p->wres) + wdone);
        wdone += wg.windows;
        j.s_tile = tiles; j.s_np = nps; j.s_ns = nss; j.s_w = sets;
        tiles += (uint64_t)j.wb * j.sh.P;
        nps += (uint64_t)j.wb * j.sh.NP;
        nss += (uint64_t)j.wb * j.sh.NS;
        sets += j.wb;
        jobs.g[jobs.count++] = j;
    }
    return jobs;
}

template <class F>
static int run_persistent(lzk_batch_plan* p, cudaStream_t st)
{
    using X = XYZZ<F>;
    PersistArgs<F> a{};
    a.bases = p->fixed ? p->table : p->bases;
    a.ent = p->ent;
    a.off = p->off;
    a.B = (uint32_t)p->total_buckets;
    a.chunk = p->chunk;
    a.chunks = p->chunks;
    a.nbases = p->fixed ? p->table_pts : p->total_pts;
    a.bsum = static_cast<X*>(p->bsum);
    a.head = static_cast<X*>(p->head);
    a.tail = static_cast<X*>(p->tail);
    a.large = p->large;
    a.bar = p->bar;
    a.desc = p->d_desc;
    a.count = (uint32_t)p->msm.size();
    a.extra = g_persist_extra.load();
    a.polls = g_persist_polls.load();
    a.wres = static_cast<const X*>(p->wres);
    RedJobs<F> jobs = plan_jobs<F>(p, a.tiles, a.nps, a.nss, a.sets);
    int per_sm = 0;
    LZK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bpersist<F>, 128, 0));
    if (per_sm <= 0) return LZK_EUNSUPPORTED;
    LZK_CUDA(cudaMemsetAsync(p->large, 0, sizeof(uint32_t), st));
    LZK_CUDA(cudaMemsetAsync(p->bar, 0, 2 * sizeof(uint32_t), st));
    void* args[] = {&a, &jobs};
    LZK_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_bpersist<F>), dim3(sm_count() * per_sm),
                                         dim3(128), args, 0, st));
    note_launch();
    return launch_status();
}

template <class F>
static int run_plan(lzk_batch_plan* p, cudaStream_t st)
{
    using X = XYZZ<F>;
    uint32_t count = (uint32_t)p->msm.size();
    if (count && p->total_pts) {
        unsigned g = grid_for(p->total_pts, 256, sm_count() * 16);
        void* tr = trace_begin("batch_msm_sort", st);
        if (!p->fixed) {
            k_bgather<F><<<g, 256, 0, st>>>(p->d_desc, p->d_ptsoff, count, p->total_pts, static_cast<Aff<F>*>(p->bases)); note_launch();
        }
        LZK_CUDA(cudaMemsetAsync(p->cnt, 0, sizeof(uint32_t) * p->total_buckets, st));
        k_bdigits<false><<<g, 256, 0, st>>>(p->d_desc, p->d_ptsoff, count, p->total_pts, p->fixed, p->off, p->cnt, p->ent); note_launch();
        LZK_TRY(scan_offsets(p->cnt, (uint32_t)p->total_buckets, p->off, p->bsums, st));
        k_bdigits<true><<<g, 256, 0, st>>>(p->d_desc, p->d_ptsoff, count, p->total_pts, p->fixed, p->off, p->cnt, p->ent); note_launch();
        trace_end(tr, st);
        if (p->persistent) {
            tr = trace_begin("batch_msm_persistent", st);
            LZK_TRY(run_persistent<F>(p, st));
            trace_end(tr, st);
            return LZK_OK;
        }
        X* bsum = static_cast<X*>(p->bsum);
        tr = trace_begin("batch_msm_accumulate", st);
        k_accumulate<F, LZK_BASES_AFFINE><<<grid_for(p->chunks, 128), 128, 0, st>>>(
            p->fixed ? p->table : p->bases, p->ent, p->off, (uint32_t)p->total_buckets, p->chunks, p->chunk,
            p->fixed ? p->table_pts : p->total_pts, bsum, static_cast<X*>(p->head), static_cast<X*>(p->tail)); note_launch();
        trace_end(tr, st);
        tr = trace_begin("batch_msm_fixup", st);
        LZK_CUDA(cudaMemsetAsync(p->large, 0, sizeof(uint32_t), st));
        k_fixup<F><<<grid_for(p->total_buckets, 256, sm_count() * 8), 256, 0, st>>>(p->off, (uint32_t)p->total_buckets, p->chunk, p->chunks, bsum,
                                                                            static_cast<X*>(p->head),
                                                                            static_cast<X*>(p->tail), p->large); note_launch();
        constexpr unsigned fx_threads = 32768 / sizeof(X);
        k_fixup_large<F><<<sm_count() * 2, fx_threads, fx_threads * sizeof(X), st>>>(p->off, p->chunk, bsum, static_cast<X*>(p->head),
                                                                             static_cast<X*>(p->tail), p->large); note_launch();
        trace_end(tr, st);
        // the bucket reductions of all window widths, in the same four launches
        tr = trace_begin("batch_msm_reduce", st);
        std::vector<RedJob<F>> jobs;
        uint64_t wdone = 0;
        for (auto& wg : p->wgroups) {
            const uint64_t o = wg.scratch_off;
            jobs.push_back(red_job<F>(bsum + wg.bucket_base, p->off + wg.bucket_base, (uint32_t)wg.windows,
                                      1u << (wg.c - 1), wg.run, static_cast<X*>(p->lr[0]) + o,
                                      static_cast<X*>(p->la[0]) + o, static_cast<X*>(p->lr[1]) + o,
                                      static_cast<X*>(p->la[1]) + o, static_cast<X*>(p->wres) + wdone));
            wdone += wg.windows;
        }
        LZK_TRY(reduce_jobs<F>(jobs.data(), jobs.size(), st));
        trace_end(tr, st);
    }
    if (count && !(p->persistent && p->total_pts)) {
        void* tr = trace_begin("batch_msm_finish", st);
        k_bfinish<F><<<count, 32, 0, st>>>(p->d_desc, count, static_cast<const X*>(p->wres)); note_launch();
        trace_end(tr, st);
    }
    return launch_status();
}

static int run_all(lzk_batch_plan* p, cudaStream_t st)
{
    if (!p->ngroups.empty()) {
        LZK_CUDA(cudaEventRecord(p->ev_fork, st));
        LZK_CUDA(cudaStreamWaitEvent(p->s_ntt, p->ev_fork, 0));
        void* tr = trace_begin("batch_ntt", p->s_ntt);
        for (auto& g : p->ngroups) LZK_TRY(ntt_run(nullptr, g.k, g.dir, g.count, 0, nullptr, p->s_ntt, g.ptrs));
        trace_end(tr, p->s_ntt);
        LZK_CUDA(cudaEventRecord(p->ev_join, p->s_ntt));
    }
    LZK_TRY(p->group == 2 ? run_plan<Fq2>(p, st) : run_plan<Fq>(p, st));
    if (!p->ngroups.empty()) LZK_CUDA(cudaStreamWaitEvent(st, p->ev_join, 0));
    return LZK_OK;
}

static void destroy_plan(lzk_batch_plan* p)
{
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->ws) cudaFree(p->ws);
    if (p->table) cudaFree(p->table);
    for (auto& g : p->ngroups) if (g.ptrs) cudaFree(g.ptrs);
    if (p->s_ntt) cudaStreamDestroy(p->s_ntt);
    if (p->ev_fork) cudaEventDestroy(p->ev_fork);
    if (p->ev_join) cudaEventDestroy(p->ev_join);
    delete p;
}

template <class F>
static int create_plan(const lzk_msm_desc* msms, size_t n_msm, const lzk_ntt_desc* ntts, size_t n_ntt,
                       lzk_batch_plan* p)
{
    using X = XYZZ<F>;
    // MSMs: widths, ordering, global layout
    std::vector<size_t> order(n_msm);
    std::vector<uint32_t> cw(n_msm);
    for (size_t i = 0; i < n_msm; i++) {
        if (!msms[i].out || (msms[i].n && (!msms[i].scalars || !msms[i].bases))) return LZK_EINVAL;
        cw[i] = msms[i].window_bits ? msms[i].window_bits : msm_autotune(p->group, msms[i].n, p->fixed);
        if (cw[i] < 2 || cw[i] > 24) return LZK_EINVAL;
        order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cw[a] < cw[b]; });
    std::vector<uint64_t> ptsoff;
    for (size_t o : order) {
        const lzk_msm_desc& m = msms[o];
        BDesc d{};
        d.scalars = reinterpret_cast<const Fr*>(m.scalars);
        d.bases = m.bases;
        d.n = m.n;
        d.out = m.out;
        d.c = cw[o];
        d.W = windows_for(d.c);
        d.nb = 1u << (d.c - 1);
        d.pts_off = p->total_pts;
        d.bucket_base = p->total_buckets;
        d.win_base = p->total_windows;
        // plain bases: a bucket set per window, combined by Horner; tables:
        // one set for all windows
        d.hw = p->fixed ? 1 : d.W;
        d.tab_off = p->table_pts;
        if (p->fixed) p->table_pts += m.n * (uint64_t)d.W;
        p->total_pts += m.n;
        p->total_buckets += (uint64_t)d.hw * d.nb;
        p->total_windows += d.hw;
        p->max_entries += m.n * (uint64_t)d.W;
        if (p->wgroups.empty() || p->wgroups.back().c != d.c) p->wgroups.push_back({d.c, d.bucket_base, 0, 0, 0, 0});
        p->wgroups.back().windows += d.hw;
        p->wgroups.back().largest = std::max<size_t>(p->wgroups.back().largest, m.n);
        ptsoff.push_back(d.pts_off);
        p->msm.push_back(d);
    }
    if (p->total_pts >= (1ull << 31) || p->table_pts >= (1ull << 31) || p->total_buckets >= (1ull << 32) - 1 ||
        p->max_entries >= (1ull << 32))
        return LZK_EINVAL;
    // the plan's largest MSM picks the accumulation chunk and reduction run
    size_t largest = 0;
    for (size_t i = 0; i < n_msm; i++) largest = std::max(largest, msms[i].n);
    p->chunk = tune_chunk(p->group, largest, p->fixed);
    p->run = tune_run(p->group, largest, p->fixed);
    // each width group reduces with the run of its own largest MSM's size class
    for (auto& g : p->wgroups) g.run = tune_run(p->group, g.largest, p->fixed);
    p->chunks = (p->max_entries + p->chunk - 1) / p->chunk;
    // the persistent launch takes every width group's reduction job at once
    if (p->persistent && p->wgroups.size() > kMaxRedJobs) return LZK_EUNSUPPORTED;
    // every width group reduces in the same launches, each in its own slice
    // of the reduction scratch
    for (auto& g : p->wgroups) {
        g.scratch_off = p->lvl;
        p->lvl += red_scratch_points((uint32_t)g.windows, 1u << (g.c - 1));
    }
    uint64_t B = std::max<uint64_t>(p->total_buckets, 1);
    Carver cv;
    size_t o_desc = cv.take<BDesc>(std::max<size_t>(n_msm, 1));
    size_t o_ptsoff = cv.take<uint64_t>(std::max<size_t>(n_msm, 1));
    size_t o_cnt = cv.take<uint32_t>(B), o_off = cv.take<uint32_t>(B + 1);
    size_t o_bsums = cv.take<uint32_t>((B + 4095) / 4096 + 1);
    size_t o_large = cv.take<uint32_t>(p->chunks / kFixSmall + 2);
    size_t o_bar = cv.take<uint32_t>(2);
    size_t o_ent = cv.take<uint32_t>(std::max<uint64_t>(p->max_entries, 1));
    size_t o_bases = cv.take<Aff<F>>(p->fixed ? 1 : std::max<uint64_t>(p->total_pts, 1));
    size_t o_bsum = cv.take<X>(B);
    size_t o_head = cv.take<X>(std::max<uint64_t>(p->chunks, 1)), o_tail = cv.take<X>(std::max<uint64_t>(p->chunks, 1));
    size_t o_lr0 = cv.take<X>(std::max<uint64_t>(p->lvl, 1)), o_lr1 = cv.take<X>(std::max<uint64_t>(p->lvl, 1));
    size_t o_la0 = cv.take<X>(std::max<uint64_t>(p->lvl, 1)), o_la1 = cv.take<X>(std::max<uint64_t>(p->lvl, 1));
    size_t o_wres = cv.take<X>(std::max<uint64_t>(p->total_windows, 1));
    p->ws_bytes = cv.off;
    LZK_TRY(dev_malloc(reinterpret_cast<void**>(&p->ws), p->ws_bytes));
    char* b = p->ws;
    p->d_desc = reinterpret_cast<BDesc*>(b + o_desc);
    p->d_ptsoff = reinterpret_cast<uint64_t*>(b + o_ptsoff);
    p->cnt = reinterpret_cast<uint32_t*>(b + o_cnt);
    p->off = reinterpret_cast<uint32_t*>(b + o_off);
    p->bsums = reinterpret_cast<uint32_t*>(b + o_bsums);
    p->large = reinterpret_cast<uint32_t*>(b + o_large);
    p->bar = reinterpret_cast<uint32_t*>(b + o_bar);
    p->ent = reinterpret_cast<uint32_t*>(b + o_ent);
    p->bases = b + o_bases;
    p->bsum = b + o_bsum;
    p->head = b + o_head;
    p->tail = b + o_tail;
    p->lr[0] = b + o_lr0; p->lr[1] = b + o_lr1; p->la[0] = b + o_la0; p->la[1] = b + o_la1;
    p->wres = b + o_wres;
    if (n_msm) {
        LZK_CUDA(cudaMemcpy(p->d_desc, p->msm.data(), sizeof(BDesc) * n_msm, cudaMemcpyHostToDevice));
        LZK_CUDA(cudaMemcpy(p->d_ptsoff, ptsoff.data(), sizeof(uint64_t) * n_msm, cudaMemcpyHostToDevice));
    }
    if (p->fixed && p->table_pts) {
        // the shifted-copy table of every MSM, entry (w, i) at tab_off + w n + i
        p->table_bytes = p->table_pts * sizeof(Aff<F>);
        LZK_TRY(dev_malloc(&p->table, p->table_bytes));
        cudaStream_t st;
        LZK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        int rc = LZK_OK;
        for (const BDesc& d : p->msm) {
            if (!d.n || rc != LZK_OK) continue;
            rc = run_precompute<F>(static_cast<const Aff<F>*>(d.bases), d.n, d.c, d.W,
                                   static_cast<Aff<F>*>(p->table) + d.tab_off, d.n, st);
        }
        if (rc == LZK_OK) rc = cuda_status(cudaStreamSynchronize(st));
        cudaStreamDestroy(st);
        LZK_TRY(rc);
    }
    // NTTs: groups of equal (size, direction) with a device pointer table each
    std::map<std::pair<uint32_t, int>, std::vector<Fr*>> groups;
    for (size_t i = 0; i < n_ntt; i++) {
        if (!ntts[i].data || ntts[i].log_n > 26 || ntts[i].direction < 0 || ntts[i].direction > 3) return LZK_EINVAL;
        groups[{ntts[i].log_n, ntts[i].direction}].push_back(reinterpret_cast<Fr*>(ntts[i].data));
    }
    LZK_TRY(ntt_prepare_launch());
    for (auto& kv : groups) {
        NttTables t; CosetTables c;
        LZK_TRY(get_tables(kv.first.first, t, c));
        for (size_t s0 = 0; s0 < kv.second.size(); s0 += 65535) {
            size_t cnt = std::min<size_t>(65535, kv.second.size() - s0);
            lzk_batch_plan::NGroup g{kv.first.first, kv.first.second, (uint32_t)cnt, nullptr};
            LZK_TRY(dev_malloc(reinterpret_cast<void**>(&g.ptrs), sizeof(Fr*) * cnt));
            p->ngroups.push_back(g);
            LZK_CUDA(cudaMemcpy(g.ptrs, kv.second.data() + s0, sizeof(Fr*) * cnt, cudaMemcpyHostToDevice));
        }
    }
    LZK_CUDA(cudaStreamCreateWithFlags(&p->s_ntt, cudaStreamNonBlocking));
    LZK_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
    LZK_CUDA(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
    return LZK_OK;
}

uint32_t debug_word_batch(bool clear) { return debug_word_here(clear); }

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_batch_plan_create_ex(int group, const lzk_msm_desc* msms, size_t n_msm, const lzk_ntt_desc* ntts,
                             size_t n_ntt, uint32_t flags, lzk_batch_plan** out)
{
    if (!out || (group != 1 && group != 2) || (n_msm && !msms) || (n_ntt && !ntts)) return LZK_EINVAL;
    if (flags & ~(LZK_BATCH_FIXED_BASES | LZK_BATCH_PERSISTENT)) return LZK_EINVAL;
    *out = nullptr;
    lzk_batch_plan* p = new (std::nothrow) lzk_batch_plan();
    if (!p) return LZK_ENOMEM;
    p->group = group;
    p->flags = flags;
    p->fixed = (flags & LZK_BATCH_FIXED_BASES) != 0;
    p->persistent = (flags & LZK_BATCH_PERSISTENT) != 0;
    int rc = group == 2 ? create_plan<Fq2>(msms, n_msm, ntts, n_ntt, p) : create_plan<Fq>(msms, n_msm, ntts, n_ntt, p);
    if (rc != LZK_OK) { destroy_plan(p); return rc; }
    *out = p;
    return LZK_OK;
}

int lzk_batch_plan_create(int group, const lzk_msm_desc* msms, size_t n_msm, const lzk_ntt_desc* ntts, size_t n_ntt,
                          lzk_batch_plan** out)
{
    return lzk_batch_plan_create_ex(group, msms, n_msm, ntts, n_ntt, 0, out);
}

int lzk_batch_plan_run(lzk_batch_plan* p, int use_graph, void* stream)
{
    if (!p) return LZK_EINVAL;
    cudaStream_t st = as_stream(stream);
    if (p->persistent) {
        // eager, and synchronous: the run ends by reading the persistent
        // launch's barrier error word
        LZK_TRY(run_all(p, st));
        uint32_t err = 0;
        LZK_CUDA(cudaMemcpyAsync(&err, p->bar + 1, sizeof(err), cudaMemcpyDeviceToHost, st));
        LZK_CUDA(cudaStreamSynchronize(st));
        return err ? LZK_ETIMEOUT : LZK_OK;
    }
    if (!use_graph) return run_all(p, st);
    if (!st) return LZK_EINVAL;   // the legacy stream cannot be captured
    if (!p->exec) {
        LZK_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = run_all(p, st);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc != LZK_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc != LZK_OK ? rc : LZK_EDEVICE;
        }
        p->graph = g;
        LZK_CUDA(cudaGraphInstantiate(&p->exec, g, 0));
    }
    LZK_CUDA(cudaGraphLaunch(p->exec, st));
    return LZK_OK;
}

int lzk_debug_persistent_barrier(uint32_t extra_arrivals, uint32_t max_polls)
{
    g_persist_extra.store(extra_arrivals);
    g_persist_polls.store(max_polls ? max_polls : kBarPolls);
    return LZK_OK;
}

size_t lzk_batch_plan_device_bytes(const lzk_batch_plan* p) { return p ? p->ws_bytes + p->table_bytes : 0; }

int lzk_batch_plan_destroy(lzk_batch_plan* p)
{
    if (!p) return LZK_EINVAL;
    cudaDeviceSynchronize();
    destroy_plan(p);
    return LZK_OK;
}

}  // extern "C"
