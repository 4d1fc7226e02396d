// trace.cu -- opt-in CUDA-event tracing of named device regions, and the
// integer multiply-add throughput probe used as the roofline denominator.
//
// Tracing replaces the reference's wall-clock Timer + CUDA_DEBUG pairs
// (timer.cu:3-16, device-utils.cuh:3), which synchronise the device after
// every phase; here a traced region only records two events on its stream,
// and durations are resolved when the host asks for them.
#include "common.cuh"
#include "field52.cuh"
#include <nvtx3/nvToolsExt.h>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace lzk {

struct TraceRec {
    std::string name;
    cudaEvent_t a, b;
    nvtxRangeId_t nvtx = 0;   // NVTX range of the region's enqueue, 0 = none
    bool events = false;      // timing events recorded
};

struct TraceSpan {
    std::string name;
    double start_ms, end_ms;
};

static std::mutex g_tr_mu;
static bool g_tr_on = false;
// names recorded while tracing is on (empty: all); each traced region puts
// two timing events in its stream, a few microseconds of stream ordering,
// so a throughput measurement traces only the regions it reads
static std::vector<std::string> g_tr_only;
static std::vector<TraceRec> g_tr_pending;
static std::map<std::string, std::pair<double, uint64_t>> g_tr_sum;
// timeline: spans relative to the first region begun since the last reset
static cudaEvent_t g_tr_origin = nullptr;
static std::vector<TraceSpan> g_tr_spans;
constexpr size_t kMaxSpans = 1u << 16;

static std::atomic<unsigned long long> g_launches{0};
static std::atomic<bool> g_nvtx{false};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

bool trace_on() { return g_tr_on; }

void* trace_begin(const char* name, cudaStream_t st)
{
    bool ev = g_tr_on, nv = g_nvtx.load(std::memory_order_relaxed);
    if (!ev && !nv) return nullptr;
    if (ev) {
        std::lock_guard<std::mutex> g(g_tr_mu);
        if (!g_tr_only.empty()) {
            bool hit = false;
            for (const auto& n : g_tr_only) hit = hit || n == name;
            ev = hit;
        }
    }
    if (ev) {
        // no timing events inside a stream capture: the graph would keep
        // recording into events that are destroyed once resolved
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) { cudaGetLastError(); ev = false; }
        else if (cs != cudaStreamCaptureStatusNone) ev = false;
    }
    if (!ev && !nv) return nullptr;
    TraceRec* r = new TraceRec{name, nullptr, nullptr, 0, ev};
    if (nv) r->nvtx = nvtxRangeStartA(name);
    if (ev) {
        cudaEventCreate(&r->a);
        cudaEventCreate(&r->b);
        {
            std::lock_guard<std::mutex> g(g_tr_mu);
            if (!g_tr_origin && cudaEventCreate(&g_tr_origin) == cudaSuccess) cudaEventRecord(g_tr_origin, st);
        }
        cudaEventRecord(r->a, st);
    }
    return r;
}

void trace_end(void* h, cudaStream_t st)
{
    if (!h) return;
    TraceRec* r = static_cast<TraceRec*>(h);
    if (r->nvtx) nvtxRangeEnd(r->nvtx);
    if (r->events) {
        cudaEventRecord(r->b, st);
        std::lock_guard<std::mutex> g(g_tr_mu);
        g_tr_pending.push_back(*r);
    }
    delete r;
}

static void resolve()
{
    for (auto& r : g_tr_pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            auto& s = g_tr_sum[r.name];
            s.first += ms;
            s.second += 1;
            float t0 = 0.f, t1 = 0.f;
            if (g_tr_origin && g_tr_spans.size() < kMaxSpans &&
                cudaEventElapsedTime(&t0, g_tr_origin, r.a) == cudaSuccess &&
                cudaEventElapsedTime(&t1, g_tr_origin, r.b) == cudaSuccess)
                g_tr_spans.push_back(TraceSpan{r.name, t0, t1});
        }
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_tr_pending.clear();
    cudaGetLastError();
}

// Independent 32-bit multiply-add carry chains: each thread runs 8
// interleaved chains of mad.lo.cc / madc.hi.cc, the instruction mix of the
// Montgomery products.
__global__ void k_imad_probe(uint32_t iters, uint32_t seed, uint32_t* sink)
{
    uint32_t x[8], y = seed ^ threadIdx.x, acc = 0;
    for (int i = 0; i < 8; i++) x[i] = seed * (i + 3) + blockIdx.x;
    for (uint32_t it = 0; it < iters; it++) {
        #pragma unroll
        for (int i = 0; i < 8; i++) {
            asm volatile("mad.lo.cc.u32 %0, %0, %1, %0;\n\tmadc.hi.cc.u32 %0, %0, %1, %0;\n\t"
                         "madc.lo.cc.u32 %0, %0, %1, %0;\n\tmadc.hi.u32 %0, %0, %1, %0;"
                         : "+r"(x[i]) : "r"(y));
        }
    }
    for (int i = 0; i < 8; i++) acc ^= x[i];
    if (acc == 0x12345678u) sink[0] = acc;
}

// Independent Montgomery products, x_k <- x_k * y with kMontChains products
// in flight per thread, so the rate is bound by the product's instructions,
// not by a dependency chain.  FP: the radix-2^52 product on the FP64 pipe
// (mont52_core, operands kept as limbs between products: the fastest form
// this library has, the roofline's denominator); INT: the 32-bit-limb
// product (mul: wide integer multiplies, then the conditional subtraction).
constexpr int kMontChains = 4;
template <bool FP>
__device__ __forceinline__ void mont_probe_body(uint32_t iters, uint32_t seed, uint32_t* sink)
{
    Fq x[kMontChains], y;
    uint32_t h = seed * 0x9e3779b9u ^ (uint32_t)gtid();
    for (int i = 0; i < 8; i++) {
        h = h * 1664525u + 1013904223u;
        y.v[i] = h;
        for (int k = 0; k < kMontChains; k++) x[k].v[i] = h ^ (0x85ebca6bu * (k + 1));
    }
    y.v[7] &= 0x0fffffffu;                       // operands below p
    for (int k = 0; k < kMontChains; k++) x[k].v[7] &= 0x0fffffffu;
    uint32_t acc = 0;
    if (FP) {
        double dx[kMontChains][5], dy[5];
        to_d52<0>(dy, y.v);
        for (int k = 0; k < kMontChains; k++) to_d52<0>(dx[k], x[k].v);
        for (uint32_t it = 0; it < iters; it++) {
            #pragma unroll
            for (int k = 0; k < kMontChains; k++) {
                uint64_t r[5];
                mont52_core<FqP>(r, dx[k], dy);
                #pragma unroll
                for (int i = 0; i < 5; i++) dx[k][i] = u52_to_d(r[i]);   // r < 2p: limbs < 2^52
            }
        }
        for (int k = 0; k < kMontChains; k++)
            for (int i = 0; i < 5; i++) acc ^= (uint32_t)__double_as_longlong(dx[k][i]);
    } else {
        for (uint32_t it = 0; it < iters; it++) {
            #pragma unroll
            for (int k = 0; k < kMontChains; k++) x[k] = mul(x[k], y);
        }
        for (int k = 0; k < kMontChains; k++)
            for (int i = 0; i < 8; i++) acc ^= x[k].v[i];
    }
    if (acc == 0x12345678u) sink[0] = acc;
}
__global__ void __launch_bounds__(128) k_mont_probe_int(uint32_t iters, uint32_t seed, uint32_t* sink)
{
    mont_probe_body<false>(iters, seed, sink);
}
__global__ void __launch_bounds__(128, 2) k_mont_probe_fp(uint32_t iters, uint32_t seed, uint32_t* sink)
{
    mont_probe_body<true>(iters, seed, sink);
}

// Measured rate of Fq Montgomery products on this device at full
// occupancy, in the FP64 form (fp) or the 32-bit-limb form.  Synchronous;
// ~0.1 s.
template <bool FP>
static int probe_mont(double* products_per_s)
{
    if (!products_per_s) return LZK_EINVAL;
    int per_sm = 0;
    auto kern = FP ? k_mont_probe_fp : k_mont_probe_int;
    LZK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0));
    if (per_sm <= 0) return LZK_EDEVICE;
    uint32_t* sink;
    LZK_CUDA(cudaMalloc(&sink, 4));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const uint32_t iters = 2048, threads = 128, blocks = sm_count() * (uint32_t)per_sm * 4;
    kern<<<blocks, threads>>>(16, 1u, sink); note_launch();  // warm-up
    cudaEventRecord(a);
    kern<<<blocks, threads>>>(iters, 1u, sink); note_launch();
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_status(e);
    *products_per_s = (double)blocks * threads * iters * kMontChains / (ms * 1e-3);
    return LZK_OK;
}

}  // namespace lzk

using namespace lzk;

extern "C" {

uint64_t lzk_launch_count(void) { return g_launches.load(); }

void lzk_trace_nvtx(int on) { g_nvtx.store(on != 0); }

void lzk_trace_enable(int on)
{
    std::lock_guard<std::mutex> g(g_tr_mu);
    g_tr_on = on != 0;
}

int lzk_trace_only(const char* names)
{
    std::lock_guard<std::mutex> g(g_tr_mu);
    g_tr_only.clear();
    if (!names) return LZK_OK;
    std::string cur;
    for (const char* c = names;; c++) {
        if (*c == ',' || *c == 0) {
            if (!cur.empty()) g_tr_only.push_back(cur);
            cur.clear();
            if (*c == 0) break;
        } else {
            cur.push_back(*c);
        }
    }
    return LZK_OK;
}

void lzk_trace_reset(void)
{
    std::lock_guard<std::mutex> g(g_tr_mu);
    resolve();
    g_tr_sum.clear();
    g_tr_spans.clear();
    if (g_tr_origin) cudaEventDestroy(g_tr_origin);
    g_tr_origin = nullptr;
}

int lzk_trace_timeline(lzk_trace_span* spans, size_t cap, size_t* count)
{
    if (!count || (cap && !spans)) return LZK_EINVAL;
    std::lock_guard<std::mutex> g(g_tr_mu);
    resolve();
    *count = g_tr_spans.size();
    for (size_t i = 0; i < cap && i < g_tr_spans.size(); i++) {
        const TraceSpan& t = g_tr_spans[i];
        size_t k = 0;
        for (; k + 1 < sizeof(spans[i].name) && k < t.name.size(); k++) spans[i].name[k] = t.name[k];
        spans[i].name[k] = 0;
        spans[i].start_ms = t.start_ms;
        spans[i].end_ms = t.end_ms;
    }
    return LZK_OK;
}

int lzk_trace_get(const char* name, double* total_ms, uint64_t* count)
{
    if (!name || !total_ms || !count) return LZK_EINVAL;
    std::lock_guard<std::mutex> g(g_tr_mu);
    resolve();
    auto it = g_tr_sum.find(name);
    *total_ms = it == g_tr_sum.end() ? 0.0 : it->second.first;
    *count = it == g_tr_sum.end() ? 0 : it->second.second;
    return LZK_OK;
}

// Measured 32-bit integer multiply-add rate of this device (operations per
// second, one mad.lo/madc.hi = one operation).  Synchronous; ~0.1 s.
int lzk_probe_imad_rate(double* ops_per_s)
{
    if (!ops_per_s) return LZK_EINVAL;
    int dev, sms;
    LZK_CUDA(cudaGetDevice(&dev));
    LZK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint32_t* sink;
    LZK_CUDA(cudaMalloc(&sink, 4));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const uint32_t iters = 4096, threads = 256, blocks = (uint32_t)sms * 8;
    k_imad_probe<<<blocks, threads>>>(64, 1u, sink); note_launch();  // warm-up
    cudaEventRecord(a);
    k_imad_probe<<<blocks, threads>>>(iters, 1u, sink); note_launch();
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_status(e);
    double ops = (double)blocks * threads * iters * 8.0 * 4.0;
    *ops_per_s = ops / (ms * 1e-3);
    return LZK_OK;
}

int lzk_probe_mont_rate(double* products_per_s) { return probe_mont<true>(products_per_s); }
int lzk_probe_mont_rate_int(double* products_per_s) { return probe_mont<false>(products_per_s); }

}  // extern "C"
