// common.cu -- status strings, version, device memory-pool policy.
#include "common.cuh"
#include <atomic>
#include <mutex>

namespace lzk {

void keep_pool_cached()
{
    static std::mutex mu;
    static bool done[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return; }
    std::lock_guard<std::mutex> g(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    done[dev] = true;
}

// remaining allocations before the forced failures begin; -1 = none forced
static std::atomic<long long> g_fail_after{-1};

static bool alloc_forced_to_fail()
{
    long long v = g_fail_after.load();
    while (v >= 0) {
        if (v == 0) return true;
        if (g_fail_after.compare_exchange_weak(v, v - 1)) return false;
    }
    return false;
}

int dev_malloc(void** p, size_t bytes)
{
    *p = nullptr;
    if (alloc_forced_to_fail()) return LZK_ENOMEM;
    if (cudaMalloc(p, bytes ? bytes : 16) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return LZK_ENOMEM;
    }
    return LZK_OK;
}

int dev_malloc_async(void** p, size_t bytes, cudaStream_t st)
{
    *p = nullptr;
    if (alloc_forced_to_fail()) return LZK_ENOMEM;
    if (cudaMallocAsync(p, bytes ? bytes : 16, st) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return LZK_ENOMEM;
    }
    return LZK_OK;
}

unsigned sm_count()
{
    static std::atomic<unsigned> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return 128; }
    unsigned v = cached[dev].load(std::memory_order_relaxed);
    if (v) return v;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return 128;
    }
    cached[dev].store((unsigned)n, std::memory_order_relaxed);
    return (unsigned)n;
}

}  // namespace lzk

extern "C" {

const char* lzk_status_string(int status)
{
    switch (status) {
        case LZK_OK: return "ok";
        case LZK_EINVAL: return "invalid argument";
        case LZK_ENOMEM: return "device out of memory";
        case LZK_ETIMEOUT: return "bounded device wait timed out";
        case LZK_EDEVICE: return "CUDA runtime error";
        case LZK_EUNSUPPORTED: return "unsupported configuration";
        case LZK_EBUSY: return "busy (pending, or refused by the memory budget)";
        case LZK_ECANCELED: return "request cancelled";
        case LZK_EREJECTED: return "request can never fit the memory budget";
        case LZK_EIO: return "file cannot be read or written, or is not a valid key file";
        default: return "unknown status";
    }
}

uint32_t lzk_debug_check_word(int clear)
{
    bool c = clear != 0;
    return lzk::debug_word_sort(c) | lzk::debug_word_g1(c) | lzk::debug_word_g2(c) | lzk::debug_word_batch(c);
}

int lzk_debug_checks_enabled(void)
{
#ifdef LZK_DEBUG_CHECKS
    return 1;
#else
    return 0;
#endif
}

int lzk_debug_fail_allocations(long long after)
{
    lzk::g_fail_after.store(after < 0 ? -1 : after);
    return LZK_OK;
}

const char* lzk_version(void) { return "liblzk_b200 0.1 (sm_100a)"; }

}  // extern "C"
