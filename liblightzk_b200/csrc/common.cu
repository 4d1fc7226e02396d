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
        default: return "unknown status";
    }
}

const char* lzk_version(void) { return "liblzk_b200 0.1 (sm_100a)"; }

}  // extern "C"
