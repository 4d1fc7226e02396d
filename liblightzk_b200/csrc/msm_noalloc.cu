// msm_noalloc.cu -- a G1 MSM entry point that never allocates device memory.
//
// Some callers cannot let a library allocate on the GPU: services that hand
// all of a device's memory to their own allocator when they start (a
// cudaMalloc inside the library would then fail, or take memory their
// budget does not know about), and request paths with hard latency limits
// that must not wait on the allocator or fail with out-of-memory halfway
// through a request.  lzk_msm_g1_noalloc serves them: its scratch is the
// file-scope array below, which the CUDA runtime reserves on every GPU that
// loads this library, once, for as long as the process lives.
//
// Limits: at most LZK_MSM_NOALLOC_MAX_POINTS points, and the scratch the
// chosen window width needs must fit in LZK_MSM_NOALLOC_SCRATCH_BYTES; larger
// requests are refused with LZK_EINVAL before any work is queued.
//
// Every call on a device uses the same array.  The MSM zeroes the counters it
// relies on at the start of each call, so a call never sees the previous
// call's data; but two calls whose work overlaps on the GPU (different
// streams without ordering between them) would race on the array.  Order
// such calls, or use lzk_msm_g1 with separate workspaces.
//
// The device address of the array is looked up with cudaGetSymbolAddress the
// first time each device is used (the array's name in host code is only a
// stand-in and must never be handed to a kernel).  That first call per device
// should therefore come before any stream capture is begun.
#include "common.cuh"
#include <mutex>

namespace lzk {

static __device__ __align__(256) unsigned char g_msm_noalloc_scratch[LZK_MSM_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[64] = {nullptr};

// device address of the scratch array on the current device
static int noalloc_scratch(void** out)
{
    int dev = 0;
    LZK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return LZK_EUNSUPPORTED;
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_msm_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return LZK_EDEVICE;
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return LZK_OK;
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_msm_g1_noalloc(const lzk_fr_t* scalars, const lzk_g1_affine_t* bases, size_t n, lzk_g1_t* out,
                       uint32_t window_bits, void* stream)
{
    if (n > LZK_MSM_NOALLOC_MAX_POINTS) return LZK_EINVAL;
    lzk_msm_cfg cfg = {};
    cfg.window_bits = window_bits;
    size_t need = lzk_msm_workspace_bytes(1, n, &cfg);
    if (need > LZK_MSM_NOALLOC_SCRATCH_BYTES) return LZK_EINVAL;
    void* scratch = nullptr;
    LZK_TRY(noalloc_scratch(&scratch));
    cfg.workspace = scratch;
    cfg.workspace_bytes = LZK_MSM_NOALLOC_SCRATCH_BYTES;
    return lzk_msm_g1(scalars, bases, n, out, &cfg, stream);
}

}  // extern "C"
