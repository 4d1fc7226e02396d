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
// Set-up: the first call on each device (n = 0 is enough) prepares that
// device before doing its own work.  Under CUDA's lazy module loading (the
// default since CUDA 12.2) kernels are loaded, and their local memory is
// sized, only when first used, and either may need device memory; a
// process whose allocator takes the device's memory right after start-up
// would then see the first MSM fail.  So the set-up runs one MSM of a
// single zero scalar over an infinite base whose inputs, output and scratch
// all lie in the array, on the caller's stream: every kernel the entry point
// launches is then loaded and has run once.  Make that first call before
// the allocator reserves its memory and before beginning any stream capture.
// A cudaDeviceReset unloads everything again, and the set-up is not
// repeated after one.
//
// The device address of the array is looked up with cudaGetSymbolAddress on
// every call (the array's name in host code is only a stand-in and must
// never be handed to a kernel); once the module is loaded the lookup is a
// table read.
#include "common.cuh"
#include <mutex>

namespace lzk {

static __device__ __align__(256) unsigned char g_msm_noalloc_scratch[LZK_MSM_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static bool g_noalloc_ready[64] = {false};

// device address of the scratch array on the current device
static int noalloc_scratch(void** out, int* dev_out)
{
    int dev = 0;
    LZK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return LZK_EUNSUPPORTED;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_msm_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return LZK_EDEVICE;
    }
    *out = p;
    *dev_out = dev;
    return LZK_OK;
}

// One-time set-up of the current device (see the file comment): an MSM of
// n = 0 (the point-at-infinity path) and one of n = 1 with a zero scalar and
// an infinite base, everything carved from the scratch array.  The first
// kilobyte holds the inputs and outputs, the rest is the MSM's workspace.
static int noalloc_setup(char* scratch, int dev, cudaStream_t st)
{
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (g_noalloc_ready[dev]) return LZK_OK;
    constexpr size_t kIo = 1024;
    lzk_fr_t* s = reinterpret_cast<lzk_fr_t*>(scratch);
    lzk_g1_affine_t* b = reinterpret_cast<lzk_g1_affine_t*>(scratch + 256);
    lzk_g1_t* out = reinterpret_cast<lzk_g1_t*>(scratch + 512);
    LZK_CUDA(cudaMemsetAsync(scratch, 0, kIo, st));
    lzk_msm_cfg cfg = {};
    cfg.window_bits = 2;
    cfg.workspace = scratch + kIo;
    cfg.workspace_bytes = LZK_MSM_NOALLOC_SCRATCH_BYTES - kIo;
    LZK_TRY(lzk_msm_g1(s, b, 0, out, &cfg, st));
    LZK_TRY(lzk_msm_g1(s, b, 1, out, &cfg, st));
    g_noalloc_ready[dev] = true;
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
    int dev = 0;
    LZK_TRY(noalloc_scratch(&scratch, &dev));
    LZK_TRY(noalloc_setup(static_cast<char*>(scratch), dev, as_stream(stream)));
    cfg.workspace = scratch;
    cfg.workspace_bytes = LZK_MSM_NOALLOC_SCRATCH_BYTES;
    return lzk_msm_g1(scalars, bases, n, out, &cfg, stream);
}

}  // extern "C"
