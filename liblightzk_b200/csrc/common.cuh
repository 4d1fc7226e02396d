// common.cuh -- status handling, stream-ordered scratch and small device
// helpers shared by every translation unit of liblzk_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include "lzk.h"

namespace lzk {

#define LZK_TRY(expr)                                   \
    do {                                                \
        int _st = (expr);                               \
        if (_st != LZK_OK) return _st;                  \
    } while (0)

#define LZK_CUDA(expr)                                  \
    do {                                                \
        cudaError_t _e = (expr);                        \
        if (_e != cudaSuccess) return ::lzk::cuda_status(_e); \
    } while (0)

inline int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return LZK_OK;
    if (e == cudaErrorMemoryAllocation) return LZK_ENOMEM;
    return LZK_EDEVICE;
}

// Launch-error check after a kernel: sticky and non-sticky errors both map
// to LZK_EDEVICE, allocation failures to LZK_ENOMEM.
inline int launch_status() { return cuda_status(cudaGetLastError()); }

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// Count of kernel launches this library has enqueued (trace.cu); every
// launch site is followed by note_launch().
void note_launch();

// Opt-in event tracing of named device regions (trace.cu): a no-op returning
// nullptr unless lzk_trace_enable(1) was called.
bool trace_on();
void* trace_begin(const char* name, cudaStream_t st);
void trace_end(void* h, cudaStream_t st);

// Make the current device's default memory pool keep freed blocks, so the
// stream-ordered scratch of repeated calls is served from the pool.
void keep_pool_cached();

// Every device allocation of the library goes through these two: cudaMalloc
// and stream-ordered cudaMallocAsync, LZK_OK or LZK_ENOMEM (the CUDA error
// cleared).  lzk_debug_fail_allocations makes them fail on demand, so the
// clean-up of every create path can be tested without running out of memory.
int dev_malloc(void** p, size_t bytes);
int dev_malloc_async(void** p, size_t bytes, cudaStream_t st);

// Streaming multiprocessors of the current device (queried once per device
// and cached); grid-stride kernels size their grids in multiples of it.
unsigned sm_count();

// Scratch carved from a caller buffer or allocated stream-ordered from the
// device pool (cudaMallocAsync / cudaFreeAsync on the same stream).
struct Scratch {
    char* base = nullptr;
    size_t size = 0;
    bool owned = false;
    cudaStream_t st = nullptr;

    int acquire(size_t need, void* user, size_t user_bytes, cudaStream_t stream)
    {
        st = stream;
        size = need;
        if (user) {
            if (user_bytes < need) return LZK_EINVAL;
            base = static_cast<char*>(user);
            return LZK_OK;
        }
        if (need == 0) return LZK_OK;
        keep_pool_cached();
        if (dev_malloc_async(reinterpret_cast<void**>(&base), need, stream) != LZK_OK) { base = nullptr; return LZK_ENOMEM; }
        owned = true;
        return LZK_OK;
    }
    ~Scratch()
    {
        if (owned && base) cudaFreeAsync(base, st);
    }
};

// Sequential carve-out of aligned sub-buffers.
struct Carver {
    size_t off = 0;
    template <class T> size_t take(size_t count) { size_t o = off; off = align_up(off + count * sizeof(T)); return o; }
};

// Debug builds (compiled with -DLZK_DEBUG_CHECKS, see build.py --debug):
// kernels check the indices their inputs imply before they use them and,
// where one is out of range, set a bit of a device error word and skip the
// access instead of reading or writing outside their buffers.  The word is
// read with lzk_debug_check_word().  Release builds compile the checks away
// (LZK_CHECK is then always true and costs nothing).
//   bit 0  a digit's bucket index beyond the bucket count (sort)
//   bit 1  a scatter slot outside its bucket's range (sort)
//   bit 2  a sorted entry naming a base beyond the table (accumulation)
//   bit 3  a bucket offset read beyond the offsets array (accumulation)
//   bit 4  a fix-up partial beyond the chunk count (fix-up)
#ifdef LZK_DEBUG_CHECKS
static __device__ uint32_t g_lzk_debug_word;
#define LZK_CHECK(cond, bit) ((cond) ? true : (atomicOr(&g_lzk_debug_word, 1u << (bit)), false))
// host side: this file's error word (cleared when clear is set)
static inline uint32_t debug_word_here(bool clear)
{
    uint32_t v = 0;
    if (cudaMemcpyFromSymbol(&v, g_lzk_debug_word, sizeof(v)) != cudaSuccess) { cudaGetLastError(); return 0; }
    if (clear) {
        uint32_t z = 0;
        if (cudaMemcpyToSymbol(g_lzk_debug_word, &z, sizeof(z)) != cudaSuccess) cudaGetLastError();
    }
    return v;
}
#else
#define LZK_CHECK(cond, bit) true
static inline uint32_t debug_word_here(bool) { return 0; }
#endif
// the error words of the files whose kernels check (msm_sort.cu, msm_g1.cu,
// msm_g2.cu, batch.cu)
uint32_t debug_word_sort(bool clear);
uint32_t debug_word_g1(bool clear);
uint32_t debug_word_g2(bool clear);
uint32_t debug_word_batch(bool clear);

__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

inline unsigned grid_for(size_t threads, unsigned block, unsigned cap = 1u << 20)
{
    size_t g = (threads + block - 1) / block;
    if (g == 0) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

// 32-byte vector load/store of an 8-limb element through the read-only path
template <class T>
__device__ __forceinline__ T ldg_elem(const T* p)
{
    static_assert(sizeof(T) % 16 == 0, "16-byte multiple");
    T r;
    const uint4* s = reinterpret_cast<const uint4*>(p);
    uint4* d = reinterpret_cast<uint4*>(&r);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = __ldg(s + i);
    return r;
}
template <class T>
__device__ __forceinline__ void st_elem(T* p, const T& v)
{
    uint4* d = reinterpret_cast<uint4*>(p);
    const uint4* s = reinterpret_cast<const uint4*>(&v);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = s[i];
}
template <class T>
__device__ __forceinline__ T ld_elem(const T* p)
{
    T r;
    const uint4* s = reinterpret_cast<const uint4*>(p);
    uint4* d = reinterpret_cast<uint4*>(&r);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = s[i];
    return r;
}

}  // namespace lzk
