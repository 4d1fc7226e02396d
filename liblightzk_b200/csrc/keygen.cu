// keygen.cu -- setup-path kernels: seeded uniform Fr vectors and fixed-base
// scalar multiplication k_i * G for G1 and G2.
//
// Replaces the reference's setup kernels fix_base_multi_scalar_multiplication
// _g1/_g2 (include/operator/msm.cuh:5-46, called from Groth16::Setup,
// groth16.cuh:88-126).  The reference's G2 kernel adds dest[] instead of the
// generator (msm.cuh:42), so its G2 keys are not k*G2; here both groups use
// their generator (alt_bn128_init.cu:130-132, 191-195).
//
// Fixed-base method: a comb table T[j][d] = d * 2^(8j) * G (j < 32,
// 1 <= d < 256, affine, built once per device) so that k*G is the sum of
// the 32 entries selected by the bytes of k -- 32 mixed XYZZ additions per
// scalar and no doublings; results are normalised to affine with one
// inversion per 8 points.
#include "keygen.cuh"
#include <map>
#include <mutex>

namespace lzk {

// ---------------- seeded uniform Fr ----------------
__device__ __forceinline__ uint64_t splitmix(uint64_t& s)
{
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Element i of stream (seed, sid): SplitMix64 seeded from (seed, sid, i);
// 254-bit candidates with rejection of values >= r, as
// Fp_model::random_element does (fp.cuh:789-816).  The candidate is used as
// the Montgomery representation.  After 64 rejections (probability < 2^-130)
// the candidate minus r is taken (< r because 2^254 < 2r).
__global__ void k_random_fr(uint64_t seed, uint64_t sid, uint64_t offset, size_t n, Fr* __restrict__ out)
{
    for (uint64_t i = gtid(); i < n; i += gstride()) {
        uint64_t s = seed * 0xd1342543de82ef95ull ^ (sid + 1) * 0x9e3779b97f4a7c15ull ^ (offset + i) * 0xc2b2ae3d27d4eb4full;
        splitmix(s);
        Fr v;
        bool ok = false;
        for (int tries = 0; tries < 64 && !ok; tries++) {
            uint64_t w[4];
            for (int k = 0; k < 4; k++) w[k] = splitmix(s);
            w[3] &= 0x3fffffffffffffffull;
            for (int k = 0; k < 4; k++) { v.v[2 * k] = (uint32_t)w[k]; v.v[2 * k + 1] = (uint32_t)(w[k] >> 32); }
            // v < r ?
            bool lt = false, decided = false;
            for (int k = 7; k >= 0 && !decided; k--) {
                if (v.v[k] != FrP::p(k)) { lt = v.v[k] < FrP::p(k); decided = true; }
            }
            ok = decided && lt;
        }
        if (!ok) {
            Fr r;
            _Pragma("unroll") for (int k = 0; k < 8; k++) r.v[k] = FrP::p(k);
            uint32_t br;
            asm("sub.cc.u32 %0, %0, %9;\n\tsubc.cc.u32 %1, %1, %10;\n\tsubc.cc.u32 %2, %2, %11;\n\t"
                "subc.cc.u32 %3, %3, %12;\n\tsubc.cc.u32 %4, %4, %13;\n\tsubc.cc.u32 %5, %5, %14;\n\t"
                "subc.cc.u32 %6, %6, %15;\n\tsubc.cc.u32 %7, %7, %16;\n\tsubc.u32 %8, 0, 0;"
                : "+r"(v.v[0]), "+r"(v.v[1]), "+r"(v.v[2]), "+r"(v.v[3]), "+r"(v.v[4]), "+r"(v.v[5]), "+r"(v.v[6]),
                  "+r"(v.v[7]), "=r"(br)
                : "r"(r.v[0]), "r"(r.v[1]), "r"(r.v[2]), "r"(r.v[3]), "r"(r.v[4]), "r"(r.v[5]), "r"(r.v[6]), "r"(r.v[7]));
            (void)br;
        }
        st_elem(out + i, v);
    }
}

// ---------------- generators ----------------
template <class F> __device__ Aff<F> generator();
template <> __device__ Aff<Fq> generator<Fq>()
{
    Fq one = Fq::one();
    return {one, add(one, one)};  // (1, 2)
}
template <> __device__ Aff<Fq2> generator<Fq2>()
{
    // Montgomery form of the G2 generator of alt_bn128_init.cu:191-195
    Fq x0{{0x02bc2026u, 0x8e83b5d1u, 0x497b0172u, 0xdceb1935u, 0x97811adfu, 0xfbb82647u, 0xaf96503bu, 0x19573841u}};
    Fq x1{{0xa84c6140u, 0xafb4737du, 0x5802d8c4u, 0x6043dd5au, 0x52a02f86u, 0x09e950fcu, 0x3aea7b6bu, 0x14fef083u}};
    Fq y0{{0x886be9f6u, 0x619dfa9du, 0xf59e9b78u, 0xfe7fd297u, 0x231b7dfeu, 0xff9e1a62u, 0xae9e4206u, 0x28fd7eebu}};
    Fq y1{{0xc71856eeu, 0x64095b56u, 0x327d3cbbu, 0xdc57f922u, 0x33351076u, 0x55f935beu, 0x93fd6482u, 0x0da4a0e6u}};
    return {Fq2{x0, x1}, Fq2{y0, y1}};
}

// base_j = 2^(8j) P for j < 32 (one thread, 248 doublings); P = the
// generator when base is null
template <class F>
__global__ void k_comb_bases(const Aff<F>* __restrict__ base, XYZZ<F>* __restrict__ bases)
{
    if (gtid() != 0) return;
    XYZZ<F> b = xyzz_from_aff(base ? *base : generator<F>());
    for (int j = 0; j < 32; j++) {
        st_elem(bases + j, b);
        for (int d = 0; d < 8; d++) b = xyzz_dbl_cold(b);
    }
}

// tmp[j*256 + d] = d * base_j (d = 0 gives infinity)
template <class F>
__global__ void k_comb_fill(const XYZZ<F>* __restrict__ bases, XYZZ<F>* __restrict__ tmp)
{
    for (uint64_t t = gtid(); t < 32 * 256; t += gstride()) {
        uint32_t j = (uint32_t)(t >> 8), d = (uint32_t)(t & 255);
        XYZZ<F> b = ld_elem(bases + j), acc = xyzz_inf<F>();
        for (int bit = 7; bit >= 0; bit--) {
            acc = xyzz_dbl_cold(acc);
            if ((d >> bit) & 1) acc = xyzz_add_cold(acc, b);
        }
        st_elem(tmp + t, acc);
    }
}

// XYZZ -> affine, G points per thread with one inversion:
// with D = ZZ*ZZZ, x = X*ZZZ/D, y = Y*ZZ/D.
template <class F>
__global__ void k_xyzz_to_aff(const XYZZ<F>* __restrict__ in, Aff<F>* __restrict__ out, size_t n)
{
    constexpr int G = 8;
    for (uint64_t t = gtid(); t * G < n; t += gstride()) {
        size_t b = t * G;
        int cnt = (int)((n - b) < G ? (n - b) : G);
        F pre[G];
        F acc = F::one();
        for (int k = 0; k < cnt; k++) {
            XYZZ<F> p = ld_elem(in + b + k);
            if (!xyzz_is_inf(p)) acc = mul(acc, mul(p.ZZ, p.ZZZ));
            pre[k] = acc;
        }
        F inv = inverse(acc);
        for (int k = cnt - 1; k >= 0; k--) {
            XYZZ<F> p = ld_elem(in + b + k);
            if (xyzz_is_inf(p)) { st_elem(out + b + k, Aff<F>{F::zero(), F::zero()}); continue; }
            F dinv = k ? mul(inv, pre[k - 1]) : inv;
            inv = mul(inv, mul(p.ZZ, p.ZZZ));
            st_elem(out + b + k, Aff<F>{mul(mul(p.X, p.ZZZ), dinv), mul(mul(p.Y, p.ZZ), dinv)});
        }
    }
}

// out_xyzz[i] = k_i * G from the comb table
template <class F>
__global__ void __launch_bounds__(128) k_fixed_base(const Fr* __restrict__ k, size_t n, const Aff<F>* __restrict__ T,
                                                     XYZZ<F>* __restrict__ out)
{
    for (uint64_t i = gtid(); i < n; i += gstride()) st_elem(out + i, comb_mul(T, from_mont(ldg_elem(k + i))));
}

template <class F>
int comb_build(const Aff<F>* base, Aff<F>* T, cudaStream_t st)
{
    Scratch ws;
    LZK_TRY(ws.acquire((32 * 256 + 32) * sizeof(XYZZ<F>), nullptr, 0, st));
    XYZZ<F>* tmp = reinterpret_cast<XYZZ<F>*>(ws.base);
    k_comb_bases<F><<<1, 32, 0, st>>>(base, tmp + 32 * 256); note_launch();
    k_comb_fill<F><<<64, 128, 0, st>>>(tmp + 32 * 256, tmp); note_launch();
    k_xyzz_to_aff<F><<<grid_for(32 * 256 / 8, 128), 128, 0, st>>>(tmp, T, 32 * 256); note_launch();
    return launch_status();
}
template int comb_build<Fq>(const Aff<Fq>*, Aff<Fq>*, cudaStream_t);
template int comb_build<Fq2>(const Aff<Fq2>*, Aff<Fq2>*, cudaStream_t);

static std::mutex g_comb_mu;
static std::map<int, void*> g_comb[3];

template <class F>
static int comb_table(const Aff<F>** out, int group)
{
    int dev;
    LZK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(g_comb_mu);
    auto it = g_comb[group].find(dev);
    if (it != g_comb[group].end()) { *out = static_cast<const Aff<F>*>(it->second); return LZK_OK; }
    Aff<F>* T = nullptr;
    LZK_TRY(dev_malloc(reinterpret_cast<void**>(&T), 32 * 256 * sizeof(Aff<F>)));
    cudaStream_t st;
    cudaError_t se = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (se != cudaSuccess) { cudaFree(T); return cuda_status(se); }
    int rc = comb_build<F>(nullptr, T, st);
    if (rc == LZK_OK) rc = cuda_status(cudaStreamSynchronize(st));
    cudaStreamDestroy(st);
    if (rc != LZK_OK) { cudaFree(T); return rc; }
    g_comb[group][dev] = T;
    *out = T;
    return LZK_OK;
}

template <class F>
static int fixed_base(const Fr* k, size_t n, Aff<F>* out, int group, cudaStream_t st)
{
    if (!n) return LZK_OK;
    if (!k || !out) return LZK_EINVAL;
    const Aff<F>* T;
    LZK_TRY(comb_table<F>(&T, group));
    Scratch ws;
    LZK_TRY(ws.acquire(n * sizeof(XYZZ<F>), nullptr, 0, st));
    XYZZ<F>* tmp = reinterpret_cast<XYZZ<F>*>(ws.base);
    k_fixed_base<F><<<grid_for(n, 128), 128, 0, st>>>(k, n, T, tmp); note_launch();
    k_xyzz_to_aff<F><<<grid_for((n + 7) / 8, 128), 128, 0, st>>>(tmp, out, n); note_launch();
    return launch_status();
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_random_fr(uint64_t seed, uint64_t stream_id, uint64_t offset, size_t n, lzk_fr_t* out, void* stream)
{
    if (!n) return LZK_OK;
    if (!out) return LZK_EINVAL;
    k_random_fr<<<grid_for(n, 256, sm_count() * 16), 256, 0, as_stream(stream)>>>(seed, stream_id, offset, n,
                                                                         reinterpret_cast<Fr*>(out)); note_launch();
    return launch_status();
}

int lzk_g1_fixed_base(const lzk_fr_t* k, size_t n, lzk_g1_affine_t* out, void* stream)
{
    return fixed_base<Fq>(reinterpret_cast<const Fr*>(k), n, reinterpret_cast<Aff<Fq>*>(out), 1, as_stream(stream));
}

int lzk_g2_fixed_base(const lzk_fr_t* k, size_t n, lzk_g2_affine_t* out, void* stream)
{
    return fixed_base<Fq2>(reinterpret_cast<const Fr*>(k), n, reinterpret_cast<Aff<Fq2>*>(out), 2, as_stream(stream));
}

}  // extern "C"
