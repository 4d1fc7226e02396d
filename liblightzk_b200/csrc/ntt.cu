// ntt.cu -- number-theoretic transforms over BN254 Fr.
//
// Replaces number_theory_transformation and its kernels (reference
// include/operator/poly.cuh:32-73): same transform, X_k = sum_j a_j w^(jk)
// in natural order with w the 2^k-th root of unity of ntt-params.cuh
// (w_k = w_28^(2^(28-k)), w_28 = 5^((r-1)/2^28)), and the same radix-2
// decimation-in-frequency butterfly c[j] = lo + hi, c[j^h] = (lo - hi) *
// w^((j mod h) << s).  Instead of one global-memory launch per stage, each
// pass loads 2^m-element groups into shared memory and runs m stages there
// (ceil(k / 11) passes for a size-2^k transform); a final pass applies the
// bit-reversal permutation in place together with the scale n^-1 and the
// coset factor.
//
// Directions: forward; inverse (w^-1, then * n^-1); coset forward (a_j *
// g^j first, g = 5 = Fr::multiplicative_generator, alt_bn128_init.cu:50);
// coset inverse (inverse, then * g^-j).
#include "ntt.cuh"
#include "tune.cuh"
#include <map>
#include <mutex>

namespace lzk {

constexpr int kNttMaxLog = 26;
constexpr uint32_t kNttThreads = 256;
constexpr uint32_t kPowLoBits = 12;    // g^j = lo[j & 4095] * hi[j >> 12]

// Montgomery form of w_28 = 5^((r-1)/2^28) and of g = 5
__device__ __forceinline__ Fr root28()
{
    return Fr{{0x80d13d9cu, 0x636e7355u, 0x2445ffd6u, 0xa22bf374u, 0x1eb203d8u, 0x56452ac0u, 0x2963f9e7u, 0x1860ef94u}};
}
__device__ __forceinline__ Fr gen5()
{
    return Fr{{0x9fffffe6u, 0x1b0d0ef9u, 0xa32a913fu, 0xeaba68a3u, 0xd8dd0689u, 0x47d8eb76u, 0x20f5bbc3u, 0x15d00855u}};
}

__device__ __forceinline__ Fr fr_pow(Fr b, uint64_t e)
{
    Fr r = Fr::one();
    while (e) {
        if (e & 1) r = mul(r, b);
        b = sqr(b);
        e >>= 1;
    }
    return r;
}

// consts[0] = w_k, [1] = w_k^-1, [2] = 2^-k, [3] = g, [4] = g^-1,
// [5] = g^(2^12), [6] = g^-(2^12)
__global__ void k_ntt_consts(uint32_t k, Fr* consts)
{
    if (gtid() != 0) return;
    Fr w = root28();
    for (uint32_t i = k; i < 28; i++) w = sqr(w);
    consts[0] = w;
    consts[1] = inverse(w);
    Fr two = add(Fr::one(), Fr::one());
    consts[2] = inverse(fr_pow(two, k));
    Fr g = gen5();
    consts[3] = g;
    consts[4] = inverse(g);
    consts[5] = fr_pow(g, 1ull << kPowLoBits);
    consts[6] = fr_pow(consts[4], 1ull << kPowLoBits);
}

// out[i] = base^i for i < count (64 consecutive powers per thread)
__global__ void k_powers(const Fr* __restrict__ basep, Fr* __restrict__ out, size_t count)
{
    const uint32_t C = 64;
    Fr base = *basep;
    for (uint64_t t = gtid(); t * C < count; t += gstride()) {
        size_t s = t * C;
        Fr v = fr_pow(base, s);
        size_t e = s + C < count ? s + C : count;
        for (size_t i = s; i < e; i++) { st_elem(out + i, v); v = mul(v, base); }
    }
}

// twiddles in radix-2^52 form: twd[kTwdStride e + i] = limb i of tw[e]
__global__ void k_tw_to_d52(const Fr* __restrict__ tw, double* __restrict__ twd, size_t count)
{
    for (uint64_t e = gtid(); e < count; e += gstride()) {
        double d[5];
        to_d52<0>(d, ldg_elem(tw + e).v);
        double* o = twd + e * kTwdStride;
        _Pragma("unroll") for (int i = 0; i < 5; i++) o[i] = d[i];
        o[5] = 0.0;
    }
}

static std::mutex g_ntt_mu;
static std::map<std::pair<int, uint32_t>, NttTables> g_ntt_tables;
static std::map<int, CosetTables> g_coset_tables;

// Build (once per device and size, synchronously, outside any stream
// capture) the twiddle tables of a size-2^k transform.
int get_tables(uint32_t k, NttTables& out, CosetTables& cos)
{
    int dev;
    LZK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(g_ntt_mu);
    auto it = g_ntt_tables.find({dev, k});
    auto ct = g_coset_tables.find(dev);
    if (it != g_ntt_tables.end() && ct != g_coset_tables.end()) { out = it->second; cos = ct->second; return LZK_OK; }
    cudaStream_t st;
    LZK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int rc = LZK_OK;
    if (it == g_ntt_tables.end()) {
        NttTables t;
        size_t half = k ? (size_t(1) << (k - 1)) : 1;
        if (dev_malloc(reinterpret_cast<void**>(&t.consts), 8 * sizeof(Fr)) != LZK_OK ||
            dev_malloc(reinterpret_cast<void**>(&t.tw[0]), half * sizeof(Fr)) != LZK_OK ||
            dev_malloc(reinterpret_cast<void**>(&t.tw[1]), half * sizeof(Fr)) != LZK_OK ||
            dev_malloc(reinterpret_cast<void**>(&t.twd[0]), half * kTwdStride * sizeof(double)) != LZK_OK ||
            dev_malloc(reinterpret_cast<void**>(&t.twd[1]), half * kTwdStride * sizeof(double)) != LZK_OK) {
            cudaFree(t.consts);
            cudaFree(t.tw[0]);
            cudaFree(t.tw[1]);
            cudaFree(t.twd[0]);
            cudaFree(t.twd[1]);
            rc = LZK_ENOMEM;
        } else {
            k_ntt_consts<<<1, 32, 0, st>>>(k, t.consts); note_launch();
            k_powers<<<grid_for((half + 63) / 64, 128), 128, 0, st>>>(t.consts + 0, t.tw[0], half); note_launch();
            k_powers<<<grid_for((half + 63) / 64, 128), 128, 0, st>>>(t.consts + 1, t.tw[1], half); note_launch();
            for (int d = 0; d < 2; d++) {
                k_tw_to_d52<<<grid_for(half, 128), 128, 0, st>>>(t.tw[d], t.twd[d], half); note_launch();
            }
            rc = cuda_status(cudaStreamSynchronize(st));
            if (rc == LZK_OK) g_ntt_tables[{dev, k}] = t;
        }
    }
    if (rc == LZK_OK && ct == g_coset_tables.end()) {
        CosetTables c;
        size_t nlo = size_t(1) << kPowLoBits, nhi = size_t(1) << (kNttMaxLog - kPowLoBits);
        Fr* cst = g_ntt_tables[{dev, k}].consts;
        bool ok = true;
        for (int d = 0; d < 2 && ok; d++)
            ok = dev_malloc(reinterpret_cast<void**>(&c.lo[d]), nlo * sizeof(Fr)) == LZK_OK &&
                 dev_malloc(reinterpret_cast<void**>(&c.hi[d]), nhi * sizeof(Fr)) == LZK_OK;
        if (!ok) {
            for (int d = 0; d < 2; d++) { cudaFree(c.lo[d]); cudaFree(c.hi[d]); }
            rc = LZK_ENOMEM;
        }
        else {
            for (int d = 0; d < 2; d++) {
                k_powers<<<grid_for(nlo / 64, 128), 128, 0, st>>>(cst + 3 + d, c.lo[d], nlo); note_launch();
                k_powers<<<grid_for(nhi / 64, 128), 128, 0, st>>>(cst + 5 + d, c.hi[d], nhi); note_launch();
            }
            rc = cuda_status(cudaStreamSynchronize(st));
            if (rc == LZK_OK) g_coset_tables[dev] = c;
        }
    }
    cudaStreamDestroy(st);
    if (rc != LZK_OK) return rc;
    out = g_ntt_tables[{dev, k}];
    cos = g_coset_tables[dev];
    return LZK_OK;
}

struct NttPass {
    uint32_t k, s0, m, lowbits, R;
};

__device__ __forceinline__ Fr coset_pow(const Fr* lo, const Fr* hi, size_t j)
{
    return mul(ldg_elem(lo + (j & ((1u << kPowLoBits) - 1))), ldg_elem(hi + (j >> kPowLoBits)));
}

__device__ __forceinline__ size_t brev_k(size_t j, uint32_t k)
{
    return k ? (size_t)(__brevll((unsigned long long)j) >> (64 - k)) : 0;
}

// Factor a pass applies to each element as it loads it (the first pass) or
// stores it (the last pass): x * scale * g^e, e = the position j, or, with
// brev set, the coefficient index brev(j) that a bit-reversed position
// holds; a null scale or null power tables stand for 1.
__device__ __forceinline__ Fr edge_apply(const NttEdge& ed, const Fr& sc, Fr x, size_t j, uint32_t k)
{
    if (ed.scale) x = mul(x, sc);
    if (ed.lo) x = mul(x, coset_pow(ed.lo, ed.hi, ed.brev ? brev_k(j, k) : j));
    return x;
}

// m radix-2 stages in shared memory over groups of 2^m elements that differ
// in index bits [lowbits, lowbits+m); R groups with consecutive (outer, low)
// index per block.  `batch` transforms of size 2^k lie `bstride` elements
// apart (or at ptrs[blockIdx.y]).
//   DIF (decimation in frequency): stages s0 .. s0+m-1, natural order in,
//     bit-reversed out after all passes; c[j] = lo + hi, c[j^h] =
//     (lo - hi) w^((j mod h) << s) (poly.cuh:38-39).
//   DIT (decimation in time): stages t = lowbits .. lowbits+m-1, bit-reversed
//     order in, natural out; with u = w^((j mod 2^t) << (k-1-t)) hi,
//     c[j] = lo + u, c[j + 2^t] = lo - u.
// Both compute X_k = sum_j a_j w^(jk).
// Twiddle e as the second operand of the product: read from the radix-2^52
// table (TWD) or converted from the 8x32-bit table.
template <bool TWD>
__device__ __forceinline__ Fr tw_mul(const Fr& x, const Fr* __restrict__ tw, const double* __restrict__ twd, size_t e)
{
    if (TWD) {
        const double2* q = reinterpret_cast<const double2*>(twd + e * kTwdStride);
        double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
        const double d[5] = {a.x, a.y, b.x, b.y, c.x};
        return mul52_pre(x, d);
    }
    return mul52(x, ldg_elem(tw + e));
}

template <bool DIT, bool TWD>
__global__ void __launch_bounds__(kNttThreads) k_ntt_pass(Fr* __restrict__ data, NttPass p, const Fr* __restrict__ tw,
                                                           const double* __restrict__ twd, NttEdge pre, NttEdge post,
                                                           size_t bstride, Fr* const* __restrict__ ptrs)
{
    extern __shared__ uint4 smem_raw[];
    Fr* sm = reinterpret_cast<Fr*>(smem_raw);
    Fr* d = ptrs ? ptrs[blockIdx.y] : data + (size_t)blockIdx.y * bstride;
    const uint32_t G = 1u << p.m, R = p.R;
    const uint32_t rbits = __ffs(R) - 1;
    const size_t lowmask = (size_t(1) << p.lowbits) - 1;
    const uint32_t tot = G * R;
    const bool use_pre = pre.scale || pre.lo, use_post = post.scale || post.lo;
    const Fr psc = pre.scale ? ldg_elem(pre.scale) : Fr::one();
    const Fr qsc = post.scale ? ldg_elem(post.scale) : Fr::one();
    for (uint32_t i = threadIdx.x; i < tot; i += blockDim.x) {
        uint32_t g = i >> rbits, r = i & (R - 1);
        size_t cidx = (size_t)blockIdx.x * R + r;
        size_t j = ((cidx >> p.lowbits) << (p.lowbits + p.m)) | ((size_t)g << p.lowbits) | (cidx & lowmask);
        Fr x = ldg_elem(d + j);
        if (use_pre) x = edge_apply(pre, psc, x, j, p.k);
        st_elem(sm + i, x);
    }
    __syncthreads();
    for (uint32_t t = 0; t < p.m; t++) {
        // DIF: group-index bit hb = m-1-t; DIT: bit hb = t
        uint32_t hb = DIT ? t : p.m - 1 - t;
        for (uint32_t b = threadIdx.x; b < tot / 2; b += blockDim.x) {
            uint32_t r = b & (R - 1), gb = b >> rbits;
            uint32_t g = ((gb >> hb) << (hb + 1)) | (gb & ((1u << hb) - 1));
            uint32_t i0 = (g << rbits) | r, i1 = ((g + (1u << hb)) << rbits) | r;
            size_t low = ((size_t)blockIdx.x * R + r) & lowmask;
            size_t jm = (((size_t)(g & ((1u << hb) - 1))) << p.lowbits) | low;
            Fr lo = ld_elem(sm + i0), hi = ld_elem(sm + i1);
            if (DIT) {
                Fr u = tw_mul<TWD>(hi, tw, twd, jm << (p.k - 1 - (p.lowbits + t)));
                st_elem(sm + i0, add(lo, u));
                st_elem(sm + i1, sub(lo, u));
            } else {
                st_elem(sm + i0, add(lo, hi));
                // lo + p - hi, unreduced: the product takes it below 2p
                st_elem(sm + i1, tw_mul<TWD>(sub_plus_p(lo, hi), tw, twd, jm << (p.s0 + t)));
            }
        }
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < tot; i += blockDim.x) {
        uint32_t g = i >> rbits, r = i & (R - 1);
        size_t cidx = (size_t)blockIdx.x * R + r;
        size_t j = ((cidx >> p.lowbits) << (p.lowbits + p.m)) | ((size_t)g << p.lowbits) | (cidx & lowmask);
        Fr x = ld_elem(sm + i);
        if (use_post) x = edge_apply(post, qsc, x, j, p.k);
        st_elem(d + j, x);
    }
}

// In-place bit reversal; each output position pos is then multiplied by
// scale (when non-null) and g^-pos (when clo != null).
__global__ void k_ntt_bitrev(Fr* __restrict__ data, uint32_t k, const Fr* __restrict__ scale,
                             const Fr* __restrict__ clo, const Fr* __restrict__ chi, size_t bstride,
                             Fr* const* __restrict__ ptrs)
{
    Fr* d = ptrs ? ptrs[blockIdx.y] : data + (size_t)blockIdx.y * bstride;
    size_t n = size_t(1) << k;
    Fr sc = scale ? ldg_elem(scale) : Fr::one();
    for (uint64_t j = gtid(); j < n; j += gstride()) {
        size_t r = brev_k(j, k);
        if (j > r) continue;
        Fr a = ld_elem(d + j), b = ld_elem(d + r);
        // after the swap position j holds b and position r holds a
        if (scale) { a = mul(a, sc); if (j != r) b = mul(b, sc); }
        if (clo) { a = mul(a, coset_pow(clo, chi, r)); if (j != r) b = mul(b, coset_pow(clo, chi, j)); }
        st_elem(d + r, a);
        if (j != r) st_elem(d + j, b);
    }
}

int ntt_prepare_launch()
{
    static std::mutex mu;
    static bool attr_set[64] = {false};
    int dev = 0;
    LZK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        // the largest block the tuning table allows (kMaxNttBlock elements)
        LZK_CUDA(cudaFuncSetAttribute(k_ntt_pass<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxNttBlock * sizeof(Fr)));
        LZK_CUDA(cudaFuncSetAttribute(k_ntt_pass<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxNttBlock * sizeof(Fr)));
        LZK_CUDA(cudaFuncSetAttribute(k_ntt_pass<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxNttBlock * sizeof(Fr)));
        LZK_CUDA(cudaFuncSetAttribute(k_ntt_pass<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxNttBlock * sizeof(Fr)));
        attr_set[dev] = true;
    }
    return LZK_OK;
}

int ntt_passes(Fr* data, uint32_t k, uint32_t count, size_t bstride, const Fr* tw, bool dit, NttEdge pre,
               NttEdge post, cudaStream_t st, Fr* const* ptrs, const double* twd)
{
    if (k == 0 || k > 30 || count == 0 || count > 65535 || (!data && !ptrs) || !tw) return LZK_EINVAL;
    LZK_TRY(ntt_prepare_launch());
    // block size from the tuning table: 2^maxm elements, at most maxm stages a pass
    const uint32_t elems = tune_ntt_block(k);
    uint32_t maxm = 0;
    while ((1u << (maxm + 1)) <= elems) maxm++;
    const uint32_t P = (k + maxm - 1) / maxm;
    const size_t n = size_t(1) << k;
    uint32_t done = 0;   // stages done by earlier passes
    for (uint32_t q = 0; q < P; q++) {
        uint32_t m = (k - done) / (P - q);    // balanced split, larger passes last
        NttPass pp;
        pp.k = k; pp.m = m;
        // DIF passes take the top index bits first, DIT passes the bottom ones
        pp.lowbits = dit ? done : k - done - m;
        pp.s0 = dit ? 0 : done;
        uint32_t G = 1u << m;
        uint32_t R = elems / G;
        if ((size_t)R > (n >> m)) R = (uint32_t)(n >> m);
        if (R == 0) R = 1;
        pp.R = R;
        size_t blocks = (n >> m) / R;
        size_t smem = (size_t)G * R * sizeof(Fr);
        NttEdge a = q == 0 ? pre : NttEdge{}, b = q == P - 1 ? post : NttEdge{};
        const dim3 grid((unsigned)blocks, count);
        if (dit && twd)
            k_ntt_pass<true, true><<<grid, kNttThreads, smem, st>>>(data, pp, tw, twd, a, b, bstride, ptrs);
        else if (dit)
            k_ntt_pass<true, false><<<grid, kNttThreads, smem, st>>>(data, pp, tw, twd, a, b, bstride, ptrs);
        else if (twd)
            k_ntt_pass<false, true><<<grid, kNttThreads, smem, st>>>(data, pp, tw, twd, a, b, bstride, ptrs);
        else
            k_ntt_pass<false, false><<<grid, kNttThreads, smem, st>>>(data, pp, tw, twd, a, b, bstride, ptrs);
        note_launch();
        done += m;
    }
    return launch_status();
}

// Enqueue `count` transforms of size 2^k (natural order in, natural order
// out) with twiddle table tw (w^e, e < n/2): DIF passes, then the bit
// reversal with the output factors.
static int ntt_enqueue(Fr* data, uint32_t k, uint32_t count, size_t bstride, const Fr* tw, const Fr* scale,
                       const Fr* pre_lo, const Fr* pre_hi, const Fr* post_lo, const Fr* post_hi, cudaStream_t st,
                       Fr* const* ptrs = nullptr, const double* twd = nullptr)
{
    LZK_TRY(ntt_prepare_launch());
    if (k > 0) {
        NttEdge pre{pre_lo, pre_hi, nullptr, 0};
        LZK_TRY(ntt_passes(data, k, count, bstride, tw, false, pre, NttEdge{}, st, ptrs, twd));
    } else if (!(scale || post_lo || pre_lo)) {
        return LZK_OK;
    }
    size_t n = size_t(1) << k;
    k_ntt_bitrev<<<dim3(grid_for(n, 256, sm_count() * 8), count), 256, 0, st>>>(data, k, scale, post_lo, post_hi, bstride, ptrs); note_launch();
    return launch_status();
}

int ntt_run(Fr* data, uint32_t k, int dir, uint32_t count, size_t bstride, const Fr* scale_override, cudaStream_t st,
            Fr* const* ptrs)
{
    if ((!data && !ptrs) || k > kNttMaxLog || dir < 0 || dir > 3 || count == 0 || count > 65535) return LZK_EINVAL;
    if (!ptrs && count > 1 && bstride < (size_t(1) << k)) return LZK_EINVAL;
    NttTables t; CosetTables c;
    LZK_TRY(get_tables(k, t, c));
    bool inv = dir & 1, coset = dir >= 2;
    const Fr* scale = scale_override ? scale_override : (inv ? t.consts + 2 : nullptr);
    return ntt_enqueue(data, k, count, bstride, t.tw[inv ? 1 : 0], scale,
                       (coset && !inv) ? c.lo[0] : nullptr, (coset && !inv) ? c.hi[0] : nullptr,
                       (coset && inv) ? c.lo[1] : nullptr, (coset && inv) ? c.hi[1] : nullptr, st, ptrs,
                       twd_for(t, inv ? 1 : 0, k));
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_ntt_prepare(uint32_t log_n)
{
    if (log_n > kNttMaxLog) return LZK_EINVAL;
    NttTables t; CosetTables c;
    return get_tables(log_n, t, c);
}

int lzk_ntt(lzk_fr_t* data, uint32_t log_n, int direction, void* stream)
{
    return ntt_run(reinterpret_cast<Fr*>(data), log_n, direction, 1, 0, nullptr, as_stream(stream));
}

int lzk_ntt_batch(lzk_fr_t* data, uint32_t log_n, uint32_t count, size_t stride, int direction, void* stream)
{
    return ntt_run(reinterpret_cast<Fr*>(data), log_n, direction, count, stride, nullptr, as_stream(stream));
}

int lzk_number_theory_transformation(size_t deg, size_t log_deg, lzk_fr_t* coeffs, const lzk_fr_t* omega_powers,
                                     const lzk_fr_t* factor, void* stream)
{
    if (!coeffs || !omega_powers || log_deg > 30 || deg != (size_t(1) << log_deg)) return LZK_EINVAL;
    return ntt_enqueue(reinterpret_cast<Fr*>(coeffs), (uint32_t)log_deg, 1, 0,
                       reinterpret_cast<const Fr*>(omega_powers), reinterpret_cast<const Fr*>(factor),
                       nullptr, nullptr, nullptr, nullptr, as_stream(stream));
}

}  // extern "C"
