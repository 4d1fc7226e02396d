// groth16.cu -- the Groth16 prove chain on one GPU.
//
// Replaces Groth16::Prove (reference include/protocol/groth16.cuh:154-222).
// A prover object keeps the circuit view, the proving key as shifted-copy
// MSM tables (built once, resident in HBM) and all scratch, so a prove is a
// fixed sequence of launches on three streams with no host round trip:
//
//   stream main : SpMV A z, B z, C z -> H polynomial -> H MSM -> assembly
//   stream s1   : A MSM, B1 MSM -> s*Ar, r*Bs1 -> L MSM
//   stream s2   : r*d1, s*d1, (-r s)*d1, s*d2 -> B2 MSM (G2)
//
// H polynomial, two modes:
//   LZK_PROVE_REFERENCE reproduces the reference chain exactly
//     (groth16.cuh:159-198): iNTT_M with scale M^-1, NTT_2M of the
//     zero-padded coefficients, A*B - C on 2M points, iNTT_2M scaled by the
//     (4M)^-1 entry of ntt_setup (groth16-operator.cuh:13), H scalars =
//     coefficients M+1 .. 2M-1.
//   LZK_PROVE_STANDARD is the standard quotient on the coset g<w_M>:
//     iNTT_M, coset NTT_M, (A*B - C) * (g^M - 1)^-1, coset iNTT_M,
//     H scalars = h_0 .. h_{M-2}; all transforms stay at size M.
// Phase 6 (groth16.cuh:211-215) runs on the device:
//   Ar = a1 + A + r d1,  Bs1 = b1 + B1 + s d1,  Bs2 = b2 + B2 + s d2,
//   Krs = s Ar + r Bs1 + (-r s) d1 + L,  proof = (Ar, Bs2, Krs + H).
#include "common.cuh"
#include "curve.cuh"
#include "msm.cuh"
#include "ntt.cuh"
#include "r1cs.cuh"
#include <new>

struct lzk_prover {
    int mode = 0;
    lzk::CsrDev A, B, C;
    uint64_t rows = 0, n_vars = 0, n_public = 0;
    uint32_t log_m = 0;
    size_t M = 0;
    // shifted-copy tables: a, b1, l, h (G1) and b2 (G2)
    lzk::Aff<lzk::Fq>* tab[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t tn[4] = {0, 0, 0, 0};
    lzk::Aff<lzk::Fq2>* tab2 = nullptr;
    size_t tn2 = 0;
    uint32_t c = 16, wins = 16;
    // constants in device memory
    lzk::Aff<lzk::Fq>* g1c = nullptr;   // alpha1, beta1, delta1
    lzk::Aff<lzk::Fq2>* g2c = nullptr;  // beta2, delta2
    lzk::Fr* zinv = nullptr;            // (g^M - 1)^-1
    // scratch
    lzk::Fr* x = nullptr;               // 3 * L
    size_t L = 0;
    lzk::Jac<lzk::Fq>* g1res = nullptr;   // A, B1, L, H MSM results
    lzk::Jac<lzk::Fq2>* g2res = nullptr;  // B2 MSM result
    lzk::XYZZ<lzk::Fq>* sm1 = nullptr;    // r d1, s d1, (-rs) d1, s Ar, r Bs1
    lzk::XYZZ<lzk::Fq2>* sm2 = nullptr;   // s d2
    void* ws[3] = {nullptr, nullptr, nullptr};
    size_t wsb[3] = {0, 0, 0};
    cudaStream_t s1 = nullptr, s2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_fixed = nullptr, ev_s1 = nullptr, ev_s2 = nullptr;
    size_t bytes = 0;
};

namespace lzk {

struct Scal {
    uint32_t v[8];
};

// canonical 254-bit scalar from Montgomery limbs on the host side of a
// kernel argument: converted in the kernel with from_mont
__device__ __forceinline__ Fr canon(const Scal& s)
{
    Fr m;
    _Pragma("unroll") for (int i = 0; i < 8; i++) m.v[i] = s.v[i];
    return from_mont(m);
}

// k * P by MSB-first double-and-add over 256 bits (curve_utils.cuh:28-49)
template <class F>
__device__ XYZZ<F> smul(const XYZZ<F>& P, const Fr& k)
{
    XYZZ<F> acc = xyzz_inf<F>();
    for (int i = 255; i >= 0; i--) {
        acc = xyzz_dbl_cold(acc);
        if ((k.v[i >> 5] >> (i & 31)) & 1) acc = xyzz_add_cold(acc, P);
    }
    return acc;
}

// the fixed-point products: thread 0 r d1, 1 s d1, 2 (-r s) d1, 3 s d2
__global__ void k_fixed_smuls(const Aff<Fq>* g1c, const Aff<Fq2>* g2c, Scal r, Scal s, XYZZ<Fq>* sm1, XYZZ<Fq2>* sm2)
{
    uint32_t t = threadIdx.x;
    if (t < 3) {
        Fr rm, sm;
        _Pragma("unroll") for (int i = 0; i < 8; i++) { rm.v[i] = r.v[i]; sm.v[i] = s.v[i]; }
        Fr k = t == 0 ? rm : (t == 1 ? sm : mul(neg(rm), sm));
        sm1[t] = smul(xyzz_from_aff(g1c[2]), from_mont(k));
    } else if (t == 3) {
        sm2[0] = smul(xyzz_from_aff(g2c[1]), canon(s));
    }
}

// thread 0: s * Ar, Ar = a1 + A + r d1; thread 1: r * Bs1, Bs1 = b1 + B1 + s d1
__global__ void k_dep_smuls(const Aff<Fq>* g1c, const Jac<Fq>* g1res, Scal r, Scal s, XYZZ<Fq>* sm1)
{
    uint32_t t = threadIdx.x;
    if (t > 1) return;
    XYZZ<Fq> base = xyzz_from_aff(g1c[t]);
    base = xyzz_add_cold(base, jac_to_xyzz(g1res[t]));
    base = xyzz_add_cold(base, sm1[t]);
    sm1[3 + t] = smul(base, canon(t == 0 ? s : r));
}

// proof.A = Ar, proof.C = s Ar + r Bs1 + (-rs) d1 + L + H, proof.B = b2 + B2 + s d2
__global__ void k_assemble(const Aff<Fq>* g1c, const Aff<Fq2>* g2c, const Jac<Fq>* g1res, const Jac<Fq2>* g2res,
                           const XYZZ<Fq>* sm1, const XYZZ<Fq2>* sm2, lzk_groth16_proof* proof)
{
    uint32_t t = threadIdx.x;
    if (t == 0) {
        XYZZ<Fq> Ar = xyzz_add_cold(xyzz_add_cold(xyzz_from_aff(g1c[0]), jac_to_xyzz(g1res[0])), sm1[0]);
        XYZZ<Fq> C = xyzz_add_cold(sm1[3], sm1[4]);
        C = xyzz_add_cold(C, sm1[2]);
        C = xyzz_add_cold(C, jac_to_xyzz(g1res[2]));
        C = xyzz_add_cold(C, jac_to_xyzz(g1res[3]));
        st_elem(reinterpret_cast<Jac<Fq>*>(&proof->A), xyzz_to_jac(Ar));
        st_elem(reinterpret_cast<Jac<Fq>*>(&proof->C), xyzz_to_jac(C));
    } else if (t == 1) {
        XYZZ<Fq2> B = xyzz_add_cold(xyzz_add_cold(xyzz_from_aff(g2c[0]), jac_to_xyzz(g2res[0])), sm2[0]);
        st_elem(reinterpret_cast<Jac<Fq2>*>(&proof->B), xyzz_to_jac(B));
    }
}

// reference mode: x0 = x0 * x1 - x2 (poly.cuh:75-85);
// standard mode: x0 = (x0 * x1 - x2) * zinv
__global__ void k_abc(Fr* __restrict__ x0, const Fr* __restrict__ x1, const Fr* __restrict__ x2, size_t n,
                      const Fr* __restrict__ zinv)
{
    Fr zi = zinv ? ldg_elem(zinv) : Fr::one();
    for (uint64_t i = gtid(); i < n; i += gstride()) {
        Fr v = sub(mul(ld_elem(x0 + i), ldg_elem(x1 + i)), ldg_elem(x2 + i));
        if (zinv) v = mul(v, zi);
        st_elem(x0 + i, v);
    }
}

// (g^M - 1)^-1, g = 5
__global__ void k_zinv(uint32_t log_m, Fr* out)
{
    if (gtid() != 0) return;
    Fr g{{0x9fffffe6u, 0x1b0d0ef9u, 0xa32a913fu, 0xeaba68a3u, 0xd8dd0689u, 0x47d8eb76u, 0x20f5bbc3u, 0x15d00855u}};
    for (uint32_t i = 0; i < log_m; i++) g = sqr(g);
    *out = inverse(sub(g, Fr::one()));
}

static Scal to_scal(const lzk_fr_t* f)
{
    Scal s;
    for (int i = 0; i < 4; i++) { s.v[2 * i] = (uint32_t)f->limb[i]; s.v[2 * i + 1] = (uint32_t)(f->limb[i] >> 32); }
    return s;
}

static void destroy(lzk_prover* p)
{
    if (!p) return;
    for (auto t : p->tab) if (t) cudaFree(t);
    if (p->tab2) cudaFree(p->tab2);
    for (auto w : p->ws) if (w) cudaFree(w);
    void* misc[] = {p->g1c, p->g2c, p->zinv, p->x, p->g1res, p->g2res, p->sm1, p->sm2};
    for (auto m : misc) if (m) cudaFree(m);
    if (p->s1) cudaStreamDestroy(p->s1);
    if (p->s2) cudaStreamDestroy(p->s2);
    cudaEvent_t evs[] = {p->ev_fork, p->ev_fixed, p->ev_s1, p->ev_s2};
    for (auto e : evs) if (e) cudaEventDestroy(e);
    delete p;
}

template <class T>
static int dalloc(lzk_prover* p, T** ptr, size_t count)
{
    size_t b = count * sizeof(T);
    if (cudaMalloc(reinterpret_cast<void**>(ptr), b ? b : 16) != cudaSuccess) { cudaGetLastError(); return LZK_ENOMEM; }
    p->bytes += b;
    return LZK_OK;
}

static int create(const lzk_groth16_circuit* c, const lzk_groth16_pk* pk, int mode, uint32_t window_bits, lzk_prover* p)
{
    if (!c || !pk || (mode != LZK_PROVE_STANDARD && mode != LZK_PROVE_REFERENCE)) return LZK_EINVAL;
    if (c->log_domain < 1 || c->log_domain > 24 || c->n_vars < c->n_public + 1) return LZK_EINVAL;
    LZK_TRY(csr_to_dev(&c->A, p->A));
    LZK_TRY(csr_to_dev(&c->B, p->B));
    LZK_TRY(csr_to_dev(&c->C, p->C));
    p->mode = mode;
    p->log_m = c->log_domain;
    p->M = size_t(1) << c->log_domain;
    p->rows = c->A.rows;
    if (c->A.rows > p->M || c->B.rows > p->M || c->C.rows > p->M) return LZK_EINVAL;
    p->n_vars = c->n_vars;
    p->n_public = c->n_public;
    if (!pk->a_query || !pk->b1_query || !pk->b2_query || !pk->h_query || (!pk->l_query && c->n_vars > c->n_public + 1))
        return LZK_EINVAL;
    p->c = window_bits ? window_bits : 16;
    if (p->c < 2 || p->c > 24) return LZK_EINVAL;
    p->wins = windows_for(p->c);

    LZK_CUDA(cudaStreamCreateWithFlags(&p->s1, cudaStreamNonBlocking));
    LZK_CUDA(cudaStreamCreateWithFlags(&p->s2, cudaStreamNonBlocking));
    LZK_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
    LZK_CUDA(cudaEventCreateWithFlags(&p->ev_fixed, cudaEventDisableTiming));
    LZK_CUDA(cudaEventCreateWithFlags(&p->ev_s1, cudaEventDisableTiming));
    LZK_CUDA(cudaEventCreateWithFlags(&p->ev_s2, cudaEventDisableTiming));
    cudaStream_t st = p->s1;

    // tables
    const lzk_g1_affine_t* q1[4] = {pk->a_query, pk->b1_query, pk->l_query, pk->h_query};
    size_t n1[4] = {c->n_vars, c->n_vars, c->n_vars - c->n_public - 1, p->M - 1};
    for (int q = 0; q < 4; q++) {
        p->tn[q] = n1[q];
        LZK_TRY(dalloc(p, &p->tab[q], (size_t)p->wins * (n1[q] ? n1[q] : 1)));
        if (n1[q])
            LZK_TRY(lzk_g1_precompute(q1[q], n1[q], p->c, p->wins, reinterpret_cast<lzk_g1_affine_t*>(p->tab[q]), n1[q], st));
    }
    p->tn2 = c->n_vars;
    LZK_TRY(dalloc(p, &p->tab2, (size_t)p->wins * p->tn2));
    LZK_TRY(lzk_g2_precompute(pk->b2_query, p->tn2, p->c, p->wins, reinterpret_cast<lzk_g2_affine_t*>(p->tab2), p->tn2, st));

    // constants
    LZK_TRY(dalloc(p, &p->g1c, 3));
    LZK_TRY(dalloc(p, &p->g2c, 2));
    const lzk_g1_affine_t g1h[3] = {pk->alpha1, pk->beta1, pk->delta1};
    const lzk_g2_affine_t g2h[2] = {pk->beta2, pk->delta2};
    LZK_CUDA(cudaMemcpyAsync(p->g1c, g1h, sizeof(g1h), cudaMemcpyHostToDevice, st));
    LZK_CUDA(cudaMemcpyAsync(p->g2c, g2h, sizeof(g2h), cudaMemcpyHostToDevice, st));
    LZK_TRY(dalloc(p, &p->zinv, 1));
    k_zinv<<<1, 32, 0, st>>>(p->log_m, p->zinv);

    // scratch
    p->L = mode == LZK_PROVE_REFERENCE ? 2 * p->M : p->M;
    LZK_TRY(dalloc(p, &p->x, 3 * p->L));
    LZK_TRY(dalloc(p, &p->g1res, 4));
    LZK_TRY(dalloc(p, &p->g2res, 1));
    LZK_TRY(dalloc(p, &p->sm1, 5));
    LZK_TRY(dalloc(p, &p->sm2, 1));
    for (int i = 0; i < 3; i++) {
        lzk_msm_cfg cfg{};
        cfg.window_bits = p->c;
        cfg.flags = LZK_MSM_PRECOMPUTED;
        cfg.precomp_windows = p->wins;
        cfg.level_stride = p->M + c->n_vars;
        size_t mx = p->M > c->n_vars ? p->M : c->n_vars;
        p->wsb[i] = lzk_msm_workspace_bytes(i == 2 ? 2 : 1, mx, &cfg);
        LZK_TRY(dalloc(p, reinterpret_cast<char**>(&p->ws[i]), p->wsb[i]));
    }
    // NTT tables for every size the chain uses
    NttTables t; CosetTables ct;
    LZK_TRY(get_tables(p->log_m, t, ct));
    if (mode == LZK_PROVE_REFERENCE) {
        LZK_TRY(get_tables(p->log_m + 1, t, ct));
        LZK_TRY(get_tables(p->log_m + 2, t, ct));
    }
    LZK_TRY(launch_status());
    LZK_CUDA(cudaStreamSynchronize(st));
    return LZK_OK;
}

static int msm_tab1(lzk_prover* p, int q, const Fr* scal, size_t n, Jac<Fq>* out, int wsi, cudaStream_t st)
{
    lzk_msm_cfg cfg{};
    cfg.window_bits = p->c;
    cfg.flags = LZK_MSM_PRECOMPUTED;
    cfg.precomp_windows = p->wins;
    cfg.level_stride = p->tn[q];
    cfg.workspace = p->ws[wsi];
    cfg.workspace_bytes = p->wsb[wsi];
    return lzk_msm_g1(reinterpret_cast<const lzk_fr_t*>(scal), reinterpret_cast<const lzk_g1_affine_t*>(p->tab[q]), n,
                      reinterpret_cast<lzk_g1_t*>(out), &cfg, st);
}

static int prove(lzk_prover* p, const Fr* z, const lzk_fr_t* r, const lzk_fr_t* s, lzk_groth16_proof* proof,
                 cudaStream_t st)
{
    if (!p || !z || !r || !s || !proof) return LZK_EINVAL;
    Scal rs = to_scal(r), ss = to_scal(s);
    void* tr = trace_begin("groth16_prove", st);
    LZK_CUDA(cudaEventRecord(p->ev_fork, st));
    LZK_CUDA(cudaStreamWaitEvent(p->s1, p->ev_fork, 0));
    LZK_CUDA(cudaStreamWaitEvent(p->s2, p->ev_fork, 0));

    // s2: fixed-point scalar products, then the G2 MSM
    k_fixed_smuls<<<1, 32, 0, p->s2>>>(p->g1c, p->g2c, rs, ss, p->sm1, p->sm2);
    LZK_CUDA(cudaEventRecord(p->ev_fixed, p->s2));
    {
        lzk_msm_cfg cfg{};
        cfg.window_bits = p->c;
        cfg.flags = LZK_MSM_PRECOMPUTED;
        cfg.precomp_windows = p->wins;
        cfg.level_stride = p->tn2;
        cfg.workspace = p->ws[2];
        cfg.workspace_bytes = p->wsb[2];
        LZK_TRY(lzk_msm_g2(reinterpret_cast<const lzk_fr_t*>(z), reinterpret_cast<const lzk_g2_affine_t*>(p->tab2),
                           p->n_vars, reinterpret_cast<lzk_g2_t*>(p->g2res), &cfg, p->s2));
    }
    LZK_CUDA(cudaEventRecord(p->ev_s2, p->s2));

    // s1: A, B1 MSMs, dependent products, L MSM
    LZK_TRY(msm_tab1(p, 0, z, p->n_vars, p->g1res + 0, 1, p->s1));
    LZK_TRY(msm_tab1(p, 1, z, p->n_vars, p->g1res + 1, 1, p->s1));
    LZK_CUDA(cudaStreamWaitEvent(p->s1, p->ev_fixed, 0));
    k_dep_smuls<<<1, 32, 0, p->s1>>>(p->g1c, p->g1res, rs, ss, p->sm1);
    size_t nl = p->n_vars - p->n_public - 1;
    LZK_TRY(msm_tab1(p, 2, z + p->n_public + 1, nl, p->g1res + 2, 1, p->s1));
    LZK_CUDA(cudaEventRecord(p->ev_s1, p->s1));

    // main: H polynomial and H MSM
    Fr* x0 = p->x;
    Fr* x1 = p->x + p->L;
    Fr* x2 = p->x + 2 * p->L;
    LZK_CUDA(cudaMemsetAsync(p->x, 0, 3 * p->L * sizeof(Fr), st));
    lzk_csr none{};
    (void)none;
    {
        CsrDev a = p->A, b = p->B, c = p->C;
        lzk_csr ca{reinterpret_cast<const lzk_fr_t*>(a.val), a.col, a.rowp, a.rows, 0, a.nnz, a.ib, 0};
        lzk_csr cb{reinterpret_cast<const lzk_fr_t*>(b.val), b.col, b.rowp, b.rows, 0, b.nnz, b.ib, 0};
        lzk_csr cc{reinterpret_cast<const lzk_fr_t*>(c.val), c.col, c.rowp, c.rows, 0, c.nnz, c.ib, 0};
        LZK_TRY(lzk_spmv3(&ca, &cb, &cc, reinterpret_cast<const lzk_fr_t*>(z), reinterpret_cast<lzk_fr_t*>(x0),
                          reinterpret_cast<lzk_fr_t*>(x1), reinterpret_cast<lzk_fr_t*>(x2), st));
    }
    const Fr* hs;
    if (p->mode == LZK_PROVE_REFERENCE) {
        LZK_TRY(ntt_run(p->x, p->log_m, LZK_NTT_INVERSE, 3, p->L, nullptr, st));
        LZK_TRY(ntt_run(p->x, p->log_m + 1, LZK_NTT_FORWARD, 3, p->L, nullptr, st));
        k_abc<<<grid_for(p->L, 256, 148 * 8), 256, 0, st>>>(x0, x1, x2, p->L, nullptr);
        NttTables t4; CosetTables ct;
        LZK_TRY(get_tables(p->log_m + 2, t4, ct));
        LZK_TRY(ntt_run(x0, p->log_m + 1, LZK_NTT_INVERSE, 1, 0, t4.consts + 2, st));
        hs = x0 + p->M + 1;
    } else {
        LZK_TRY(ntt_run(p->x, p->log_m, LZK_NTT_INVERSE, 3, p->L, nullptr, st));
        LZK_TRY(ntt_run(p->x, p->log_m, LZK_NTT_COSET_FORWARD, 3, p->L, nullptr, st));
        k_abc<<<grid_for(p->L, 256, 148 * 8), 256, 0, st>>>(x0, x1, x2, p->L, p->zinv);
        LZK_TRY(ntt_run(x0, p->log_m, LZK_NTT_COSET_INVERSE, 1, 0, nullptr, st));
        hs = x0;
    }
    LZK_TRY(msm_tab1(p, 3, hs, p->M - 1, p->g1res + 3, 0, st));

    // join and assemble
    LZK_CUDA(cudaStreamWaitEvent(st, p->ev_s1, 0));
    LZK_CUDA(cudaStreamWaitEvent(st, p->ev_s2, 0));
    k_assemble<<<1, 32, 0, st>>>(p->g1c, p->g2c, p->g1res, p->g2res, p->sm1, p->sm2, proof);
    trace_end(tr, st);
    return launch_status();
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_prover_create(const lzk_groth16_circuit* c, const lzk_groth16_pk* pk, int mode, uint32_t window_bits,
                      lzk_prover** out)
{
    if (!out) return LZK_EINVAL;
    *out = nullptr;
    lzk_prover* p = new (std::nothrow) lzk_prover();
    if (!p) return LZK_ENOMEM;
    int rc = create(c, pk, mode, window_bits, p);
    if (rc != LZK_OK) { destroy(p); return rc; }
    *out = p;
    return LZK_OK;
}

int lzk_prover_destroy(lzk_prover* p)
{
    if (!p) return LZK_EINVAL;
    cudaDeviceSynchronize();
    destroy(p);
    return LZK_OK;
}

size_t lzk_prover_device_bytes(const lzk_prover* p) { return p ? p->bytes : 0; }

int lzk_groth16_prove(lzk_prover* p, const lzk_fr_t* z, const lzk_fr_t* r, const lzk_fr_t* s,
                      lzk_groth16_proof* proof, void* stream)
{
    return prove(p, reinterpret_cast<const Fr*>(z), r, s, proof, as_stream(stream));
}

}  // extern "C"
