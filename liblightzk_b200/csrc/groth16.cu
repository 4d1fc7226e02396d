// groth16.cu -- the Groth16 prove chain on one GPU.
//
// Replaces Groth16::Prove (reference include/protocol/groth16.cuh:154-222).
// A prover object keeps the circuit view, the proving key as shifted-copy
// MSM tables (built once, resident in HBM) and all scratch, so a prove is a
// fixed sequence of launches on three streams with no host round trip:
//
//   stream main : SpMV A z, B z, C z -> H polynomial -> L + H MSM -> assembly
//   stream s1   : A MSM, B1 MSM
//   stream s2   : B2 MSM (G2), after the A MSM
//   stream s3   : fixed-point products r d1, s a1, r b1, (r s) d1, s d2 from
//                 comb tables; after B1: s*A and r*B1 (variable base)
//
// H polynomial, two modes:
//   LZK_PROVE_REFERENCE reproduces the reference chain exactly
//     (groth16.cuh:159-198): iNTT_M with scale M^-1, NTT_2M of the
//     zero-padded coefficients, A*B - C on 2M points, iNTT_2M scaled by the
//     (4M)^-1 entry of ntt_setup (groth16-operator.cuh:13), H scalars =
//     coefficients M+1 .. 2M-1.
//   LZK_PROVE_STANDARD is the standard quotient on the coset g<w_M>:
//     iNTT_M, coset NTT_M, (A*B - C) * (g^M - 1)^-1, coset iNTT_M,
//     H scalars = h_0 .. h_{M-2}; all transforms stay at size M and none
//     has a bit-reversal pass: decimation-in-frequency passes for the
//     inverses and decimation-in-time passes for the coset transforms, so
//     the H coefficients end in bit-reversed order, the order in which the
//     prover stores the H query.
// Phase 6 (groth16.cuh:211-215) runs on the device.  The reference forms
//   Ar = a1 + A + r d1,  Bs1 = b1 + B1 + s d1,  Bs2 = b2 + B2 + s d2,
//   Krs = s Ar + r Bs1 + (-r s) d1 + L,  proof = (Ar, Bs2, Krs + H);
// expanding s Ar and r Bs1 gives the same group element
//   Krs + H = s a1 + r b1 + s A + r B1 + (r s) d1 + L + H,
// whose fixed-base terms come from per-prover comb tables (32 mixed
// additions each) and whose only variable-base products are s A and r B1.
#include "common.cuh"
#include "curve.cuh"
#include "msm.cuh"
#include "ntt.cuh"
#include "keygen.cuh"
#include "prover.cuh"
#include <new>

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

// fixed-base products from comb tables: thread 0 r d1, 1 s a1, 2 r b1,
// 3 (r s) d1, 4 s d2
__global__ void k_fixed_products(const Aff<Fq>* __restrict__ comb1, const Aff<Fq2>* __restrict__ comb2, Scal r, Scal s,
                                 XYZZ<Fq>* __restrict__ sm1, XYZZ<Fq2>* __restrict__ sm2)
{
    uint32_t t = threadIdx.x;
    if (t > 4) return;
    Fr rm, sm;
    _Pragma("unroll") for (int i = 0; i < 8; i++) { rm.v[i] = r.v[i]; sm.v[i] = s.v[i]; }
    if (t == 4) { sm2[0] = comb_mul(comb2, from_mont(sm)); return; }
    const int table[4] = {2, 0, 1, 2};   // d1, a1, b1, d1
    Fr k = t == 0 ? rm : t == 1 ? sm : t == 2 ? rm : mul(rm, sm);
    sm1[t] = comb_mul(comb1 + table[t] * 8192, from_mont(k));
}

// k * P, 4-bit fixed window: 15 precomputed multiples, then per nibble four
// doublings and one addition (curve_utils.cuh:28-49 computes the same
// product bit by bit).  Run by a whole warp with warp-uniform point
// operations: every lane holds P, k and the table, and gets the product.
template <class F>
__device__ XYZZ<F> smul_w4_warp(const XYZZ<F>& P, const Fr& k)
{
    XYZZ<F> tab[16];
    tab[0] = xyzz_inf<F>();
    tab[1] = P;
    for (int i = 2; i < 16; i++) tab[i] = (i & 1) ? xyzz_add_warp(tab[i - 1], P) : xyzz_dbl_warp(tab[i >> 1]);
    XYZZ<F> acc = xyzz_inf<F>();
    for (int w = 63; w >= 0; w--) {
        for (int d = 0; d < 4; d++) acc = xyzz_dbl_warp(acc);
        uint32_t nib = (k.v[w >> 3] >> (4 * (w & 7))) & 15u;
        if (nib) acc = xyzz_add_warp(acc, tab[nib]);
    }
    return acc;
}

// variable-base products: warp 0 s * A, warp 1 r * B1 (<<<1, 64>>>)
__global__ void k_dep_products(const Jac<Fq>* __restrict__ g1res, Scal r, Scal s, XYZZ<Fq>* __restrict__ sm1)
{
    const uint32_t w = threadIdx.x >> 5;
    if (w > 1) return;
    XYZZ<Fq> x = smul_w4_warp(jac_to_xyzz(g1res[w]), canon(w == 0 ? s : r));
    if ((threadIdx.x & 31) == 0) sm1[4 + w] = x;
}

// proof.A = a1 + A + r d1; proof.B = b2 + B2 + s d2;
// proof.C = s a1 + r b1 + (r s) d1 + s A + r B1 + L + H
// One warp per proof point (<<<1, 96>>>), warp-uniform additions: the
// assembly ends every proof, so its chain of additions is on the critical
// path.
__global__ void k_assemble(const Aff<Fq>* g1c, const Aff<Fq2>* g2c, const Jac<Fq>* g1res, const Jac<Fq2>* g2res,
                           const XYZZ<Fq>* sm1, const XYZZ<Fq2>* sm2, lzk_groth16_proof* proof)
{
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w == 0) {
        XYZZ<Fq> A = xyzz_add_warp(xyzz_add_warp(xyzz_from_aff(g1c[0]), jac_to_xyzz(g1res[0])), sm1[0]);
        Jac<Fq> j = xyzz_to_jac_warp(A);
        if (lane == 0) st_elem(reinterpret_cast<Jac<Fq>*>(&proof->A), j);
    } else if (w == 1) {
        XYZZ<Fq> C = xyzz_add_warp(sm1[1], sm1[2]);
        C = xyzz_add_warp(C, sm1[3]);
        C = xyzz_add_warp(C, sm1[4]);
        C = xyzz_add_warp(C, sm1[5]);
        C = xyzz_add_warp(C, jac_to_xyzz(g1res[2]));   // L + H
        Jac<Fq> j = xyzz_to_jac_warp(C);
        if (lane == 0) st_elem(reinterpret_cast<Jac<Fq>*>(&proof->C), j);
    } else if (w == 2) {
        XYZZ<Fq2> B = xyzz_add_warp(xyzz_add_warp(xyzz_from_aff(g2c[0]), jac_to_xyzz(g2res[0])), sm2[0]);
        Jac<Fq2> j = xyzz_to_jac_warp(B);
        if (lane == 0) st_elem(reinterpret_cast<Jac<Fq2>*>(&proof->B), j);
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

// out[i] = in[brev(i)] over log_m-bit indices, i < n (n <= 2^log_m - 1, so
// brev(i) < n: the bit reversal is an involution that fixes 2^log_m - 1)
__global__ void k_gather_brev(const Aff<Fq>* __restrict__ in, size_t n, uint32_t log_m, Aff<Fq>* __restrict__ out)
{
    for (uint64_t i = gtid(); i < n; i += gstride()) {
        size_t j = (size_t)(__brevll((unsigned long long)i) >> (64 - log_m));
        st_elem(out + i, ldg_elem(in + j));
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

lzk_msm_cfg prover_msm_cfg(const lzk_prover* p, int i, size_t level_stride)
{
    lzk_msm_cfg cfg{};
    cfg.window_bits = p->c;
    cfg.flags = LZK_MSM_PRECOMPUTED;
    cfg.precomp_windows = p->wins;
    cfg.level_stride = level_stride;
    cfg.acc_chunk = p->chunk[i];
    cfg.reduce_run = p->run[i];
    return cfg;
}

template <class T>
static int dalloc(size_t* acct, T** ptr, size_t count)
{
    size_t b = count * sizeof(T);
    LZK_TRY(dev_malloc(reinterpret_cast<void**>(ptr), b));
    *acct += b;
    return LZK_OK;
}

void ctx_destroy(ProveCtx* x)
{
    if (!x) return;
    for (auto w : x->ws) if (w) cudaFree(w);
    void* misc[] = {x->x, x->g1res, x->g2res, x->sm1, x->sm2, x->z, x->proof,
                    x->zs_cnt, x->zs_off, x->zs_ent, x->zs_bsums};
    for (auto m : misc) if (m) cudaFree(m);
    if (x->proof_host) cudaFreeHost(x->proof_host);
    if (x->ev_done) cudaEventDestroy(x->ev_done);
    cudaStream_t sts[] = {x->s0, x->s1, x->s2, x->s3};
    for (auto t : sts) if (t) cudaStreamDestroy(t);
    cudaEvent_t evs[] = {x->ev_fork, x->ev_b1, x->ev_s1, x->ev_s2, x->ev_s3, x->ev_sorted};
    for (auto e : evs) if (e) cudaEventDestroy(e);
    delete x;
}

// Scratch for one proof of prover p; serving contexts also get their own
// main stream and witness and proof buffers.
int ctx_create(const lzk_prover* p, bool serving, ProveCtx** out)
{
    *out = nullptr;
    ProveCtx* x = new (std::nothrow) ProveCtx();
    if (!x) return LZK_ENOMEM;
    int rc = LZK_OK;
    do {
        if ((rc = dalloc(&x->bytes, &x->x, 3 * p->L))) break;
        if ((rc = dalloc(&x->bytes, &x->g1res, 4))) break;
        if ((rc = dalloc(&x->bytes, &x->g2res, 1))) break;
        if ((rc = dalloc(&x->bytes, &x->sm1, 6))) break;
        if ((rc = dalloc(&x->bytes, &x->sm2, 1))) break;
        for (int i = 0; i < 3 && rc == LZK_OK; i++) {
            // ws[0]: the concatenated L and H MSM; ws[1]: A and B1; ws[2]: B2
            size_t n = i == 0 ? p->tn[2] : p->n_vars;
            lzk_msm_cfg cfg = prover_msm_cfg(p, i, n);
            x->wsb[i] = lzk_msm_workspace_bytes(i == 2 ? 2 : 1, n, &cfg);
            rc = dalloc(&x->bytes, reinterpret_cast<char**>(&x->ws[i]), x->wsb[i]);
        }
        if (rc) break;
        {
            // the A, B1 and B2 tables all have level stride n_vars
            SortWords w = msm_sort_words(p->n_vars, p->c, p->n_vars);
            if ((rc = dalloc(&x->bytes, &x->zs_cnt, w.cnt))) break;
            if ((rc = dalloc(&x->bytes, &x->zs_off, w.off))) break;
            if ((rc = dalloc(&x->bytes, &x->zs_ent, w.ent))) break;
            if ((rc = dalloc(&x->bytes, &x->zs_bsums, w.bsums))) break;
        }
        if (serving) {
            if ((rc = dalloc(&x->bytes, &x->z, p->n_vars))) break;
            if ((rc = dalloc(&x->bytes, &x->proof, 1))) break;
            if (cudaStreamCreateWithFlags(&x->s0, cudaStreamNonBlocking) != cudaSuccess) { rc = LZK_EDEVICE; break; }
            if (cudaEventCreateWithFlags(&x->ev_done, cudaEventDisableTiming) != cudaSuccess) { rc = LZK_EDEVICE; break; }
            if (cudaMallocHost(&x->proof_host, sizeof(lzk_groth16_proof)) != cudaSuccess) { rc = LZK_ENOMEM; break; }
        }
        cudaStream_t* sts[] = {&x->s1, &x->s2, &x->s3};
        for (auto t : sts) if (cudaStreamCreateWithFlags(t, cudaStreamNonBlocking) != cudaSuccess) rc = LZK_EDEVICE;
        cudaEvent_t* evs[] = {&x->ev_fork, &x->ev_b1, &x->ev_s1, &x->ev_s2, &x->ev_s3, &x->ev_sorted};
        for (auto e : evs) if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) rc = LZK_EDEVICE;
    } while (0);
    if (rc != LZK_OK) { cudaGetLastError(); ctx_destroy(x); return rc; }
    *out = x;
    return LZK_OK;
}

static void destroy(lzk_prover* p)
{
    if (!p) return;
    ctx_destroy(p->ctx0);
    for (auto t : p->tab) if (t) cudaFree(t);
    if (p->tab2) cudaFree(p->tab2);
    void* misc[] = {p->g1c, p->g2c, p->zinv, p->comb1, p->comb2};
    for (auto m : misc) if (m) cudaFree(m);
    delete p;
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
    p->L = mode == LZK_PROVE_REFERENCE ? 2 * p->M : p->M;
    p->rows = c->A.rows;
    if (c->A.rows > p->M || c->B.rows > p->M || c->C.rows > p->M) return LZK_EINVAL;
    p->n_vars = c->n_vars;
    p->n_public = c->n_public;
    if (!pk->a_query || !pk->b1_query || !pk->b2_query || !pk->h_query || (!pk->l_query && c->n_vars > c->n_public + 1))
        return LZK_EINVAL;
    p->c = window_bits ? window_bits : 17;
    if (p->c < 2 || p->c > 24) return LZK_EINVAL;
    p->wins = windows_for(p->c);
    // level strides of the tables (ctx_create sizes the MSM workspaces by them)
    p->tn[0] = p->tn[1] = c->n_vars;
    p->nl = c->n_vars - c->n_public - 1;
    p->tn[2] = p->nl + (p->M - 1);
    for (int i = 0; i < 3; i++) {
        size_t n = i == 0 ? p->tn[2] : p->n_vars;
        int group = i == 2 ? 2 : 1;
        p->chunk[i] = tune_chunk(group, n, true);
        p->run[i] = tune_run(group, n, true);
    }

    LZK_TRY(ctx_create(p, false, &p->ctx0));
    cudaStream_t st = p->ctx0->s1;

    // tables: a and b1 (level stride n_vars); l and h concatenated in one
    // table of level stride n_l + M - 1, since the L and H MSMs enter the
    // proof only through their sum and run as one MSM
    const lzk_g1_affine_t* q1[2] = {pk->a_query, pk->b1_query};
    for (int q = 0; q < 2; q++) {
        LZK_TRY(dalloc(&p->bytes, &p->tab[q], (size_t)p->wins * p->tn[q]));
        LZK_TRY(lzk_g1_precompute(q1[q], p->tn[q], p->c, p->wins, reinterpret_cast<lzk_g1_affine_t*>(p->tab[q]),
                                  p->tn[q], st));
    }
    LZK_TRY(dalloc(&p->bytes, &p->tab[2], (size_t)p->wins * p->tn[2]));
    if (p->nl)
        LZK_TRY(lzk_g1_precompute(pk->l_query, p->nl, p->c, p->wins, reinterpret_cast<lzk_g1_affine_t*>(p->tab[2]),
                                  p->tn[2], st));
    {
        // standard mode leaves the H coefficients in bit-reversed order (the
        // transforms skip their bit reversal), so its H table holds the
        // query in that order: entry i = h_query[brev(i)]
        const lzk_g1_affine_t* hq = pk->h_query;
        Aff<Fq>* perm = nullptr;
        if (mode == LZK_PROVE_STANDARD) {
            size_t scratch = 0;
            LZK_TRY(dalloc(&scratch, &perm, p->M - 1));
            k_gather_brev<<<grid_for(p->M - 1, 256, sm_count() * 8), 256, 0, st>>>(
                reinterpret_cast<const Aff<Fq>*>(pk->h_query), p->M - 1, p->log_m, perm); note_launch();
            hq = reinterpret_cast<const lzk_g1_affine_t*>(perm);
        }
        int rc = lzk_g1_precompute(hq, p->M - 1, p->c, p->wins, reinterpret_cast<lzk_g1_affine_t*>(p->tab[2] + p->nl),
                                   p->tn[2], st);
        if (perm) {
            cudaStreamSynchronize(st);
            cudaFree(perm);
        }
        LZK_TRY(rc);
    }
    p->tn2 = c->n_vars;
    LZK_TRY(dalloc(&p->bytes, &p->tab2, (size_t)p->wins * p->tn2));
    LZK_TRY(lzk_g2_precompute(pk->b2_query, p->tn2, p->c, p->wins, reinterpret_cast<lzk_g2_affine_t*>(p->tab2), p->tn2, st));

    // constants
    LZK_TRY(dalloc(&p->bytes, &p->g1c, 3));
    LZK_TRY(dalloc(&p->bytes, &p->g2c, 2));
    const lzk_g1_affine_t g1h[3] = {pk->alpha1, pk->beta1, pk->delta1};
    const lzk_g2_affine_t g2h[2] = {pk->beta2, pk->delta2};
    LZK_CUDA(cudaMemcpyAsync(p->g1c, g1h, sizeof(g1h), cudaMemcpyHostToDevice, st));
    LZK_CUDA(cudaMemcpyAsync(p->g2c, g2h, sizeof(g2h), cudaMemcpyHostToDevice, st));
    LZK_TRY(dalloc(&p->bytes, &p->zinv, 1));
    k_zinv<<<1, 32, 0, st>>>(p->log_m, p->zinv); note_launch();
    LZK_TRY(dalloc(&p->bytes, &p->comb1, 3 * 8192));
    LZK_TRY(dalloc(&p->bytes, &p->comb2, 8192));
    for (int i = 0; i < 3; i++) LZK_TRY(comb_build<Fq>(p->g1c + i, p->comb1 + i * 8192, st));
    LZK_TRY(comb_build<Fq2>(p->g2c + 1, p->comb2, st));
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

static int msm_tab1(const lzk_prover* p, ProveCtx* x, int q, const Fr* scal, size_t n, Jac<Fq>* out, int wsi,
                    cudaStream_t st, bool presorted = false)
{
    lzk_msm_cfg cfg = prover_msm_cfg(p, wsi, p->tn[q]);
    cfg.workspace = x->ws[wsi];
    cfg.workspace_bytes = x->wsb[wsi];
    if (presorted) return msm_g1_presorted(scal, p->tab[q], n, out, &cfg, st, x->zs_off, x->zs_ent);
    return lzk_msm_g1(reinterpret_cast<const lzk_fr_t*>(scal), reinterpret_cast<const lzk_g1_affine_t*>(p->tab[q]), n,
                      reinterpret_cast<lzk_g1_t*>(out), &cfg, st);
}

int prove_ctx(const lzk_prover* p, ProveCtx* x, const Fr* z, const lzk_fr_t* r, const lzk_fr_t* s,
              lzk_groth16_proof* proof, cudaStream_t st)
{
    if (!p || !z || !r || !s || !proof) return LZK_EINVAL;
    Scal rs = to_scal(r), ss = to_scal(s);
    void* tr = trace_begin("groth16_prove", st);
    LZK_CUDA(cudaEventRecord(x->ev_fork, st));
    LZK_CUDA(cudaStreamWaitEvent(x->s1, x->ev_fork, 0));
    LZK_CUDA(cudaStreamWaitEvent(x->s2, x->ev_fork, 0));
    LZK_CUDA(cudaStreamWaitEvent(x->s3, x->ev_fork, 0));

    // s3: fixed-base products
    void* tr_fx = trace_begin("groth16_fixed_products", x->s3);
    k_fixed_products<<<1, 32, 0, x->s3>>>(p->comb1, p->comb2, rs, ss, x->sm1, x->sm2); note_launch();
    trace_end(tr_fx, x->s3);

    // s1: one digit sort of z for the A, B1 and B2 MSMs (same scalars, same
    // window width, tables of the same level stride n_vars)
    LZK_TRY(msm_sort_scalars(z, p->n_vars, p->c, p->n_vars, x->zs_cnt, x->zs_off, x->zs_ent, x->zs_bsums, x->s1));

    // s1: A and B1 MSMs; s3 picks up A and B1 for s*A and r*B1
    LZK_TRY(msm_tab1(p, x, 0, z, p->n_vars, x->g1res + 0, 1, x->s1, true));

    // s2: the G2 MSM, from the same sort, once the A MSM is done: started
    // beside the A MSM its 2000-block accumulation kept the A MSM's fix-up
    // and reduction waiting, which delayed B1 and the products that end the
    // proof (measured 30.00 -> 29.73 ms per proof)
    LZK_CUDA(cudaEventRecord(x->ev_sorted, x->s1));
    LZK_CUDA(cudaStreamWaitEvent(x->s2, x->ev_sorted, 0));
    {
        lzk_msm_cfg cfg = prover_msm_cfg(p, 2, p->tn2);
        cfg.workspace = x->ws[2];
        cfg.workspace_bytes = x->wsb[2];
        LZK_TRY(msm_g2_presorted(z, p->tab2, p->n_vars, x->g2res, &cfg, x->s2, x->zs_off, x->zs_ent));
    }
    LZK_CUDA(cudaEventRecord(x->ev_s2, x->s2));

    LZK_TRY(msm_tab1(p, x, 1, z, p->n_vars, x->g1res + 1, 1, x->s1, true));
    LZK_CUDA(cudaEventRecord(x->ev_b1, x->s1));
    LZK_CUDA(cudaStreamWaitEvent(x->s3, x->ev_b1, 0));
    void* tr_dep = trace_begin("groth16_dep_products", x->s3);
    k_dep_products<<<1, 64, 0, x->s3>>>(x->g1res, rs, ss, x->sm1); note_launch();
    trace_end(tr_dep, x->s3);
    LZK_CUDA(cudaEventRecord(x->ev_s3, x->s3));
    LZK_CUDA(cudaEventRecord(x->ev_s1, x->s1));

    // main: H polynomial, then the L + H MSM
    Fr* x0 = x->x;
    Fr* x1 = x->x + p->L;
    Fr* x2 = x->x + 2 * p->L;
    void* tr_h = trace_begin("groth16_h_poly", st);
    LZK_CUDA(cudaMemsetAsync(x->x, 0, 3 * p->L * sizeof(Fr), st));
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
        LZK_TRY(ntt_run(x->x, p->log_m, LZK_NTT_INVERSE, 3, p->L, nullptr, st));
        LZK_TRY(ntt_run(x->x, p->log_m + 1, LZK_NTT_FORWARD, 3, p->L, nullptr, st));
        k_abc<<<grid_for(p->L, 256, sm_count() * 8), 256, 0, st>>>(x0, x1, x2, p->L, nullptr); note_launch();
        NttTables t4; CosetTables ct;
        LZK_TRY(get_tables(p->log_m + 2, t4, ct));
        LZK_TRY(ntt_run(x0, p->log_m + 1, LZK_NTT_INVERSE, 1, 0, t4.consts + 2, st));
        hs = x0 + p->M + 1;
    } else {
        // no bit reversal anywhere: the inverse transforms are DIF passes
        // (natural -> bit-reversed, unscaled), the coset transforms DIT passes
        // (bit-reversed -> natural) whose first pass applies M^-1 g^j to
        // coefficient j, and the last inverse's final pass applies
        // M^-1 g^-j, leaving h_j at position brev(j) (the H table's order)
        NttTables t; CosetTables ct;
        LZK_TRY(get_tables(p->log_m, t, ct));
        const Fr* minv = t.consts + 2;
        LZK_TRY(ntt_passes(x->x, p->log_m, 3, p->L, t.tw[1], false, NttEdge{}, NttEdge{}, st, nullptr,
                           twd_for(t, 1, p->log_m)));
        LZK_TRY(ntt_passes(x->x, p->log_m, 3, p->L, t.tw[0], true, NttEdge{ct.lo[0], ct.hi[0], minv, 1}, NttEdge{}, st,
                           nullptr, twd_for(t, 0, p->log_m)));
        k_abc<<<grid_for(p->L, 256, sm_count() * 8), 256, 0, st>>>(x0, x1, x2, p->L, p->zinv); note_launch();
        LZK_TRY(ntt_passes(x0, p->log_m, 1, 0, t.tw[1], false, NttEdge{}, NttEdge{ct.lo[1], ct.hi[1], minv, 1}, st,
                           nullptr, twd_for(t, 1, p->log_m)));
        hs = x0;
    }
    trace_end(tr_h, st);
    // L and H as one MSM: scalars z_(n_public+1) .. z_(n_vars-1), then the
    // H coefficients, over the concatenated table
    {
        lzk_msm_cfg cfg = prover_msm_cfg(p, 0, p->tn[2]);
        cfg.workspace = x->ws[0];
        cfg.workspace_bytes = x->wsb[0];
        LZK_TRY(msm_g1_concat(z + p->n_public + 1, p->nl, hs, p->M - 1, p->tab[2], x->g1res + 2, &cfg, st));
    }

    // join and assemble
    LZK_CUDA(cudaStreamWaitEvent(st, x->ev_s1, 0));
    LZK_CUDA(cudaStreamWaitEvent(st, x->ev_s2, 0));
    LZK_CUDA(cudaStreamWaitEvent(st, x->ev_s3, 0));
    void* tr_as = trace_begin("groth16_assemble", st);
    k_assemble<<<1, 96, 0, st>>>(p->g1c, p->g2c, x->g1res, x->g2res, x->sm1, x->sm2, proof); note_launch();
    trace_end(tr_as, st);
    trace_end(tr, st);
    return launch_status();
}

// ---------------- proof wire format ----------------
// Affine coordinates as canonical little-endian integers; infinity = zeros.
__device__ __forceinline__ Fq wire_out(const Fq& a) { return from_mont(a); }
__device__ __forceinline__ Fq2 wire_out(const Fq2& a) { return {from_mont(a.c0), from_mont(a.c1)}; }
__device__ __forceinline__ Fq wire_in(const Fq& a) { return to_mont(a); }
__device__ __forceinline__ Fq2 wire_in(const Fq2& a) { return {to_mont(a.c0), to_mont(a.c1)}; }

// a < p, compared limb by limb from the top
__device__ __forceinline__ bool canonical(const Fq& a)
{
    for (int i = 7; i >= 0; i--) {
        if (a.v[i] != FqP::p(i)) return a.v[i] < FqP::p(i);
    }
    return false;
}
__device__ __forceinline__ bool canonical(const Fq2& a) { return canonical(a.c0) && canonical(a.c1); }

template <class F>
__device__ void point_to_wire(const Jac<F>& J, Aff<F>* w)
{
    if (J.Z.is_zero()) { *w = Aff<F>{F::zero(), F::zero()}; return; }
    F zi = inverse(J.Z);
    F zi2 = mul(zi, zi);
    *w = Aff<F>{wire_out(mul(J.X, zi2)), wire_out(mul(J.Y, mul(zi2, zi)))};
}

template <class F>
__device__ void point_from_wire(const Aff<F>& w, Jac<F>* J, uint32_t* bad)
{
    if (w.x.is_zero() && w.y.is_zero()) { *J = Jac<F>{F::zero(), F::one(), F::zero()}; return; }
    if (!canonical(w.x) || !canonical(w.y)) {
        if (bad) *bad = 1u;
        *J = Jac<F>{F::zero(), F::one(), F::zero()};
        return;
    }
    *J = Jac<F>{wire_in(w.x), wire_in(w.y), F::one()};
}

// one thread per proof point: 0 = A, 1 = B, 2 = C
__global__ void k_proof_to_wire(const Jac<Fq>* A, const Jac<Fq2>* B, const Jac<Fq>* C, uint32_t* wire)
{
    Aff<Fq>* w1 = reinterpret_cast<Aff<Fq>*>(wire);
    if (threadIdx.x == 0) point_to_wire(*A, w1);
    if (threadIdx.x == 1) point_to_wire(*B, reinterpret_cast<Aff<Fq2>*>(wire + 16));
    if (threadIdx.x == 2) point_to_wire(*C, reinterpret_cast<Aff<Fq>*>(wire + 48));
}

__global__ void k_proof_from_wire(const uint32_t* wire, Jac<Fq>* A, Jac<Fq2>* B, Jac<Fq>* C, uint32_t* bad)
{
    if (threadIdx.x == 0) point_from_wire(*reinterpret_cast<const Aff<Fq>*>(wire), A, bad);
    if (threadIdx.x == 1) point_from_wire(*reinterpret_cast<const Aff<Fq2>*>(wire + 16), B, bad);
    if (threadIdx.x == 2) point_from_wire(*reinterpret_cast<const Aff<Fq>*>(wire + 48), C, bad);
}

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_groth16_proof_to_wire(const lzk_groth16_proof* proof, void* wire, void* stream)
{
    if (!proof || !wire) return LZK_EINVAL;
    if (reinterpret_cast<uintptr_t>(proof) % 4 || reinterpret_cast<uintptr_t>(wire) % 4) return LZK_EINVAL;
    k_proof_to_wire<<<1, 32, 0, as_stream(stream)>>>(reinterpret_cast<const Jac<Fq>*>(&proof->A),
                                                     reinterpret_cast<const Jac<Fq2>*>(&proof->B),
                                                     reinterpret_cast<const Jac<Fq>*>(&proof->C),
                                                     static_cast<uint32_t*>(wire)); note_launch();
    return launch_status();
}

int lzk_groth16_proof_from_wire(const void* wire, lzk_groth16_proof* proof, uint32_t* bad, void* stream)
{
    if (!proof || !wire) return LZK_EINVAL;
    if (reinterpret_cast<uintptr_t>(proof) % 4 || reinterpret_cast<uintptr_t>(wire) % 4) return LZK_EINVAL;
    if (bad) LZK_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), as_stream(stream)));
    k_proof_from_wire<<<1, 32, 0, as_stream(stream)>>>(static_cast<const uint32_t*>(wire),
                                                       reinterpret_cast<Jac<Fq>*>(&proof->A),
                                                       reinterpret_cast<Jac<Fq2>*>(&proof->B),
                                                       reinterpret_cast<Jac<Fq>*>(&proof->C), bad); note_launch();
    return launch_status();
}

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

size_t lzk_prover_device_bytes(const lzk_prover* p) { return p ? p->bytes + (p->ctx0 ? p->ctx0->bytes : 0) : 0; }

int lzk_poly_a_times_b_minus_c(lzk_fr_t* A, const lzk_fr_t* B, const lzk_fr_t* C, size_t n, void* stream)
{
    if (!n) return LZK_OK;
    if (!A || !B || !C) return LZK_EINVAL;
    k_abc<<<grid_for(n, 256, sm_count() * 8), 256, 0, as_stream(stream)>>>(reinterpret_cast<Fr*>(A), reinterpret_cast<const Fr*>(B),
                                                                     reinterpret_cast<const Fr*>(C), n, nullptr); note_launch();
    return launch_status();
}

int lzk_groth16_prove(lzk_prover* p, const lzk_fr_t* z, const lzk_fr_t* r, const lzk_fr_t* s,
                      lzk_groth16_proof* proof, void* stream)
{
    if (!p) return LZK_EINVAL;
    return prove_ctx(p, p->ctx0, reinterpret_cast<const Fr*>(z), r, s, proof, as_stream(stream));
}

}  // extern "C"
