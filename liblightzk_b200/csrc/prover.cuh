// prover.cuh -- the Groth16 prover's resident state and per-proof contexts,
// shared by the prove chain (groth16.cu) and the serving loop (server.cu).
#pragma once
#include "common.cuh"
#include "curve.cuh"
#include "r1cs.cuh"

struct lzk_prover;
namespace lzk {
// the MSM configuration of the prover's workspace i (see lzk_prover::chunk)
lzk_msm_cfg prover_msm_cfg(const lzk_prover* p, int i, size_t level_stride);
}

namespace lzk {

// Scratch and streams of one proof in flight.  A prover owns one (used by
// lzk_groth16_prove); the serving loop creates more, one per admitted
// request, all sharing the prover's resident tables.
struct ProveCtx {
    Fr* x = nullptr;                  // 3 * L: A z, B z, C z and the H polynomial
    Jac<Fq>* g1res = nullptr;         // A, B1 and L + H MSM results
    Jac<Fq2>* g2res = nullptr;        // B2 MSM result
    XYZZ<Fq>* sm1 = nullptr;          // r d1, s a1, r b1, (r s) d1, s A, r B1
    XYZZ<Fq2>* sm2 = nullptr;         // s d2
    void* ws[3] = {nullptr, nullptr, nullptr};
    size_t wsb[3] = {0, 0, 0};
    // one digit sort of the witness, shared by the A, B1 and B2 MSMs
    uint32_t *zs_cnt = nullptr, *zs_off = nullptr, *zs_ent = nullptr, *zs_bsums = nullptr;
    Fr* z = nullptr;                  // witness buffer (serving contexts only)
    lzk_groth16_proof* proof = nullptr;   // proof buffer (serving contexts only)
    lzk_groth16_proof* proof_host = nullptr;   // pinned copy target (serving contexts only)
    cudaEvent_t ev_done = nullptr;             // end of the proof on s0 (serving contexts only)
    cudaStream_t s0 = nullptr, s1 = nullptr, s2 = nullptr, s3 = nullptr;   // s0: serving contexts only
    cudaEvent_t ev_fork = nullptr, ev_b1 = nullptr, ev_s1 = nullptr, ev_s2 = nullptr, ev_s3 = nullptr,
                ev_sorted = nullptr;
    size_t bytes = 0;
};

}  // namespace lzk

struct lzk_prover {
    int mode = 0;
    lzk::CsrDev A, B, C;
    uint64_t rows = 0, n_vars = 0, n_public = 0;
    uint32_t log_m = 0;
    size_t M = 0, L = 0;
    // shifted-copy tables: a, b1, l and h concatenated (G1), b2 (G2); tn =
    // level strides
    lzk::Aff<lzk::Fq>* tab[3] = {nullptr, nullptr, nullptr};
    size_t tn[3] = {0, 0, 0};
    size_t nl = 0;          // points of the l query (n_vars - n_public - 1)
    lzk::Aff<lzk::Fq2>* tab2 = nullptr;
    size_t tn2 = 0;
    uint32_t c = 16, wins = 16;
    // accumulation chunk and reduction run of the three MSM workspaces (0:
    // the L + H MSM, 1: A and B1, 2: B2), read from the tuning table when
    // the prover is made
    uint32_t chunk[3] = {0, 0, 0}, run[3] = {0, 0, 0};
    // constants in device memory
    lzk::Aff<lzk::Fq>* g1c = nullptr;   // alpha1, beta1, delta1
    lzk::Aff<lzk::Fq2>* g2c = nullptr;  // beta2, delta2
    lzk::Fr* zinv = nullptr;            // (g^M - 1)^-1
    lzk::Aff<lzk::Fq>* comb1 = nullptr;   // comb tables of a1, b1, d1 (3 x 8192)
    lzk::Aff<lzk::Fq2>* comb2 = nullptr;  // comb table of d2
    lzk::ProveCtx* ctx0 = nullptr;
    size_t bytes = 0;       // resident bytes (tables, constants)
};

namespace lzk {

// scratch (and, for serving, streams and witness/proof buffers) of one proof
int ctx_create(const lzk_prover* p, bool serving, ProveCtx** out);
void ctx_destroy(ProveCtx* x);
// enqueue one proof on stream st using context x (x's side streams join st)
int prove_ctx(const lzk_prover* p, ProveCtx* x, const Fr* z, const lzk_fr_t* r, const lzk_fr_t* s,
              lzk_groth16_proof* proof, cudaStream_t st);

}  // namespace lzk
