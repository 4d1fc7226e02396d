/* lzk.h -- C ABI of the B200 Groth16 prover hot path (BN254).
 *
 * Drop-in boundary for the operator and protocol layer of LibLightZK
 * (include/operator/msm.cuh, include/operator/poly.cuh,
 * include/protocol/groth16.cuh).  The reference exposes these as C++
 * templates called with device pointers on the default stream; this ABI
 * exposes the same operators as plain extern "C" functions over device
 * pointers, an explicit CUDA stream (passed as void*, may be NULL for the
 * legacy default stream) and an int status.
 *
 * Data layout (bit-identical to the reference's host arithmetic, so host
 * arrays of libff::alt_bn128_* values can be copied to the device as is):
 *   lzk_fr_t / lzk_fq_t  four little-endian 64-bit limbs, Montgomery form
 *                        with R = 2^256 (fp.cuh:33).
 *   lzk_fq2_t            c0 + c1*i, i^2 = -1 (alt_bn128_init.cu:77).
 *   lzk_g1_t, lzk_g2_t   Jacobian (X, Y, Z), the layouts of
 *                        libff::alt_bn128_G1 / alt_bn128_G2
 *                        (alt_bn128_g1.cuh:27, alt_bn128_g2.cuh:28).
 *   lzk_g1_affine_t ...  affine (x, y); the point at infinity is x = y = 0.
 *
 * Every function returns LZK_OK (0) or a negative LZK_E* code and never
 * aborts the process.  Work is enqueued on `stream` and completes
 * asynchronously unless stated otherwise.
 */
#ifndef LZK_H
#define LZK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LZK_OK            0
#define LZK_EINVAL       -1   /* bad argument (size, alignment, null) */
#define LZK_ENOMEM       -2   /* device allocation failed */
#define LZK_ETIMEOUT     -3   /* a bounded device-side wait gave up */
#define LZK_EDEVICE      -4   /* CUDA runtime error */
#define LZK_EUNSUPPORTED -5   /* configuration not supported */
#define LZK_EBUSY        -6   /* busy: pending, or refused by the memory budget */
#define LZK_ECANCELED    -7   /* request cancelled before it started */
#define LZK_EREJECTED    -8   /* request can never fit the memory budget */
#define LZK_EIO          -9   /* a file cannot be read or written, or is not a valid key file */

typedef struct { uint64_t limb[4]; } lzk_fr_t;
typedef struct { uint64_t limb[4]; } lzk_fq_t;
typedef struct { lzk_fq_t c0, c1; } lzk_fq2_t;
typedef struct { lzk_fq_t x, y; } lzk_g1_affine_t;
typedef struct { lzk_fq2_t x, y; } lzk_g2_affine_t;
typedef struct { lzk_fq_t X, Y, Z; } lzk_g1_t;
typedef struct { lzk_fq2_t X, Y, Z; } lzk_g2_t;

/* Human-readable text for a status code. */
const char* lzk_status_string(int status);
/* Library version string. */
const char* lzk_version(void);

/* ---------------------------------------------------------- field ops
 * Element-wise arithmetic on device arrays of n elements: out[i] = a[i] op
 * b[i] (b unused by the unary ops).  Replaces the device mont_t operators
 * (operator*, sqr, +=, -=, cneg, reciprocal, from/to Montgomery;
 * mont_t.cuh:396-430, 208-302, 465-629) and fp2_t's (alt_bn128_t.cuh:
 * 97-224) for code that works on whole vectors.  Elements are in Montgomery
 * form (FROM_MONT returns the canonical integer, TO_MONT takes one); every
 * result is canonical (< p).  The products go through the same device
 * routines as the MSM, NTT and point formulas, so this is also how those
 * routines are checked against host arithmetic.  INV of zero gives zero.
 * out may alias a or b. */
#define LZK_FIELD_FR  0
#define LZK_FIELD_FQ  1
#define LZK_FIELD_FQ2 2   /* elements are lzk_fq2_t */
#define LZK_FOP_ADD       0
#define LZK_FOP_SUB       1
#define LZK_FOP_MUL       2
#define LZK_FOP_SQR       3
#define LZK_FOP_NEG       4
#define LZK_FOP_INV       5
#define LZK_FOP_FROM_MONT 6
#define LZK_FOP_TO_MONT   7
int lzk_field_op(int field, int op, const void* a, const void* b, void* out, size_t n, void* stream);

/* ------------------------------------------------------------------ MSM
 * out = sum_i scalars[i] * bases[i], a Pippenger bucket method with signed
 * c-bit digits, counting-sorted bucket lists and XYZZ accumulation.
 * Replaces multi_scalar_multiplication_g1/_g2 (msm.cuh:210-247).
 *
 * scalars : n Fr elements, Montgomery form (as the reference's MSM takes
 *           them, msm.cuh:83-84).
 * bases   : with flags = 0, n affine points.
 *           With LZK_MSM_PRECOMPUTED, a table of `precomp_windows` shifted
 *           copies: entry (j, i) at bases[j * level_stride + i] holds
 *           2^(j * window_bits) * P_i in affine form -- the layout that
 *           pre_comp_g1/_g2 build (msm.cuh:48-75, points[i + j*length]),
 *           with affine entries.  Every window then shares one set of
 *           buckets, so no doubling chain combines the windows.
 * out     : one Jacobian point (device memory).
 * cfg     : may be NULL (autotuned window width, library-managed scratch).
 */
#define LZK_MSM_PRECOMPUTED 0x1u

/* Layout of the bases (or table entries):
 *   LZK_BASES_AFFINE        lzk_g1_affine_t / lzk_g2_affine_t
 *   LZK_BASES_REF_G1_JAC    the reference's G1 records: Jacobian lzk_g1_t
 *                           (96 B) with Z = 1, as pre_comp_g1 leaves its
 *                           table (msm.cuh:48-61); Z = 0 is infinity
 *   LZK_BASES_REF_G2_LANES  the reference's device G2 records: two 96-B
 *                           halves [X.c0 Y.c0 Z.c0][X.c1 Y.c1 Z.c1] per
 *                           point (alt_bn128_t.cuh:247-256), Z = 1
 * so a reference table built by pre_comp_g1/_g2 is consumed in place. */
#define LZK_BASES_AFFINE        0u
#define LZK_BASES_REF_G1_JAC    1u
#define LZK_BASES_REF_G2_LANES  2u

typedef struct lzk_msm_cfg {
    uint32_t window_bits;     /* c; 0 = autotune.  Must equal the table's
                                 window width with LZK_MSM_PRECOMPUTED.     */
    uint32_t flags;           /* LZK_MSM_* */
    uint32_t precomp_windows; /* shifted copies in the table (PRECOMPUTED) */
    uint32_t base_layout;     /* LZK_BASES_*                                */
    size_t level_stride;      /* points between copies (PRECOMPUTED)        */
    void* workspace;          /* optional device scratch; NULL = allocate
                                 stream-ordered from the device pool        */
    size_t workspace_bytes;
    uint32_t acc_chunk;       /* sorted bucket entries one accumulation
                                 thread adds (power of two, 8..512);
                                 0 = the tuning table (default 64)          */
    uint32_t reduce_run;      /* buckets per lane run in the bucket-
                                 reduction tiles (power of two, 1..16); 0 =
                                 the tuning table (default 4)               */
} lzk_msm_cfg;

int lzk_msm_g1(const lzk_fr_t* scalars, const void* bases, size_t n,
               lzk_g1_t* out, const lzk_msm_cfg* cfg, void* stream);
int lzk_msm_g2(const lzk_fr_t* scalars, const void* bases, size_t n,
               lzk_g2_t* out, const lzk_msm_cfg* cfg, void* stream);
/* Scratch bytes lzk_msm_g1/_g2 need for this n and cfg (group 1 or 2). */
size_t lzk_msm_workspace_bytes(int group, size_t n, const lzk_msm_cfg* cfg);
/* Window width the autotuner picks for an MSM of n points (group 1 or 2,
 * precomputed or not). */
uint32_t lzk_msm_autotune_window(int group, size_t n, uint32_t flags);

/* G1 MSM over plain affine bases that allocates no device memory, for
 * callers that cannot let a library allocate: processes that give all device
 * memory to their own allocator at start-up, and latency-bound request paths
 * that must not wait on the allocator or run out of memory mid-request.  No
 * counterpart in the reference (its MSM allocates scratch on every call,
 * msm.cuh:216-219, with no alternative).
 *
 * Scratch is a fixed LZK_MSM_NOALLOC_SCRATCH_BYTES array in device memory
 * that the library reserves on every GPU that loads it, for the life of the
 * process.  n may be at most LZK_MSM_NOALLOC_MAX_POINTS, and the scratch of
 * the chosen window (window_bits, 0 = autotuned) must fit; otherwise the call
 * returns LZK_EINVAL without queuing work.  The first call on each device
 * (n = 0 is enough) also sets that device up: under CUDA's lazy module
 * loading the MSM kernels are loaded, and their local memory sized, on
 * first use, which can need device memory, so that call runs one small MSM
 * entirely inside the array.  Make it before your allocator reserves the
 * device's memory and before beginning any stream capture (or run with
 * CUDA_MODULE_LOADING=EAGER); after a cudaDeviceReset the set-up is not
 * repeated.  All calls on a device share the
 * array: the counters that must start at zero are cleared by every call, but
 * calls whose work overlaps on the GPU race -- order them. */
#define LZK_MSM_NOALLOC_MAX_POINTS   65536u
#define LZK_MSM_NOALLOC_SCRATCH_BYTES (32u << 20)
int lzk_msm_g1_noalloc(const lzk_fr_t* scalars, const lzk_g1_affine_t* bases, size_t n, lzk_g1_t* out,
                       uint32_t window_bits, void* stream);

/* Build the shifted-copy table for LZK_MSM_PRECOMPUTED: table[j*level_stride
 * + i] = 2^(j*window_bits) * bases[i], affine, j < windows.  Replaces
 * pre_comp_g1/_g2 (msm.cuh:48-75).  level_stride >= n. */
int lzk_g1_precompute(const lzk_g1_affine_t* bases, size_t n, uint32_t window_bits,
                      uint32_t windows, lzk_g1_affine_t* table, size_t level_stride, void* stream);
int lzk_g2_precompute(const lzk_g2_affine_t* bases, size_t n, uint32_t window_bits,
                      uint32_t windows, lzk_g2_affine_t* table, size_t level_stride, void* stream);
/* Windows a table needs for window width c: ceil(255 / c). */
uint32_t lzk_msm_precomp_windows(uint32_t window_bits);

/* Jacobian <-> affine conversion on the device (batch inversion). */
int lzk_g1_to_affine(const lzk_g1_t* in, lzk_g1_affine_t* out, size_t n, void* stream);
int lzk_g2_to_affine(const lzk_g2_t* in, lzk_g2_affine_t* out, size_t n, void* stream);

/* ------------------------------------------------------------------ NTT
 * In-place transform of 2^log_n Fr elements (Montgomery form), natural order
 * in and out.  Replaces number_theory_transformation (poly.cuh:65-73) with
 * the roots of ntt-params.cuh: forward X_k = sum_j a_j w^(jk), w the
 * 2^log_n-th root of the table; inverse uses w^-1 and scales by 2^-log_n;
 * the coset forms evaluate on / interpolate from g*<w>, g = 5
 * (alt_bn128_init.cu:50): COSET_FORWARD multiplies a_j by g^j first,
 * COSET_INVERSE multiplies the result by g^-j.  log_n <= 26. */
#define LZK_NTT_FORWARD       0
#define LZK_NTT_INVERSE       1
#define LZK_NTT_COSET_FORWARD 2
#define LZK_NTT_COSET_INVERSE 3

int lzk_ntt(lzk_fr_t* data, uint32_t log_n, int direction, void* stream);
/* `count` transforms of the same size, transform t at data + t*stride. */
int lzk_ntt_batch(lzk_fr_t* data, uint32_t log_n, uint32_t count, size_t stride, int direction, void* stream);
/* Build this device's twiddle tables for size 2^log_n now (they are
 * otherwise built on first use, synchronously; call before stream capture). */
int lzk_ntt_prepare(uint32_t log_n);
/* The reference's own signature (poly.cuh:65-66): omega_powers is the
 * caller's table (omega_powers[e] = w^e, e < deg/2, as ntt_setup builds it,
 * groth16-operator.cuh:6-31) and factor an optional device scalar applied
 * to every output. */
int lzk_number_theory_transformation(size_t deg, size_t log_deg, lzk_fr_t* coeffs, const lzk_fr_t* omega_powers,
                                     const lzk_fr_t* factor, void* stream);

/* ------------------------------------------------------------------ SpMV
 * R1CS evaluation out = M*z over Fr (Montgomery).  Replaces
 * batch_sparse_matrix_vector_multiplication (poly.cuh:5-30) and its
 * descriptor xpu::spmat_descript (xpu-spmat.cuh:20-25).  Row i covers
 * [row_ptr[i], row_ptr[i+1]); the last row ends at nnz, so both the
 * reference's `rows`-entry row_ptr and a standard rows+1 one work.
 * index_bytes = 8 for the reference's size_t arrays, 4 for uint32. */
typedef struct lzk_csr {
    const lzk_fr_t* val;
    const void* col_idx;
    const void* row_ptr;
    uint64_t rows, cols, nnz;
    uint32_t index_bytes;
    uint32_t reserved;
} lzk_csr;

/* A[i] = A[i] * B[i] - C[i] for i < n (polynomial_A_times_B_minus_C,
 * poly.cuh:75-85). */
int lzk_poly_a_times_b_minus_c(lzk_fr_t* A, const lzk_fr_t* B, const lzk_fr_t* C, size_t n, void* stream);

/* Az, Bz, Cz in one launch; a NULL matrix skips its output. */
int lzk_spmv3(const lzk_csr* A, const lzk_csr* B, const lzk_csr* C, const lzk_fr_t* z,
              lzk_fr_t* Az, lzk_fr_t* Bz, lzk_fr_t* Cz, void* stream);
int lzk_spmv(const lzk_csr* M, const lzk_fr_t* z, lzk_fr_t* out, void* stream);

/* ------------------------------------------------------------ setup path
 * Seeded uniform Fr vector: out[i] is element offset+i of stream
 * (seed, stream_id), drawn like Fp_model::random_element (fp.cuh:789-816)
 * and used as Montgomery limbs.  Deterministic for equal arguments. */
int lzk_random_fr(uint64_t seed, uint64_t stream_id, uint64_t offset, size_t n, lzk_fr_t* out, void* stream);
/* Fixed-base products out[i] = k[i] * G (G the group generator of
 * alt_bn128_init.cu:130-132 / 191-195), affine.  Replaces
 * fix_base_multi_scalar_multiplication_g1/_g2 (msm.cuh:5-46). */
int lzk_g1_fixed_base(const lzk_fr_t* k, size_t n, lzk_g1_affine_t* out, void* stream);
int lzk_g2_fixed_base(const lzk_fr_t* k, size_t n, lzk_g2_affine_t* out, void* stream);
/* Witness solving for circuits whose row i of C starts with the variable it
 * defines (coefficient one): z[def_i] = (A_i z)(B_i z) - (rest of C_i z),
 * for rows [row_begin, row_end), which may only read variables defined by
 * earlier calls. */
int lzk_r1cs_solve(const lzk_csr* A, const lzk_csr* B, const lzk_csr* C, lzk_fr_t* z, uint64_t row_begin,
                   uint64_t row_end, void* stream);
/* *bad_rows (device) = number of rows with (A_i z)(B_i z) != C_i z. */
int lzk_r1cs_check(const lzk_csr* A, const lzk_csr* B, const lzk_csr* C, const lzk_fr_t* z,
                   unsigned long long* bad_rows, void* stream);

/* --------------------------------------------------------------- Groth16
 * Replaces Groth16<...>::Prove (groth16.cuh:154-222).  A prover holds the
 * circuit view, the proving key as resident shifted-copy MSM tables and its
 * scratch; lzk_groth16_prove enqueues one proof on `stream` (internally
 * forked onto two more streams and joined back) with no host round trip.
 * One proof at a time per prover: calls on different streams must be
 * ordered by the caller.
 *
 * mode LZK_PROVE_REFERENCE reproduces the reference chain bit for bit: the
 * 2M-point H path with the (4M)^-1 scale of groth16-operator.cuh:13 and H
 * scalars taken from coefficients M+1..2M-1 (groth16.cuh:168-198).
 * mode LZK_PROVE_STANDARD computes the standard quotient h on the coset
 * 5*<w_M> with size-M transforms and uses h_0..h_{M-2}.
 * Phase 6 (groth16.cuh:211-215) runs on the device. */
#define LZK_PROVE_STANDARD  0
#define LZK_PROVE_REFERENCE 1

typedef struct lzk_groth16_circuit {
    lzk_csr A, B, C;          /* device CSR; rows = constraints <= 2^log_domain */
    uint64_t n_vars;          /* N + 1 (z[0] = 1) */
    uint64_t n_public;        /* k: the L query covers z[k+1 .. N] */
    uint32_t log_domain;      /* M = 2^log_domain, 1..24 */
    uint32_t reserved;
} lzk_groth16_circuit;

typedef struct lzk_groth16_pk {
    const lzk_g1_affine_t* a_query;   /* device, n_vars points       (a1)  */
    const lzk_g1_affine_t* b1_query;  /* device, n_vars               (b1)  */
    const lzk_g2_affine_t* b2_query;  /* device, n_vars               (b2)  */
    const lzk_g1_affine_t* l_query;   /* device, n_vars - n_public - 1 (Kpk) */
    const lzk_g1_affine_t* h_query;   /* device, M - 1                (Z1)  */
    lzk_g1_affine_t alpha1, beta1, delta1;   /* host values */
    lzk_g2_affine_t beta2, delta2;
} lzk_groth16_pk;

typedef struct lzk_groth16_proof {
    lzk_g1_t A;   /* Ar */
    lzk_g2_t B;   /* Bs2 */
    lzk_g1_t C;   /* Krs + HZ */
} lzk_groth16_proof;

typedef struct lzk_prover lzk_prover;

/* window_bits: MSM window of the resident tables (0 = 17).  The query
 * arrays of pk are read only during creation; the circuit's CSR arrays must
 * stay valid while the prover lives. */
int lzk_prover_create(const lzk_groth16_circuit* circuit, const lzk_groth16_pk* pk, int mode,
                      uint32_t window_bits, lzk_prover** out);
int lzk_prover_destroy(lzk_prover* prover);
size_t lzk_prover_device_bytes(const lzk_prover* prover);
/* z: device witness (n_vars Fr); r, s: HOST Fr values (Montgomery);
 * proof: device memory. */
int lzk_groth16_prove(lzk_prover* prover, const lzk_fr_t* z, const lzk_fr_t* r, const lzk_fr_t* s,
                      lzk_groth16_proof* proof, void* stream);

/* Proving keys on disk.  The reference regenerates its key on every run
 * from unseeded randomness (Groth16::Setup, groth16.cuh:48-152); a service
 * saves each circuit's key once and loads it when it makes the circuit's
 * prover (lzk_prover_create reads the key only while it builds its tables,
 * so the loaded copy can be freed right after).
 *
 * File layout (little-endian, version 1): a 128-byte header -- magic
 * "LZKG16PK", u32 version, u32 header size (128), u64 n_vars, u64 n_public,
 * u32 log_domain, u32 0, u64 point counts of the a, b1, b2, l, h queries
 * (n_vars, n_vars, n_vars, n_vars - n_public - 1, 2^log_domain - 1), u64
 * checksum of the body, zeros -- then the body: alpha1, beta1, delta1 (G1
 * affine), beta2, delta2 (G2 affine), and the five query arrays in that
 * order.  Coordinates are the Montgomery limbs of the lzk_* types above.
 *
 * lzk_pk_save writes pk (query arrays in device memory) for a circuit of
 * the given shape; lzk_pk_load checks the header, the sizes and the
 * checksum (LZK_EIO on any mismatch, a missing or short file), copies the
 * arrays into one device allocation owned by *out and fills *view (ready
 * for lzk_prover_create) and *info (may be NULL).  Both are synchronous. */
typedef struct lzk_pk_info {
    uint64_t n_vars, n_public;
    uint32_t log_domain;
    uint32_t version;          /* filled by lzk_pk_load */
} lzk_pk_info;
typedef struct lzk_pk lzk_pk;
int lzk_pk_save(const char* path, const lzk_groth16_pk* pk, const lzk_pk_info* info);
int lzk_pk_load(const char* path, lzk_pk** out, lzk_groth16_pk* view, lzk_pk_info* info);
int lzk_pk_free(lzk_pk* pk);

/* Proof wire format (LZK_PROOF_WIRE_BYTES): the affine coordinates of A, B
 * and C as canonical (not Montgomery) little-endian 256-bit integers, in the
 * order A.x, A.y, B.x.c0, B.x.c1, B.y.c0, B.y.c1, C.x, C.y; a point at
 * infinity is all zeros.  These are the numbers Groth16::Prove prints as its
 * proof (groth16.cuh:219-221, via print() of the affine point).  Both calls
 * take device memory and are enqueued on `stream`.  from_wire writes
 * Jacobian points with Z = 1 (infinity as (0, 1, 0)); a coordinate >= p sets
 * *bad (device uint32, may be NULL) to 1 and decodes that point as
 * infinity. */
#define LZK_PROOF_WIRE_BYTES 256
int lzk_groth16_proof_to_wire(const lzk_groth16_proof* proof, void* wire, void* stream);
int lzk_groth16_proof_from_wire(const void* wire, lzk_groth16_proof* proof, uint32_t* bad, void* stream);

/* -------------------------------------------------------------- serving
 * A prove-request server over resident provers with continuous batching.
 * A worker thread admits queued requests (oldest first) into proof
 * contexts -- an idle context of the request's circuit, or a new one while
 * the device-memory budget allows (idle contexts of other circuits are
 * released to make room) -- and runs each on its own streams, so requests
 * that arrive while others run start as soon as a context and memory are
 * free and their work overlaps on the device.  Resident provers count
 * against the budget when added.  Latency is submission to completion.
 * New relative to the reference, which proves once per process
 * (groth16.cuh:48-222). */
typedef struct lzk_server lzk_server;

typedef struct lzk_server_cfg {
    size_t hbm_budget_bytes;   /* resident provers + all proof contexts */
    uint32_t max_inflight;     /* proofs running at once */
    uint32_t reserved;
} lzk_server_cfg;

typedef struct lzk_server_stats {
    uint64_t submitted, completed, rejected, cancelled, queued, running;
    size_t device_bytes;       /* resident + contexts in use or cached */
    double p50_ms, p99_ms, mean_ms, max_ms;
    double proofs_per_s;       /* completed / (last completion - first submission) */
} lzk_server_stats;

/* the witness is pinned host memory that stays unchanged until the request
 * completes (otherwise the server copies it at submission) */
#define LZK_REQ_WITNESS_PINNED 0x1u

int lzk_server_create(const lzk_server_cfg* cfg, lzk_server** out);
/* The prover stays owned by the caller and must outlive the server. */
int lzk_server_add_circuit(lzk_server* server, lzk_prover* prover, uint32_t* circuit_id);
/* z: HOST witness (n_vars Fr); r, s: host values. */
int lzk_server_submit(lzk_server* server, uint32_t circuit_id, const lzk_fr_t* z, const lzk_fr_t* r,
                      const lzk_fr_t* s, uint32_t flags, uint64_t* request_id);
/* LZK_OK: done, *proof (host) filled, request forgotten; LZK_EBUSY: not done;
 * LZK_ECANCELED / LZK_EREJECTED: finished without a proof (forgotten). */
int lzk_server_poll(lzk_server* server, uint64_t request_id, lzk_groth16_proof* proof, double* latency_ms);
/* cancel a request that has not started (LZK_EBUSY once it has) */
int lzk_server_cancel(lzk_server* server, uint64_t request_id);
/* wait until nothing is queued or running; LZK_ETIMEOUT after timeout_ms */
int lzk_server_wait_idle(lzk_server* server, int timeout_ms);
int lzk_server_get_stats(lzk_server* server, lzk_server_stats* stats);
int lzk_server_reset_stats(lzk_server* server);
/* drops queued requests, waits for running ones, frees all contexts */
int lzk_server_destroy(lzk_server* server);

/* ------------------------------------------------------------ batching
 * Many MSMs (one group: 1 = G1, 2 = G2; plain affine bases) and NTTs of
 * uneven sizes as one plan.  All MSMs share one global bucket space, so each
 * MSM phase is a single launch for the whole batch; NTTs are grouped by
 * (size, direction) on a second stream.  The plan allocates everything when
 * it is created, so running it is launches only; with use_graph the plan
 * captures those launches into a CUDA graph on the first run (stream must
 * then be a created stream, not the legacy default) and replays it after.
 * The descriptors' buffers must stay valid while the plan lives; their
 * contents may change between runs.  Extends the reference's one-call-per-
 * operator interface (msm.cuh:210-247, poly.cuh:65-73). */
typedef struct lzk_msm_desc {
    const lzk_fr_t* scalars;   /* device, n Fr (Montgomery) */
    const void* bases;         /* device, n affine points */
    size_t n;
    void* out;                 /* device, one Jacobian point */
    uint32_t window_bits;      /* 0 = autotuned */
    uint32_t reserved;
} lzk_msm_desc;

typedef struct lzk_ntt_desc {
    lzk_fr_t* data;            /* device, 2^log_n Fr, transformed in place */
    uint32_t log_n;
    int direction;             /* LZK_NTT_* */
} lzk_ntt_desc;

typedef struct lzk_batch_plan lzk_batch_plan;

int lzk_batch_plan_create(int group, const lzk_msm_desc* msms, size_t n_msm, const lzk_ntt_desc* ntts, size_t n_ntt,
                          lzk_batch_plan** out);
/* The same with flags.  LZK_BATCH_FIXED_BASES: the MSMs' bases are read once,
 * at creation, into shifted-copy tables (as lzk_g1_precompute builds; the
 * plan then holds sum_k n_k * ceil(255 / c_k) points), so every window of an
 * MSM shares one bucket set and no window combination remains; later
 * changes to the bases arrays are not seen (the scalars are still read at
 * every run).  For bases that stay fixed, such as a proving key's queries.
 * Window widths come from LZK_TUNE_MSM_TABLE_WINDOW. */
#define LZK_BATCH_FIXED_BASES 0x1u
/* LZK_BATCH_PERSISTENT: the MSM phases after the digit sort (accumulation,
 * fix-up, the bucket reductions of every window width, the window
 * combination) run as one cooperative persistent launch of exactly the
 * blocks the device holds at once, with a grid-wide barrier between phases,
 * instead of nine launches.  Its barrier waits are bounded (about 2 s; then
 * LZK_ETIMEOUT).  Runs are eager and synchronous (use_graph is ignored); at
 * most 20 distinct window widths (else LZK_EUNSUPPORTED at creation).  The
 * NTTs still run on a second stream beside it. */
#define LZK_BATCH_PERSISTENT 0x2u
int lzk_batch_plan_create_ex(int group, const lzk_msm_desc* msms, size_t n_msm, const lzk_ntt_desc* ntts,
                             size_t n_ntt, uint32_t flags, lzk_batch_plan** out);
int lzk_batch_plan_run(lzk_batch_plan* plan, int use_graph, void* stream);
size_t lzk_batch_plan_device_bytes(const lzk_batch_plan* plan);
int lzk_batch_plan_destroy(lzk_batch_plan* plan);

/* Tuning table.  Per knob, group (1 = G1, 2 = G2; ignored for NTT knobs)
 * and size class log_n = ceil(log2 n), the value an operator uses when its
 * configuration leaves it open:
 *   LZK_TUNE_MSM_WINDOW      window width of plain-base MSMs (cfg
 *                            window_bits = 0); unset: the cost model
 *   LZK_TUNE_MSM_CHUNK       sorted entries per accumulation thread of a
 *                            plain-base MSM (cfg acc_chunk = 0), 8..512,
 *                            power of two; unset: 64
 *   LZK_TUNE_MSM_REDUCE_RUN  buckets per lane run in the reduction tiles of
 *                            a plain-base MSM (cfg reduce_run = 0), 1..16;
 *                            unset: 4
 *   LZK_TUNE_NTT_BLOCK       elements per block of an NTT pass (the stages
 *                            a pass runs in shared memory), 256..4096, power
 *                            of two; unset: 2048
 *   LZK_TUNE_MSM_TABLE_WINDOW window width of MSMs over shifted-copy tables
 *                            that leave it open (batch plans with
 *                            LZK_BATCH_FIXED_BASES); unset: the cost model
 *   LZK_TUNE_MSM_TABLE_CHUNK, LZK_TUNE_MSM_TABLE_RUN
 *                            chunk and run of MSMs over shifted-copy tables
 *                            (LZK_MSM_PRECOMPUTED, Groth16 provers, fixed-
 *                            base batch plans), whose single bucket set
 *                            wants other values than a plain MSM's per-
 *                            window sets; unset: 64 and 4
 * The reference fixes all of these at compile time (c = 12 with 4096
 * buckets, msm.cuh:216-227; one launch per NTT stage, poly.cuh:42-63).
 * value 0 clears an entry.  A Groth16 prover and a batch plan read the table
 * once, when they are created.  Filled from device timings by
 * liblightzk_b200.autotune. */
#define LZK_TUNE_MSM_WINDOW     0
#define LZK_TUNE_MSM_CHUNK      1
#define LZK_TUNE_MSM_REDUCE_RUN 2
#define LZK_TUNE_NTT_BLOCK      3
#define LZK_TUNE_MSM_TABLE_WINDOW 4
#define LZK_TUNE_MSM_TABLE_CHUNK  5
#define LZK_TUNE_MSM_TABLE_RUN    6
int lzk_tune_set(int knob, int group, uint32_t log_n, uint32_t value);
/* The value in effect (the entry, or the default; 0 for an unset window). */
uint32_t lzk_tune_get(int knob, int group, uint32_t log_n);
/* lzk_tune_set(LZK_TUNE_MSM_WINDOW, group, log_n, window_bits). */
int lzk_msm_set_window(int group, uint32_t log_n, uint32_t window_bits);

/* ------------------------------------------------------------ tracing
 * Opt-in CUDA-event timing of named device regions ("msm_g1",
 * "msm_g1_accumulate", "msm_g2", "msm_g2_accumulate", "groth16_prove").
 * Replaces the reference's synchronising Timer/CUDA_DEBUG pairs
 * (timer.cu:3-16, device-utils.cuh:3). */
void lzk_trace_enable(int on);
/* NVTX ranges for the same named regions (independent of
 * lzk_trace_enable): each region's host-side enqueue -- the calls that
 * launch its kernels -- becomes one NVTX range (nvtxRangeStartA/End, so
 * regions on different streams may overlap), which a profiler such as
 * Nsight Systems shows beside the kernels they launched.  Off by default;
 * without a profiler attached a range costs a few nanoseconds. */
void lzk_trace_nvtx(int on);
/* Restrict tracing to the comma-separated region names (NULL or "" = all
 * regions).  Every traced region records two timing events in its stream,
 * which costs a few microseconds of stream ordering each (about 1 % of a
 * proof with every region traced), so throughput measurements trace only
 * the regions they read. */
int lzk_trace_only(const char* names);
void lzk_trace_reset(void);
/* Total device milliseconds and count of completed regions named `name`
 * since the last reset (waits for pending regions). */
int lzk_trace_get(const char* name, double* total_ms, uint64_t* count);
/* The completed regions since the last reset as a timeline: device
 * milliseconds from the start of the first region begun after the reset,
 * in completion-resolution order (at most 65 536 kept).  Writes up to `cap`
 * spans and sets *count to the number held.  Shows which stream's work ends
 * a multi-stream call such as a proof. */
typedef struct lzk_trace_span {
    char name[40];
    double start_ms;
    double end_ms;
} lzk_trace_span;
int lzk_trace_timeline(lzk_trace_span* spans, size_t cap, size_t* count);
/* Testing hook: after `after` more device allocations, every allocation
 * the library makes fails as if the device were out of memory (LZK_ENOMEM
 * from the call that needed it, with everything it had allocated released);
 * a negative value turns the failures off.  Process-wide. */
int lzk_debug_fail_allocations(long long after);
/* Test hook of the persistent batch launch (LZK_BATCH_PERSISTENT): every
 * grid barrier also waits for extra_arrivals arrivals that never come (0 =
 * normal) and gives up after max_polls polls (0 = the default, about 2 s),
 * so a test can make the bounded waits run out and see LZK_ETIMEOUT without
 * any fault.  No counterpart in the reference. */
int lzk_debug_persistent_barrier(uint32_t extra_arrivals, uint32_t max_polls);
/* Debug builds (liblzk_b200_debug.so, compiled with LZK_DEBUG_CHECKS): the
 * digit sort, bucket accumulation and fix-up kernels check every index their
 * inputs imply and, instead of an out-of-range read or write, set a bit of a
 * device error word and skip the access.  lzk_debug_check_word returns the
 * bits set since it was last cleared on the current device (bit 0: bucket
 * index, 1: scatter slot, 2: base index of a sorted entry, 3: bucket offset,
 * 4: fix-up partial), clearing them when clear != 0; always 0 in release
 * builds, which lzk_debug_checks_enabled tells apart (1 = checks compiled
 * in).  The reference's counterparts are its CUDA_DEBUG prints and device
 * traps (device-utils.cuh:3, mont_t.cuh:1108). */
uint32_t lzk_debug_check_word(int clear);
int lzk_debug_checks_enabled(void);
/* Number of kernels this library has launched so far (all devices). */
uint64_t lzk_launch_count(void);
/* Measured 32-bit integer multiply-add rate of the current device
 * (mad.lo/madc.hi operations per second); synchronous. */
int lzk_probe_imad_rate(double* ops_per_s);
/* Measured rate of Fq Montgomery products per second on the current device
 * in the fastest form this library has: the radix-2^52 product on the FP64
 * pipe with operands already in limb form (independent products, full
 * occupancy); synchronous. */
int lzk_probe_mont_rate(double* products_per_s);
/* The same for the 32-bit-limb integer product (wide multiplies on the
 * integer multiplier); synchronous. */
int lzk_probe_mont_rate_int(double* products_per_s);

#ifdef __cplusplus
}
#endif

#endif /* LZK_H */
