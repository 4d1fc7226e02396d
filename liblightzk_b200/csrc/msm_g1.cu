// msm_g1.cu -- G1 instantiation of the MSM, the shifted-base table
// builder and the Jacobian -> affine converter (templates in msm.cuh).
#include "msm.cuh"

using namespace lzk;

namespace lzk {
uint32_t debug_word_g1(bool clear) { return debug_word_here(clear); }

int msm_g1_presorted(const Fr* scalars, const void* table, size_t n, Jac<Fq>* out, const lzk_msm_cfg* cfg,
                     cudaStream_t st, const uint32_t* off, const uint32_t* ent)
{
    if (!cfg || !(cfg->flags & LZK_MSM_PRECOMPUTED) || !off || !ent) return LZK_EINVAL;
    return run_msm<G1>(scalars, table, n, out, cfg, st, cfg->window_bits, off, ent);
}

int msm_g1_concat(const Fr* lo, size_t n_lo, const Fr* hi, size_t n_hi, const void* table, Jac<Fq>* out,
                  const lzk_msm_cfg* cfg, cudaStream_t st)
{
    size_t n = n_lo + n_hi;
    if (!cfg || !(cfg->flags & LZK_MSM_PRECOMPUTED) || !cfg->workspace || !out || !table) return LZK_EINVAL;
    if ((n_lo && !lo) || (n_hi && !hi) || n == 0 || n >= (1ull << 31)) return LZK_EINVAL;
    uint32_t c = cfg->window_bits;
    if (c < 2 || c > 24 || cfg->precomp_windows < windows_for(c) || cfg->level_stride < n) return LZK_EINVAL;
    if ((size_t)windows_for(c) * cfg->level_stride >= (1ull << 31)) return LZK_EINVAL;
    MsmPlan p;
    plan_msm<G1>(p, n, c, true, cfg->level_stride, msm_chunk(cfg, 1, n), msm_run(cfg, 1, n));
    if (cfg->workspace_bytes < p.bytes) return LZK_EINVAL;
    // sort into the workspace at the offsets run_msm carves from it
    char* base = static_cast<char*>(cfg->workspace);
    uint32_t* off = reinterpret_cast<uint32_t*>(base + p.o_off);
    uint32_t* ent = reinterpret_cast<uint32_t*>(base + p.o_ent);
    void* tr = trace_begin("msm_g1_sort", st);
    LZK_TRY(msm_sort(p, n_lo ? lo : hi, reinterpret_cast<uint32_t*>(base + p.o_cnt), off, ent,
                     reinterpret_cast<uint32_t*>(base + p.o_scan), st, hi, n_lo));
    trace_end(tr, st);
    return run_msm<G1>(n_lo ? lo : hi, table, n, out, cfg, st, c, off, ent);
}
}  // namespace lzk

extern "C" {

int lzk_msm_g1(const lzk_fr_t* scalars, const void* bases, size_t n, lzk_g1_t* out,
               const lzk_msm_cfg* cfg, void* stream)
{
    bool shared = cfg && (cfg->flags & LZK_MSM_PRECOMPUTED);
    return run_msm<G1>(reinterpret_cast<const Fr*>(scalars), bases, n,
                       reinterpret_cast<Jac<Fq>*>(out), cfg, as_stream(stream), msm_autotune(1, n, shared));
}

int lzk_g1_precompute(const lzk_g1_affine_t* bases, size_t n, uint32_t window_bits, uint32_t windows,
                      lzk_g1_affine_t* table, size_t level_stride, void* stream)
{
    return run_precompute<Fq>(reinterpret_cast<const Aff<Fq>*>(bases), n, window_bits, windows,
                              reinterpret_cast<Aff<Fq>*>(table), level_stride, as_stream(stream));
}

int lzk_g1_to_affine(const lzk_g1_t* in, lzk_g1_affine_t* out, size_t n, void* stream)
{
    if ((!in || !out) && n) return LZK_EINVAL;
    if (!n) return LZK_OK;
    k_jac_to_aff<Fq><<<grid_for((n + 7) / 8, 128), 128, 0, as_stream(stream)>>>(
        reinterpret_cast<const Jac<Fq>*>(in), reinterpret_cast<Aff<Fq>*>(out), n); note_launch();
    return launch_status();
}

}  // extern "C"
