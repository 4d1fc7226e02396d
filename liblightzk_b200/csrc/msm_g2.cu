// msm_g2.cu -- G2 instantiation of the MSM, the shifted-base table
// builder and the Jacobian -> affine converter (templates in msm.cuh).
#include "msm.cuh"

using namespace lzk;

namespace lzk {
uint32_t debug_word_g2(bool clear) { return debug_word_here(clear); }

int msm_g2_presorted(const Fr* scalars, const void* table, size_t n, Jac<Fq2>* out, const lzk_msm_cfg* cfg,
                     cudaStream_t st, const uint32_t* off, const uint32_t* ent)
{
    if (!cfg || !(cfg->flags & LZK_MSM_PRECOMPUTED) || !off || !ent) return LZK_EINVAL;
    return run_msm<G2>(scalars, table, n, out, cfg, st, cfg->window_bits, off, ent);
}
}  // namespace lzk

extern "C" {

int lzk_msm_g2(const lzk_fr_t* scalars, const void* bases, size_t n, lzk_g2_t* out,
               const lzk_msm_cfg* cfg, void* stream)
{
    bool shared = cfg && (cfg->flags & LZK_MSM_PRECOMPUTED);
    return run_msm<G2>(reinterpret_cast<const Fr*>(scalars), bases, n,
                       reinterpret_cast<Jac<Fq2>*>(out), cfg, as_stream(stream), msm_autotune(2, n, shared));
}

int lzk_g2_precompute(const lzk_g2_affine_t* bases, size_t n, uint32_t window_bits, uint32_t windows,
                      lzk_g2_affine_t* table, size_t level_stride, void* stream)
{
    return run_precompute<Fq2>(reinterpret_cast<const Aff<Fq2>*>(bases), n, window_bits, windows,
                               reinterpret_cast<Aff<Fq2>*>(table), level_stride, as_stream(stream));
}

int lzk_g2_to_affine(const lzk_g2_t* in, lzk_g2_affine_t* out, size_t n, void* stream)
{
    if ((!in || !out) && n) return LZK_EINVAL;
    if (!n) return LZK_OK;
    k_jac_to_aff<Fq2><<<grid_for((n + 7) / 8, 128), 128, 0, as_stream(stream)>>>(
        reinterpret_cast<const Jac<Fq2>*>(in), reinterpret_cast<Aff<Fq2>*>(out), n); note_launch();
    return launch_status();
}

}  // extern "C"
