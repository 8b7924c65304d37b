// Instantiation of the fused stage for one order (BBW_FUSED_N) and one
// element tile (BBW_FUSED_E, 32 or 16): both bases, 8 and 16 warps, every
// operator placement / pipelining variant.
#include "fused_kernel.cuh"

#define BBW_CAT3(a, b, c, d) a##b##c##d
#define BBW_NAME(a, n, e) BBW_CAT3(a, n, _e, e)

namespace bbw {

bbw_status BBW_NAME(fused_prepare_n, BBW_FUSED_N, BBW_FUSED_E)(FusedPlan &pl) {
  return pl.bb ? prepare<BBW_FUSED_N, true, BBW_FUSED_E>(pl)
               : prepare<BBW_FUSED_N, false, BBW_FUSED_E>(pl);
}

bbw_status BBW_NAME(fused_launch_n, BBW_FUSED_N, BBW_FUSED_E)(const FusedPlan &pl, const float *Qin,
                                                              float *Qout, float *res, float fa,
                                                              float fb, float fdt, float cstage,
                                                              cudaStream_t st) {
  return pl.bb
             ? launch_fused<BBW_FUSED_N, true, BBW_FUSED_E>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st)
             : launch_fused<BBW_FUSED_N, false, BBW_FUSED_E>(pl, Qin, Qout, res, fa, fb, fdt, cstage,
                                                             st);
}

}  // namespace bbw
