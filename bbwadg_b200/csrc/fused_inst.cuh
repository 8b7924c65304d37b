// Instantiation of the fused stage for one order (BBW_FUSED_N), both bases,
// 8 and 16 warps, every operator placement / pipelining variant.
#include "fused_kernel.cuh"

#define BBW_CAT2(a, b) a##b
#define BBW_CAT(a, b) BBW_CAT2(a, b)

namespace bbw {

bbw_status BBW_CAT(fused_prepare_n, BBW_FUSED_N)(FusedPlan &pl) {
  return pl.bb ? prepare<BBW_FUSED_N, true>(pl) : prepare<BBW_FUSED_N, false>(pl);
}

bbw_status BBW_CAT(fused_launch_n, BBW_FUSED_N)(const FusedPlan &pl, const float *Qin, float *Qout,
                                                float *res, float fa, float fb, float fdt,
                                                float cstage, cudaStream_t st) {
  return pl.bb ? launch_fused<BBW_FUSED_N, true>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st)
               : launch_fused<BBW_FUSED_N, false>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
}

}  // namespace bbw
