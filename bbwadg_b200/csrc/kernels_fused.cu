// Dispatch of the fused stage over the order N (instantiations in
// kernels_fused_n<N>.cu; kernel template in fused_kernel.cuh).
#include <cuda_runtime.h>

#include "bbwadg.h"
#include "device_common.cuh"
#include "fused.h"

namespace bbw {

#define BBW_DECL(n)                                                                         \
  bbw_status fused_prepare_n##n(FusedPlan &pl);                                             \
  bbw_status fused_launch_n##n(const FusedPlan &pl, const float *Qin, float *Qout, float *res, \
                               float fa, float fb, float fdt, float cstage, cudaStream_t st);
BBW_DECL(1) BBW_DECL(2) BBW_DECL(3) BBW_DECL(4) BBW_DECL(5) BBW_DECL(6) BBW_DECL(7) BBW_DECL(8)
#undef BBW_DECL

int fused_default_warps(int N) { return N <= 3 ? 8 : 16; }

bbw_status fused_prepare(FusedPlan &pl) {
  if (pl.W == 0) pl.W = fused_default_warps(pl.N);
  switch (pl.N) {
    case 1: return fused_prepare_n1(pl);
    case 2: return fused_prepare_n2(pl);
    case 3: return fused_prepare_n3(pl);
    case 4: return fused_prepare_n4(pl);
    case 5: return fused_prepare_n5(pl);
    case 6: return fused_prepare_n6(pl);
    case 7: return fused_prepare_n7(pl);
    case 8: return fused_prepare_n8(pl);
  }
  return set_error(BBW_ERR_UNSUPPORTED, "fused stage: N out of range");
}

bbw_status fused_launch(const FusedPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                        float fb, float fdt, float cstage, cudaStream_t st) {
#define CALL(n) fused_launch_n##n(pl, Qin, Qout, res, fa, fb, fdt, cstage, st)
  switch (pl.N) {
    case 1: return CALL(1);
    case 2: return CALL(2);
    case 3: return CALL(3);
    case 4: return CALL(4);
    case 5: return CALL(5);
    case 6: return CALL(6);
    case 7: return CALL(7);
    case 8: return CALL(8);
  }
#undef CALL
  return set_error(BBW_ERR_UNSUPPORTED, "fused stage: N out of range");
}

}  // namespace bbw
