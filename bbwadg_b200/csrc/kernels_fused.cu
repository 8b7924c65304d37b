// Dispatch of the fused stage over the order N (instantiations in
// kernels_fused_n<N>.cu; kernel template in fused_kernel.cuh).
#include <cuda_runtime.h>

#include "bbwadg.h"
#include "device_common.cuh"
#include "fused.h"

namespace bbw {

#define BBW_DECL1(n, e)                                                                     \
  bbw_status fused_prepare_n##n##_e##e(FusedPlan &pl);                                      \
  bbw_status fused_launch_n##n##_e##e(const FusedPlan &pl, const float *Qin, float *Qout,   \
                                      float *res, float fa, float fb, float fdt, float cstage, \
                                      cudaStream_t st);
#define BBW_DECL(n) BBW_DECL1(n, 32) BBW_DECL1(n, 16)
BBW_DECL(1) BBW_DECL(2) BBW_DECL(3) BBW_DECL(4) BBW_DECL(5) BBW_DECL(6) BBW_DECL(7) BBW_DECL(8)
#undef BBW_DECL
#undef BBW_DECL1

int fused_default_warps(int N) { return N <= 3 ? 8 : 16; }
// 32-element tiles up to N = 7; at N = 8 (Np = 165 and 729 cubature points
// with the Stroud rule) the arrays of a 32-element tile exceed one SM's
// shared memory, those of a 16-element tile fit
int fused_default_tile(int N) { return N <= 7 ? 32 : 16; }

bbw_status fused_prepare(FusedPlan &pl) {
  if (pl.W == 0) pl.W = fused_default_warps(pl.N);
  if (pl.E == 0) pl.E = fused_default_tile(pl.N);
  if (pl.E != 16 && pl.E != 32)
    return set_error(BBW_ERR_ARG, "fused stage: element tile must be 16 or 32");
  const bool e16 = pl.E == 16;
#define CASE(n) \
  case n: return e16 ? fused_prepare_n##n##_e16(pl) : fused_prepare_n##n##_e32(pl);
  switch (pl.N) { CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) }
#undef CASE
  return set_error(BBW_ERR_UNSUPPORTED, "fused stage: N out of range");
}

bbw_status fused_launch(const FusedPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                        float fb, float fdt, float cstage, cudaStream_t st) {
  const bool e16 = pl.E == 16;
#define CASE(n)                                                               \
  case n:                                                                     \
    return e16 ? fused_launch_n##n##_e16(pl, Qin, Qout, res, fa, fb, fdt, cstage, st) \
               : fused_launch_n##n##_e32(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
  switch (pl.N) { CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) }
#undef CASE
  return set_error(BBW_ERR_UNSUPPORTED, "fused stage: N out of range");
}

}  // namespace bbw
