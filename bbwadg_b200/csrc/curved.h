// Internal interface of the fused curved-element stage (kernels_curved.cu),
// used by the curvilinear solver handle (capi_curved.cu).
#pragma once
#include <cuda_runtime.h>

#include "bbwadg.h"

namespace bbw {

// One LSRK stage of the curved elements k = k_off + i, i < KC.  Geometry rows
// are compact (row i): vgeoq [KC][9][Nq], Jq [KC][Nq], fgeoq [KC][4][4][Nfq],
// Jr / c2q [KC][Nr] at the update's cubature.  Operators column-major as the
// reference uploads them; vmapP [K][4Nfp] in the handle's element order.
struct CurvedStageArgs {
  int KC, k_off, Nq, Nfq, Nr, EB;
  const float *vgeoq, *Jq, *fgeoq, *Jr, *c2q;
  const float *Vq, *Vrq, *Vsq, *Vtq, *Pq, *Prq, *Psq, *Ptq, *VfqFace, *Pfq, *Vqr, *Pqr;
  const int *Fmask, *vmapP;
  float fa, fb, fdt;
};

// reads Qold (own element and neighbour traces), writes Qnew and res of the
// KC curved elements
bbw_status curved_stage(int N, const CurvedStageArgs &A, const float *Qold, float *Qnew,
                        float *res, cudaStream_t st);

}  // namespace bbw
