// Host-visible description of a prepared fused-stage launch (kernels_fused.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "bbwadg.h"

namespace bbw {

// element-tile row stride (floats) of the fused kernel's shared-memory arrays
constexpr int kFusedRowStride = 33;

struct FusedPlan {
  int N = 0, K = 0, Nq = 0, RQ = 0, PRQ = 0, bc = 0, npat = 0;
  bool bb = false, pipe = false;
  int grid = 0;
  size_t smem = 0;
  const float *vgeo = nullptr, *fgeo = nullptr, *c2q = nullptr;
  const int *nbr = nullptr;
  const float *ops = nullptr;
  int ops_floats = 0, ops_smem = 0;     // total / staged in shared memory
  int off_lift = 0, off_pq = 0, off_vq = 0;
  const int *tables = nullptr;
  int table_ints = 0, pat_off = 0, bb_off = 0;
};

int fused_warps(int N);
bbw_status fused_prepare(FusedPlan &pl);
bbw_status fused_launch(const FusedPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                        float fb, float fdt, cudaStream_t st);

}  // namespace bbw
