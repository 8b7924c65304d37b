// Host-visible description of a prepared fused-stage launch (kernels_fused.cu).
#pragma once
#include <cuda_fp16.h>

#include <cstdint>
#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "bbwadg.h"

namespace bbw {

struct FusedPlan {
  int N = 0, K = 0, Nq = 0, RQ = 0, PRQ = 0, bc = 0, npat = 0;
  int W = 0;                            // warps per CTA (8 or 16; 0 = default for N)
  int E = 0;                            // elements per tile (16 or 32; 0 = default for N)
  int Kc = 0;                           // elements advanced (0 = all K; rest are halo copies)
  int K0 = 0;                           // first element advanced (a launch covers [K0, Kc))
  int want_ops = -1, want_pipe = -1;    // requested placement (-1: first that fits)
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
  int S = 1, nsm = 148;  // shots per launch, SM count
  int max_ctas = 0;      // cap on the persistent grid (0: one CTA per SM)
  const int *src_off = nullptr, *src_elem = nullptr;  // sources (null: none)
  const float *src_vec = nullptr;
  float f0 = 0.f, tR = 0.f, samp = 0.f;
  const double *time = nullptr;
  float *vq_out = nullptr;  // [S][Nq][K] pre-c2 cubature values of rhs_p (adjoint recomputation)
};

int fused_default_warps(int N);
int fused_default_tile(int N);
// cubature rows per accumulator block of the fused kernel's Vq product, by
// the number of thread groups (row blocks) per CTA
__host__ __device__ constexpr int fused_vq_block(int groups) { return groups == 8 ? 12 : 8; }
// thread groups of a fused-stage CTA: W warps, one thread per element of an
// E-element tile
constexpr int fused_groups(int W, int E) { return 32 * W / E; }

// operators packed per thread group for a fused kernel with G groups (capi.cu)
struct FusedOps {
  std::vector<float> ops;
  int off_lift = 0, off_pq = 0, off_vq = 0, RQ = 0, PRQ = 0;
};
void pack_fused_ops(int N, int Nq, int G, bool bb, const float *Dr, const float *Ds,
                    const float *Dt, const float *LIFT, const float *Vq, const float *Pq,
                    FusedOps &out);

// ---- tensor-core (tcgen05) stage, kernels_tc.cu
constexpr int TC_GEO = 28;  // floats per element geometry record: fgeo 16 | vgeo 9 | pad 3

struct TcLayout {
  int KV = 0, KF = 0, KQ = 0, MQ = 0;   // padded K extents, rows of the Vq MMA (64 or 128)
  int MR = 0, MRQ = 0;                  // operator rows stored: Np and Nq rounded up (see tc_layout)
  int oD = 0, oL = 0, oPq = 0, oVq = 0; // operator offsets (halves)
  int ops_halfs = 0;
  int ops = 0, Bp = 0, BU = 0, BF = 0, BW = 0, raw = 0, geo = 0, nbr = 0, tab = 0, misc = 0;  // bytes
  int total = 0;
};

struct TcPlan {
  int N = 0, K = 0, Nq = 0, bc = 0, grid = 0, nsm = 148;
  int S = 1;         // shots per launch (state [S][K][4][Np])
  int max_ctas = 0;  // cap on the persistent grid (0: one CTA per SM)
  TcLayout L;
  const float *geo = nullptr, *c2q = nullptr;
  const int *nbr = nullptr, *tables = nullptr;
  const void *ops = nullptr;
  bool bf = false;  // split-BF16 operands instead of split-FP16
  int table_ints = 0, pat_off = 0;
  int *err = nullptr;
  // sources, as FusedPlan (null: none)
  const int *src_tile = nullptr, *src_elem = nullptr;  // [S * ntiles + 1] entries per item
  const float *src_vec = nullptr;
  float f0 = 0.f, tR = 0.f, samp = 0.f;
  const double *time = nullptr;
  float *vq_out = nullptr;  // [S][Nq][K] pre-c2 cubature values of rhs_p (adjoint recomputation)
};

TcLayout tc_layout(int N, int Nq, int table_ints);
bool tc_supported(int N, int Nq);
bbw_status tc_prepare(TcPlan &pl);
bbw_status tc_launch(const TcPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                     float fb, float fdt, float cstage, cudaStream_t st);
void tc_pack_operator(const float *A, int nrows, int ncols, int ld_row, int ld_col, int rows,
                      int kp, uint16_t *hi, uint16_t *lo, bool bf);
bbw_status fused_prepare(FusedPlan &pl);
bbw_status fused_launch(const FusedPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                        float fb, float fdt, float cstage, cudaStream_t st);
// receivers of all shots after a step, then time += dt, step += 1
// state copies of listed elements (all shots) to / from a packed buffer
bbw_status gather_elements(int Np, int K, int S, const float *Q, int n, const int *idx,
                           float *buf, cudaStream_t st);
bbw_status scatter_elements(int Np, int K, int S, float *Q, int n, const int *idx,
                            const float *buf, cudaStream_t st);
bbw_status record_and_advance(int N, int K, int S, const float *Q, int R, const int *rec_elem,
                              const float *rec_w, float *traces, int max_steps, double *time,
                              int *step, float dt, cudaStream_t st);

}  // namespace bbw
