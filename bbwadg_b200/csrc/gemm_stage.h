// Precision-study form of the stage (gemm_stage.cu): the dense contractions
// over all elements as cuBLAS GEMMs (split FP16 or split BF16 with three
// products per pair, or TF32), flux, operand splits and the LSRK update in
// this library's kernels.  Used where the fused tensor-core stage does not
// fit one SM (N >= 6) and for TF32 at every order.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "bbwadg.h"

namespace bbw {

struct GemmStage {
  int N = 0, K = 0, Nq = 0, Np = 0, Nfp = 0, bc = 0, precision = 0;
  void *handle = nullptr;  // cublasHandle_t
  void *workspace = nullptr;
  size_t workspace_bytes = 0;
  // operators: FP32 copies (TF32) or hi / lo planes of the operand type,
  // column-major as the reference's: D_d [Np x Np], LIFT [Np x 4 Nfp],
  // Vq [Nq x Np], Pq [Np x Nq]
  void *D[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  void *LIFT[2] = {nullptr, nullptr}, *Vq[2] = {nullptr, nullptr}, *Pq[2] = {nullptr, nullptr};
  // B operands, [rows x K] column-major (column = element): p, U_r, U_s,
  // U_t, pflux (4 Nfp rows), rhs_p, c2 * p_q (Nq rows); hi / lo planes, or
  // one FP32 plane for TF32
  void *Bp[2] = {nullptr, nullptr}, *BU[3][2] = {{nullptr, nullptr}, {nullptr, nullptr},
                                                 {nullptr, nullptr}};
  void *BF[2] = {nullptr, nullptr}, *BR[2] = {nullptr, nullptr}, *BC[2] = {nullptr, nullptr};
  // GEMM results (FP32, [rows x K]): gradient r,s,t, divergence, lift per
  // face, Vq rhs_p, Pq (c2 p_q)
  float *G[3] = {nullptr, nullptr, nullptr}, *Div = nullptr, *Lf[4] = {nullptr, nullptr, nullptr,
                                                                       nullptr};
  float *W = nullptr, *Z = nullptr;
  float *scale = nullptr;  // [K][5] per-element power-of-two scales: p, U, flux, rhs_p, c2 p_q
};

// element operand splits and GEMM form of one stage; geometry, maps and the
// c^2 field are the context's (vgeo [K][9], fgeo [K][16], neighbour codes and
// face-permutation tables as the fused stage's)
bbw_status gemm_stage_create(GemmStage &g, int N, int K, int Nq, int bc, int precision,
                             const std::vector<float> (&D)[3], const std::vector<float> &LIFT,
                             const std::vector<float> &Vq, const std::vector<float> &Pq);
void gemm_stage_release(GemmStage &g);
struct GemmInputs {
  const float *vgeo, *fgeo, *c2q;
  const int *nbr, *tables;
  int pat_off;
};
bbw_status gemm_stage_launch(GemmStage &g, const GemmInputs &in, const float *Qin, float *Qout,
                             float *res, float fa, float fb, float fdt, cudaStream_t st);

}  // namespace bbw
