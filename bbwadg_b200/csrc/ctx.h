// Solver context shared by the runtime translation units (capi.cu,
// adjoint.cu).  Internal: the public surface is include/bbwadg.h.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "bbwadg.h"
#include "device_common.cuh"
#include "fused.h"
#include "gemm_stage.h"

namespace bbw {

// device operators and maps of the discrete adjoint (uploaded on first use)
struct AdjOps {
  bool ready = false;
  float *D[3] = {nullptr, nullptr, nullptr};   // Dr, Ds, Dt
  float *DT[3] = {nullptr, nullptr, nullptr};  // their transposes
  float *LIFT = nullptr, *Vq = nullptr, *Pq = nullptr;
  int *Fmask = nullptr, *vmapP = nullptr;
  int *fidx = nullptr;  // [4][Np]: index of node n on face f, or -1
  int *mapP = nullptr;  // [K][4Nfp]: matching face node k2*4Nfp + m2, -1 on the boundary
  // padded layouts read by the reverse-stage kernels (contraction index
  // outer, rows padded to a multiple of 4): Pq^T [Np][ld(Nq)], Vq^T
  // [Nq][ld(Np)], D^T [3][Np][ld(Np)], LIFT^T per face [4][Np][ld(Nfp)]
  float *PqT = nullptr, *VqT = nullptr, *DTp = nullptr, *LTp = nullptr;
};

// LSRK45 coefficients (Carpenter-Kennedy), cpp/src/StartUp3d.cpp:517-537
extern const double kRK4A[5], kRK4B[5], kRK4C[5];

template <class T>
bbw_status upload(T **dst, const T *src, size_t n, const char *what) {
  cudaError_t e = cudaMalloc((void **)dst, n * sizeof(T) + 16);
  if (e != cudaSuccess) return set_cuda_error(e, what);
  if (src) e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  else e = cudaMemset(*dst, 0, n * sizeof(T));
  return set_cuda_error(e, what);
}

// adjoint kernels (kernels_adj.cu)
bbw_status adj_wadg(int N, int S, int K, int Nq, const float *PqT, const float *VqT,
                    const float *c2q, const float *lamQ, float *lamR, float a, float b, float dt,
                    const float *vq, float *z, double *grad, cudaStream_t st);
bbw_status adj_sigma(int N, int S, int K, const float *fgeo, const float *LTp, const float *z,
                     float *sigma, cudaStream_t st);
bbw_status adj_volume(int N, int S, int K, const float *vgeo, const float *DTp, const float *z,
                      float *vol, cudaStream_t st);
bbw_status adj_gather(int N, int S, int K, int bc, float dt, const float *fgeo, const int *fidx,
                      const int *mapP, const float *sigma, const float *vol, float *lamQ,
                      cudaStream_t st);
bbw_status adj_receivers(int S, int K, int Np, int R, const int *rec_elem, const float *rec_w,
                         const float *g, int nsteps, int n, float *lamQ, cudaStream_t st);
bbw_status set_device_double(double *p, double v, cudaStream_t st);

}  // namespace bbw

struct bbw_ctx {
  int N = 0, K = 0, Nq = 0, Np = 0, Nfp = 0, variant = 0, bc = 0, device = 0;
  cudaStream_t stream = nullptr;
  float *Q[2] = {nullptr, nullptr};
  int cur = 0;
  float *res = nullptr;
  float *vgeo = nullptr, *fgeo = nullptr, *c2q = nullptr, *ops = nullptr;
  int *nbr = nullptr, *tables = nullptr;
  bbw::FusedPlan plan;
  int precision = BBW_PREC_FP32;
  int S = 1;  // shots
  double *d_time = nullptr;
  int *d_step = nullptr;
  int *src_off = nullptr, *src_elem = nullptr;
  int *src_tile = nullptr;  // [S * ceil(K / 32) + 1] entry offsets per (shot, 32-element tile)
  float *src_vec = nullptr;
  int src_stage_times = 0;
  int R = 0, max_steps = 0;
  int *rec_elem = nullptr;
  float *rec_w = nullptr, *traces = nullptr;
  bbw::TcPlan tc;
  bbw::GemmStage *gs = nullptr;  // precision-study GEMM form (null: fused or tensor-core stage)
  float *geo_tc = nullptr;
  void *ops_tc = nullptr;
  int *err = nullptr;
  // one graph per starting buffer parity, for one LSRK45 step of size dt
  cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
  uint32_t graph_dt_bits[2] = {0, 0};
  // host copies for the adjoint: dense operators of the chosen basis
  // (column-major Np x Np / Np x 4Nfp / Nq x Np / Np x Nq), Fmask, vmapP
  std::vector<float> hD[3], hLIFT, hVq, hPq;
  std::vector<int> hFmask, hvmapP;
  bbw::AdjOps adj;
};


// one LSRK45 step launched stage by stage that also stores each stage's
// pre-c^2 cubature values at vq + i * vqn (capi.cu)
bbw_status step_storing_cubature(bbw_ctx *c, float dt, float *vq, size_t vqn);

namespace bbw {
void adj_release(bbw_ctx *c);

// Makes a context's device current for the duration of one entry point and
// restores the caller's device on return: contexts of one process may live
// on different devices, and their streams, buffers and launches belong to
// that device.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int device) {  // device < 0: nothing to do
    int cur = -1;
    if (device >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != device &&
        cudaSetDevice(device) == cudaSuccess)
      prev = cur;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
};
}  // namespace bbw
