// Receivers and the device-resident simulation clock.
//
// A receiver samples p at a point of one element: trace = sum_n w[n] p_n
// with w the basis values at the point (nodal: Lagrange interpolation
// weights; BB: Bernstein values), for every shot after every full LSRK step.
// The clock (time, step) lives in device memory so that one captured CUDA
// graph per step serves the whole run; the source wavelet is evaluated from
// it at the stage times t + c_s dt (c_s = rk4c, cpp/src/StartUp3d.cpp:531-537).
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "fused.h"

namespace bbw {

__global__ void k_receivers(int K, int Np, int S, const float *__restrict__ Q, int R,
                            const int *__restrict__ rec_elem, const float *__restrict__ rec_w,
                            float *__restrict__ traces, int max_steps, const int *__restrict__ step) {
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= S * R) return;
  const int s = w / R, r = w - s * R;
  const float *q = Q + ((size_t)s * K + rec_elem[r]) * 4 * Np;  // field p
  float acc = 0.f;
  for (int n = lane; n < Np; n += 32) acc += rec_w[(size_t)r * Np + n] * q[n];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const int st = *step;
  if (lane == 0 && st < max_steps) traces[((size_t)s * R + r) * max_steps + st] = acc;
}

__global__ void k_clock(double *time, int *step, float dt) {
  if (threadIdx.x == 0) {
    *time += (double)dt;
    *step += 1;
  }
}

// buf[s][j][0..4Np) <-> Q[s][idx[j]][0..4Np); one warp per (shot, element)
__global__ void k_move_elements(int Np4, int K, int S, float *Q, int n, const int *idx,
                                float *buf, int to_buf) {
  const long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= (long long)S * n) return;
  const int s = (int)(w / n), j = (int)(w - (long long)s * n);
  const int k = idx[j];
  if (k < 0 || k >= K) return;  // indices outside the mesh are skipped
  float *q = Q + ((size_t)s * K + k) * Np4;
  float *b = buf + ((size_t)s * n + j) * Np4;
  if (to_buf)
    for (int i = lane; i < Np4; i += 32) b[i] = q[i];
  else
    for (int i = lane; i < Np4; i += 32) q[i] = b[i];
}

static bbw_status move_elements(int Np, int K, int S, float *Q, int n, const int *idx, float *buf,
                                int to_buf, cudaStream_t st) {
  if (n <= 0) return BBW_OK;
  const long long warps = (long long)S * n;
  const int wpb = 8;
  k_move_elements<<<(int)((warps + wpb - 1) / wpb), 32 * wpb, 0, st>>>(4 * Np, K, S, Q, n, idx,
                                                                        buf, to_buf);
  return check_launch("element copy");
}

bbw_status gather_elements(int Np, int K, int S, const float *Q, int n, const int *idx,
                           float *buf, cudaStream_t st) {
  return move_elements(Np, K, S, const_cast<float *>(Q), n, idx, buf, 1, st);
}

bbw_status scatter_elements(int Np, int K, int S, float *Q, int n, const int *idx,
                            const float *buf, cudaStream_t st) {
  return move_elements(Np, K, S, Q, n, idx, const_cast<float *>(buf), 0, st);
}

bbw_status record_and_advance(int N, int K, int S, const float *Q, int R, const int *rec_elem,
                              const float *rec_w, float *traces, int max_steps, double *time,
                              int *step, float dt, cudaStream_t st) {
  if (R > 0 && traces) {
    const int threads = 256, warps = S * R;
    k_receivers<<<(warps * 32 + threads - 1) / threads, threads, 0, st>>>(
        K, NP(N), S, Q, R, rec_elem, rec_w, traces, max_steps, step);
    bbw_status s = check_launch("receivers");
    if (s != BBW_OK) return s;
  }
  k_clock<<<1, 32, 0, st>>>(time, step, dt);
  return check_launch("clock");
}

}  // namespace bbw
