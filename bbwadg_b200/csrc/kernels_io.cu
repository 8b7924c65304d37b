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
