// bbw_rk_stage_noalloc: the reference's three-launch LSRK stage
// (rk_volume, rk_surface, rk_update_WADG) for callers that must not
// allocate device memory.
//
// Who cannot allocate, and why: the kernel-level entry points take the rhs
// buffer (K x 4 x Np floats) from the caller.  Some callers have no way to
// provide one: code that runs inside another framework's device-memory pool
// (which owns all device memory and must not see untracked cudaMalloc
// calls), real-time loops where cudaMalloc/cudaFree would synchronise the
// device and stall other streams, and host code that cannot keep a buffer
// between calls.  This entry point needs no buffer from them: its rhs
// scratch is a fixed array in the library's own device image, reserved when
// the library's module is loaded on a device.
//
// Limits and rules:
// * The scratch holds kNoAllocScratchFloats floats (16 MiB): K * 4 * Np
//   must not exceed it (N = 3: K <= 52 428; N = 5: K <= 18 724); larger
//   meshes are rejected with BBW_ERR_UNSUPPORTED before anything runs.
// * The scratch address is looked up (cudaGetSymbolAddress, with the
//   device current) and cached per device.  The first call on each device
//   does this set-up and must come before any stream capture.  Every later
//   call whose stream is not capturing looks the address up again, so after
//   a cudaDeviceReset (which reloads the module and may move the array) the
//   next such call picks up the new address.
// * Nothing in the scratch has to start at zero: rk_volume overwrites every
//   rhs entry of the K elements before rk_surface accumulates into it.
// * There is one scratch per device: calls that overlap in time on the same
//   device (different streams or host threads without ordering) race on it
//   and give wrong results.  Order them on one stream.
// * It calls no cudaMalloc / cudaFree and no allocating library.
#include <cuda_runtime.h>

#include <mutex>

#include "bbwadg.h"
#include "device_common.cuh"

namespace {

constexpr size_t kNoAllocScratchFloats = (size_t)4 << 20;  // 16 MiB
constexpr int kMaxDevices = 64;

__device__ __align__(256) float g_stage_scratch[kNoAllocScratchFloats];

std::mutex g_scratch_mu;
float *g_scratch_ptr[kMaxDevices] = {};

bbw_status scratch_for_current_device(cudaStream_t stream, float **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bbw::set_cuda_error(e, "bbw_rk_stage_noalloc: current device");
  if (dev < 0 || dev >= kMaxDevices)
    return bbw::set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_stage_noalloc: device index above 63");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &cap);
  if (e != cudaSuccess) return bbw::set_cuda_error(e, "bbw_rk_stage_noalloc: stream");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (cap == cudaStreamCaptureStatusNone || !g_scratch_ptr[dev]) {
    if (cap != cudaStreamCaptureStatusNone)
      return bbw::set_error(BBW_ERR_STATE,
                            "bbw_rk_stage_noalloc: first call on a device inside a stream "
                            "capture; make one call outside the capture first");
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_stage_scratch);
    if (e != cudaSuccess)
      return bbw::set_cuda_error(e, "bbw_rk_stage_noalloc: scratch address");
    g_scratch_ptr[dev] = static_cast<float *>(p);
  }
  *out = g_scratch_ptr[dev];
  return BBW_OK;
}

}  // namespace

extern "C" bbw_status bbw_rk_stage_noalloc(int N, int K, int Nq, int bc, const float *vgeo,
                                           const float *Dr, const float *Ds, const float *Dt,
                                           const float *fgeo, const int *Fmask,
                                           const int *vmapP, const float *LIFT, const float *Vq,
                                           const float *Pq, const float *Jq, const float *c2q,
                                           float fa, float fb, float fdt, float *resQ, float *Q,
                                           void *stream) {
  if (N < 1 || N > BBW_MAX_N) return bbw::set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_stage_noalloc: N");
  if (K < 0 || Nq <= 0 || (bc != 0 && bc != 1))
    return bbw::set_error(BBW_ERR_ARG, "bbw_rk_stage_noalloc: bad size or bc");
  if (K == 0) return BBW_OK;
  if (!vgeo || !Dr || !Ds || !Dt || !fgeo || !Fmask || !vmapP || !LIFT || !Vq || !Pq || !Jq ||
      !c2q || !resQ || !Q)
    return bbw::set_error(BBW_ERR_ARG, "bbw_rk_stage_noalloc: NULL array");
  const size_t need = (size_t)K * 4 * NP(N);
  if (need > kNoAllocScratchFloats)
    return bbw::set_error(BBW_ERR_UNSUPPORTED,
                          "bbw_rk_stage_noalloc: K * 4 * Np exceeds the 16 MiB static scratch "
                          "(4 Mi floats); use the kernel-level entry points with your own rhs "
                          "buffer or a bbw_ctx");
  float *rhs = nullptr;
  bbw_status s = scratch_for_current_device(static_cast<cudaStream_t>(stream), &rhs);
  if (s != BBW_OK) return s;
  if ((s = bbw_rk_volume(N, K, vgeo, Dr, Ds, Dt, Q, rhs, stream)) != BBW_OK) return s;
  if ((s = bbw_rk_surface(N, K, bc, fgeo, Fmask, vmapP, LIFT, Q, rhs, stream)) != BBW_OK) return s;
  return bbw_rk_update_wadg(N, K, Nq, Vq, Pq, Jq, c2q, fa, fb, fdt, rhs, resQ, Q, stream);
}
