// Shared device-side definitions of the CUDA translation units.
#pragma once
#include <cuda_runtime.h>

#include "bbwadg.h"

namespace bbw {

#define NP(N) (((N) + 1) * ((N) + 2) * ((N) + 3) / 6)
#define NFP(N) (((N) + 1) * ((N) + 2) / 2)
// elements per CTA of the kernel-level entry points (256 threads)
#define VOL_EB(N) (512 / NP(N) > 0 ? 512 / NP(N) : 1)
#define SURF_EB(N) (512 / (4 * NFP(N)) > 0 ? 512 / (4 * NFP(N)) : 1)
#define UPD_EB(N) (256 / NP(N) > 0 ? 256 / NP(N) : 1)

// thread-local error record (errors.cu)
bbw_status set_error(bbw_status s, const char *msg);
bbw_status set_cuda_error(cudaError_t e, const char *where);
// checks the launch configuration error of the last kernel launch
bbw_status check_launch(const char *what);
// Raises `func`'s dynamic shared-memory limit on the current device to at
// least `bytes` (never lowers it).  The attribute is per kernel and per
// device, so it is tracked per (kernel, device); thread-safe; the CUDA
// status of the call is returned.
bbw_status ensure_smem_limit(const void *func, int bytes, const char *what);
template <class F>
inline bbw_status ensure_smem_limit(F *func, int bytes, const char *what) {
  return ensure_smem_limit(reinterpret_cast<const void *>(func), bytes, what);
}
// the device's opt-in maximum of dynamic shared memory per block (bytes)
int device_smem_optin();

}  // namespace bbw
