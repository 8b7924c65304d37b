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

}  // namespace bbw
