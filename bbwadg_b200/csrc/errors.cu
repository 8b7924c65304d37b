// Status strings and the per-thread last-error record of the C ABI.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include "device_common.cuh"

namespace bbw {

static thread_local char g_last[512] = "";

bbw_status set_error(bbw_status s, const char *msg) {
  if (s != BBW_OK) snprintf(g_last, sizeof g_last, "%s", msg);
  return s;
}

bbw_status set_cuda_error(cudaError_t e, const char *where) {
  if (e == cudaSuccess) return BBW_OK;
  snprintf(g_last, sizeof g_last, "%s: %s", where, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? BBW_ERR_NOMEM : BBW_ERR_CUDA;
}

bbw_status check_launch(const char *what) { return set_cuda_error(cudaGetLastError(), what); }

bbw_status ensure_smem_limit(const void *func, int bytes, const char *what) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> done;  // (kernel, device) -> limit set
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error(e, what);
  std::lock_guard<std::mutex> lock(mu);
  auto it = done.find(std::make_pair(func, dev));
  if (it != done.end() && it->second >= bytes) return BBW_OK;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return set_cuda_error(e, what);
  done[std::make_pair(func, dev)] = bytes;
  return BBW_OK;
}

int device_smem_optin() {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 48 * 1024;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 48 * 1024;
  return v;
}

}  // namespace bbw

extern "C" const char *bbw_status_string(bbw_status s) {
  switch (s) {
    case BBW_OK: return "ok";
    case BBW_ERR_ARG: return "invalid argument";
    case BBW_ERR_CUDA: return "CUDA error";
    case BBW_ERR_NOMEM: return "out of memory";
    case BBW_ERR_STATE: return "call out of sequence";
    case BBW_ERR_MESH: return "inconsistent mesh";
    case BBW_ERR_NUMERIC: return "operator construction failed";
    case BBW_ERR_UNSUPPORTED: return "unsupported size or option";
    case BBW_ERR_TIMEOUT: return "bounded device wait gave up";
  }
  return "unknown status";
}

extern "C" const char *bbw_last_error(void) { return bbw::g_last; }

extern "C" const char *bbw_version(void) { return "bbwadg_b200 0.1 (sm_100a)"; }
