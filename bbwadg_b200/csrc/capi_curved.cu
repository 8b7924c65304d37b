// Curvilinear WADG solver handle: the reference's stage RK_step_WADG
// (cpp/src/WaveOKL3d.cpp:2111-2185) and its LSRK45 loop (Wave_RK with
// useWADG = 2, cpp/src/WaveOKL3d.cpp:2014-2079), B200 layout:
//
// * elements are renumbered planar first, curved last (host permutation on
//   set/get; the kernel-level entry points keep the reference's numbering);
// * the planar elements [0, KP) advance with the fused affine stage kernel
//   (one pass: volume, surface, WADG projection of p with c^2, LSRK update).
//   For an affine element J is constant, so the reference's J-weighted
//   planar kernels followed by the 1/J update reduce to the unweighted
//   stage with Pq diag(c^2) Vq on p and the identity on u, v, w (Pq Vq = I);
// * the curved elements [KP, K) advance with one fused kernel
//   (k_curved_stage: skew volume + skew surface + 1/J, c^2 WADG update +
//   LSRK update), reading the same old state and writing the same new
//   state buffer, so one stage is two launches and no rhs array exists.
//   The two write disjoint elements, so the curved kernel runs on a second
//   stream beside the planar one (fork / join by events each stage): the
//   planar kernel is bound by its shared-memory pipe, the curved one by
//   latency, and their CTAs share the SMs.
// bbw_curved_steps captures one LSRK45 step per buffer parity in a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "bbwadg.h"
#include "ctx.h"
#include "curved.h"
#include "device_common.cuh"


using namespace bbw;

struct bbw_curved {
  int N = 0, K = 0, Np = 0, KC = 0, KP = 0, device = 0;
  cudaStream_t stream = nullptr, side = nullptr;  // main stream; the curved kernel's
  cudaEvent_t fork = nullptr, join = nullptr;
  bbw_ctx *aff = nullptr;             // fused affine stage of the planar elements
  float *Q[2] = {nullptr, nullptr};   // state buffers (the affine context's when it exists)
  float *res = nullptr;
  int cur = 0;
  std::vector<int> perm;              // new element index -> reference index
  CurvedStageArgs args{};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  uint32_t graph_dt_bits[2] = {0, 0};
  std::vector<void *> owned;
  std::vector<float> host;            // permutation scratch
};

namespace {

template <class T>
bbw_status own_upload(bbw_curved *h, T **dst, const T *src, size_t n, const char *what) {
  bbw_status s = upload(dst, src, n, what);
  if (s == BBW_OK) h->owned.push_back((void *)*dst);
  return s;
}

template <class T>
const T *own_upload_c(bbw_curved *h, const T *src, size_t n, bbw_status &s) {
  T *d = nullptr;
  if (s == BBW_OK) s = own_upload(h, &d, src, n, "bbw_curved_create: upload");
  return d;
}

void release(bbw_curved *h) {
  for (auto &g : h->graph)
    if (g) cudaGraphExecDestroy(g);
  if (h->aff) bbw_destroy(h->aff);
  for (void *p : h->owned) cudaFree(p);
  if (h->fork) cudaEventDestroy(h->fork);
  if (h->join) cudaEventDestroy(h->join);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

// rows of a [K][w] array in the new element order (from position `from`)
template <class T>
std::vector<T> rows(const T *a, const std::vector<int> &perm, size_t w, int from = 0) {
  std::vector<T> out((perm.size() - from) * w);
  for (size_t i = from; i < perm.size(); ++i)
    std::memcpy(&out[(i - from) * w], a + (size_t)perm[i] * w, w * sizeof(T));
  return out;
}

bbw_status stage(bbw_curved *h, float fa, float fb, float fdt) {
  const float *Qin = h->Q[h->cur];
  float *Qout = h->Q[h->cur ^ 1];
  const bool both = h->KP > 0 && h->KC > 0;
  cudaStream_t cst = both ? h->side : h->stream;
  bbw_status s = BBW_OK;
  if (both) {  // fork: the curved kernel waits for everything before this stage
    cudaError_t e = cudaEventRecord(h->fork, h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->side, h->fork, 0);
    s = set_cuda_error(e, "curved stage: fork");
  }
  if (s == BBW_OK && h->KP > 0)
    s = fused_launch(h->aff->plan, Qin, Qout, h->res, fa, fb, fdt, 0.f, h->stream);
  if (s == BBW_OK && h->KC > 0) {
    CurvedStageArgs A = h->args;
    A.fa = fa, A.fb = fb, A.fdt = fdt;
    s = curved_stage(h->N, A, Qin, Qout, h->res, cst);
  }
  if (both) {  // join: the next stage reads what both wrote (always joined)
    cudaError_t e = cudaEventRecord(h->join, h->side);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->stream, h->join, 0);
    if (s == BBW_OK) s = set_cuda_error(e, "curved stage: join");
  }
  if (s == BBW_OK) h->cur ^= 1;
  return s;
}

void drop_graphs(bbw_curved *h) {
  for (int i = 0; i < 2; ++i) {
    if (h->graph[i]) cudaGraphExecDestroy(h->graph[i]);
    h->graph[i] = nullptr;
  }
}

}  // namespace

extern "C" bbw_status bbw_curved_create(const bbw_curved_desc *d, int device, bbw_curved **out) {
  if (!out || !d) return set_error(BBW_ERR_ARG, "bbw_curved_create: NULL argument");
  *out = nullptr;
  const int N = d->N, K = d->K;
  if (N < 1 || N > BBW_MAX_N) return set_error(BBW_ERR_UNSUPPORTED, "bbw_curved_create: N");
  const int Np = NP(N), Nfp = NFP(N), NF = 4 * Nfp;
  if (K < 1 || d->Nq < Np || d->Nfq < 1 || d->Nq_reduced < 1 || d->KCurved < 0 ||
      d->KPlanar < 0 || d->KCurved + d->KPlanar != K || (long long)K * 4 * Np >= (1LL << 31))
    return set_error(BBW_ERR_ARG, "bbw_curved_create: bad sizes");
  const void *req[] = {d->vgeo, d->fgeo, d->Jplanar, d->Fmask, d->vmapP, d->Jq_reduced, d->c2q,
                       d->Dr, d->Ds, d->Dt, d->LIFT, d->Vq_reduced, d->Pq_reduced};
  for (const void *p : req)
    if (!p) return set_error(BBW_ERR_ARG, "bbw_curved_create: missing array");
  if (d->KCurved > 0) {
    const void *creq[] = {d->KlistCurved, d->vgeoq, d->Jq, d->fgeoq, d->Vq, d->Vrq, d->Vsq,
                          d->Vtq, d->Pq, d->Prq, d->Psq, d->Ptq, d->VfqFace, d->Pfq};
    for (const void *p : creq)
      if (!p) return set_error(BBW_ERR_ARG, "bbw_curved_create: missing curved-element array");
  }
  if (d->KPlanar > 0 && !d->KlistPlanar)
    return set_error(BBW_ERR_ARG, "bbw_curved_create: missing planar list");
  // every element in exactly one list: planar first, then curved
  std::vector<int> perm, inv(K, -1);
  for (int pass = 0; pass < 2; ++pass) {
    const int n = pass ? d->KCurved : d->KPlanar;
    const int *L = pass ? d->KlistCurved : d->KlistPlanar;
    for (int i = 0; i < n; ++i) {
      if (L[i] < 0 || L[i] >= K || inv[L[i]] >= 0)
        return set_error(BBW_ERR_ARG, "bbw_curved_create: element lists must partition 0..K-1");
      inv[L[i]] = (int)perm.size();
      perm.push_back(L[i]);
    }
  }
  for (int i = 0; i < NF; ++i)
    if (d->Fmask[i] < 0 || d->Fmask[i] >= Np)
      return set_error(BBW_ERR_ARG, "bbw_curved_create: Fmask entry out of range");
  std::vector<int> vmapP((size_t)K * NF);
  for (int i = 0; i < K; ++i)
    for (int m = 0; m < NF; ++m) {
      const int v = d->vmapP[(size_t)perm[i] * NF + m];
      if (v < 0 || v >= K * 4 * Np || v % (4 * Np) >= Np)
        return set_error(BBW_ERR_ARG, "bbw_curved_create: vmapP entry out of range");
      vmapP[(size_t)i * NF + m] = inv[v / (4 * Np)] * 4 * Np + v % (4 * Np);
    }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_create: device");
  if (device < 0 || device >= ndev)
    return set_error(BBW_ERR_ARG, "bbw_curved_create: no such device");
  DeviceGuard dg(device);  // the caller's current device is restored on return
  bbw_curved *h = new bbw_curved;
  h->N = N, h->K = K, h->Np = Np, h->KC = d->KCurved, h->KP = d->KPlanar, h->device = device;
  h->perm = perm;
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    release(h);
    return set_cuda_error(e, "bbw_curved_create: stream");
  }
  const size_t ns = (size_t)K * 4 * Np;
  const int Nq = d->Nq, Nfq = d->Nfq, Nr = d->Nq_reduced, KP = d->KPlanar;
  bbw_status s = BBW_OK;
  std::vector<float> c2 = rows(d->c2q, perm, Nr);
  if (KP > 0) {  // fused affine stage over the planar prefix
    std::vector<float> vgeo = rows(d->vgeo, perm, 9), fgeo = rows(d->fgeo, perm, 16);
    bbw_mesh_desc md{N, K, Nr, vgeo.data(), fgeo.data(), d->Fmask, vmapP.data(), c2.data(),
                     nullptr};
    bbw_ops_desc od{};
    od.Dr = d->Dr, od.Ds = d->Ds, od.Dt = d->Dt, od.LIFT = d->LIFT;
    od.Vq = d->Vq_reduced, od.Pq = d->Pq_reduced;
    s = bbw_create(&md, &od, BBW_NODAL, BBW_BC_PRESSURE_RELEASE, &h->aff);
    if (s == BBW_OK && KP < K) s = bbw_set_compute_range(h->aff, KP);
    if (s == BBW_OK) h->Q[0] = h->aff->Q[0], h->Q[1] = h->aff->Q[1], h->res = h->aff->res;
  } else {
    if (s == BBW_OK) s = own_upload(h, &h->Q[0], (const float *)nullptr, ns, "bbw_curved_create");
    if (s == BBW_OK) s = own_upload(h, &h->Q[1], (const float *)nullptr, ns, "bbw_curved_create");
    if (s == BBW_OK) s = own_upload(h, &h->res, (const float *)nullptr, ns, "bbw_curved_create");
  }
  if (d->KCurved > 0) {  // compact rows of the curved tail
    CurvedStageArgs &A = h->args;
    A.KC = d->KCurved, A.k_off = KP, A.Nq = Nq, A.Nfq = Nfq, A.Nr = Nr;
    const size_t nq = Nq, nr = Nr, nf = Nfq;
    std::vector<float> t;
    t = rows(d->vgeoq, perm, 9 * nq, KP), A.vgeoq = own_upload_c(h, t.data(), t.size(), s);
    t = rows(d->Jq, perm, nq, KP), A.Jq = own_upload_c(h, t.data(), t.size(), s);
    t = rows(d->fgeoq, perm, 16 * nf, KP), A.fgeoq = own_upload_c(h, t.data(), t.size(), s);
    t = rows(d->Jq_reduced, perm, nr, KP), A.Jr = own_upload_c(h, t.data(), t.size(), s);
    A.c2q = own_upload_c(h, c2.data() + (size_t)KP * Nr, (size_t)d->KCurved * Nr, s);
    const size_t mq = nq * Np, mr = nr * Np;
    A.Vq = own_upload_c(h, d->Vq, mq, s), A.Vrq = own_upload_c(h, d->Vrq, mq, s);
    A.Vsq = own_upload_c(h, d->Vsq, mq, s), A.Vtq = own_upload_c(h, d->Vtq, mq, s);
    A.Pq = own_upload_c(h, d->Pq, mq, s), A.Prq = own_upload_c(h, d->Prq, mq, s);
    A.Psq = own_upload_c(h, d->Psq, mq, s), A.Ptq = own_upload_c(h, d->Ptq, mq, s);
    A.VfqFace = own_upload_c(h, d->VfqFace, nf * Nfp, s);
    A.Pfq = own_upload_c(h, d->Pfq, (size_t)Np * 4 * nf, s);
    A.Vqr = own_upload_c(h, d->Vq_reduced, mr, s), A.Pqr = own_upload_c(h, d->Pq_reduced, mr, s);
    A.Fmask = own_upload_c(h, d->Fmask, (size_t)NF, s);
    A.vmapP = own_upload_c(h, vmapP.data(), vmapP.size(), s);
  }
  // one stage on the zero state (it stays zero) sets the kernels' launch
  // attributes outside any later graph capture
  if (s == BBW_OK) s = stage(h, 0.f, 0.f, 0.f);
  if (s == BBW_OK) s = set_cuda_error(cudaStreamSynchronize(h->stream), "bbw_curved_create");
  if (s != BBW_OK) {
    release(h);
    return s;
  }
  h->cur = 0;
  *out = h;
  return BBW_OK;
}

extern "C" bbw_status bbw_curved_destroy(bbw_curved *h) {
  if (!h) return BBW_OK;
  DeviceGuard dg(h->device);
  cudaStreamSynchronize(h->stream);
  drop_graphs(h);
  release(h);
  return BBW_OK;
}

// host [K][4][Np] in the reference's element order <-> device buffer
static bbw_status copy_state(bbw_curved *h, float *dev, const float *src, float *dst,
                             const char *what) {
  if (!h || (!src && !dst)) return set_error(BBW_ERR_ARG, what);
  const size_t w = (size_t)4 * h->Np, n = (size_t)h->K * w;
  h->host.resize(n);
  cudaError_t e;
  if (src) {
    for (int i = 0; i < h->K; ++i)
      std::memcpy(&h->host[i * w], src + (size_t)h->perm[i] * w, w * sizeof(float));
    e = cudaMemcpyAsync(dev, h->host.data(), n * sizeof(float), cudaMemcpyHostToDevice,
                        h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  } else {
    e = cudaMemcpyAsync(h->host.data(), dev, n * sizeof(float), cudaMemcpyDeviceToHost,
                        h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess)
      for (int i = 0; i < h->K; ++i)
        std::memcpy(dst + (size_t)h->perm[i] * w, &h->host[i * w], w * sizeof(float));
  }
  return set_cuda_error(e, what);
}

extern "C" bbw_status bbw_curved_set_state(bbw_curved *h, const float *Q) {
  DeviceGuard dg(h ? h->device : -1);
  bbw_status s = copy_state(h, h ? h->Q[h->cur] : nullptr, Q, nullptr, "bbw_curved_set_state");
  if (s != BBW_OK) return s;
  const size_t n = (size_t)h->K * 4 * h->Np * sizeof(float);
  cudaError_t e = cudaMemsetAsync(h->res, 0, n, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return set_cuda_error(e, "bbw_curved_set_state");
}

extern "C" bbw_status bbw_curved_get_state(bbw_curved *h, float *Q) {
  DeviceGuard dg(h ? h->device : -1);
  return copy_state(h, h ? h->Q[h->cur] : nullptr, nullptr, Q, "bbw_curved_get_state");
}

extern "C" bbw_status bbw_curved_get_residual(bbw_curved *h, float *r) {
  DeviceGuard dg(h ? h->device : -1);
  return copy_state(h, h ? h->res : nullptr, nullptr, r, "bbw_curved_get_residual");
}

extern "C" bbw_status bbw_curved_stage(bbw_curved *h, float fa, float fb, float fdt) {
  DeviceGuard dg(h ? h->device : -1);
  if (!h) return set_error(BBW_ERR_ARG, "bbw_curved_stage: NULL handle");
  return stage(h, fa, fb, fdt);
}

extern "C" bbw_status bbw_curved_steps(bbw_curved *h, float dt, int nsteps) {
  DeviceGuard dg(h ? h->device : -1);
  if (!h || nsteps < 0) return set_error(BBW_ERR_ARG, "bbw_curved_steps: bad argument");
  uint32_t bits;
  std::memcpy(&bits, &dt, 4);
  for (int step = 0; step < nsteps; ++step) {
    const int par = h->cur;
    if (!h->graph[par] || h->graph_dt_bits[par] != bits) {
      if (h->graph[par]) cudaGraphExecDestroy(h->graph[par]);
      h->graph[par] = nullptr;
      cudaGraph_t g;
      cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_steps: capture");
      bbw_status s = BBW_OK;
      for (int i = 0; i < 5 && s == BBW_OK; ++i)
        s = stage(h, (float)kRK4A[i], (float)kRK4B[i], dt);
      e = cudaStreamEndCapture(h->stream, &g);
      h->cur = par;  // capture recorded the launches without running them
      if (s != BBW_OK) {
        if (e == cudaSuccess) cudaGraphDestroy(g);
        return s;
      }
      if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_steps: end capture");
      e = cudaGraphInstantiate(&h->graph[par], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_steps: instantiate");
      h->graph_dt_bits[par] = bits;
    }
    cudaError_t e = cudaGraphLaunch(h->graph[par], h->stream);
    if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_steps: launch");
    h->cur ^= 1;  // five stages swap the buffers an odd number of times
  }
  return BBW_OK;
}

extern "C" bbw_status bbw_curved_sync(bbw_curved *h) {
  DeviceGuard dg(h ? h->device : -1);
  if (!h) return set_error(BBW_ERR_ARG, "bbw_curved_sync: NULL handle");
  return set_cuda_error(cudaStreamSynchronize(h->stream), "bbw_curved_sync");
}

extern "C" void *bbw_curved_stream(bbw_curved *h) { return h ? (void *)h->stream : nullptr; }

extern "C" bbw_status bbw_curved_autotune(bbw_curved *h, float dt, int stages, int *config) {
  DeviceGuard dg(h ? h->device : -1);
  if (!h || !(dt > 0.f) || stages < 1)
    return set_error(BBW_ERR_ARG, "bbw_curved_autotune: bad argument");
  if (config) *config = 0;
  if (!h->aff) return BBW_OK;  // no planar element: nothing to choose
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->side);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_autotune");
  // the captured steps hold the planar variant's operator buffer, which
  // bbw_set_config frees: recapture after tuning
  drop_graphs(h);
  const size_t n = (size_t)h->K * 4 * h->Np;
  float *saveQ = nullptr, *saveR = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto cleanup = [&]() {
    cudaFree(saveQ), cudaFree(saveR);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  e = cudaMalloc(&saveQ, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&saveR, n * sizeof(float));
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int cur0 = h->cur;
  if (e == cudaSuccess)
    e = cudaMemcpy(saveQ, h->Q[cur0], n * sizeof(float), cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(saveR, h->res, n * sizeof(float), cudaMemcpyDeviceToDevice);
  if (e != cudaSuccess) {
    cleanup();
    return set_cuda_error(e, "bbw_curved_autotune: scratch");
  }
  float best_ms = 0.f;
  int best = -1;
  bbw_status s = BBW_OK;
  for (int e16 = 0; e16 < 2 && s == BBW_OK; ++e16)
  for (int W = 8; W <= 16 && s == BBW_OK; W += 8)
    for (int v = 0; v < 4 && s == BBW_OK; ++v) {
      const int code = W | (v < 2 ? 1 << 8 : 0) | (v % 2 == 0 ? 1 << 9 : 0) | e16 << 10;
      if (bbw_set_config(h->aff, code) != BBW_OK) continue;  // does not fit
      for (int i = 0; i < 2 && s == BBW_OK; ++i) s = stage(h, 0.f, (float)kRK4B[0], dt);
      if (s == BBW_OK) e = cudaEventRecord(e0, h->stream);
      for (int i = 0; i < stages && s == BBW_OK && e == cudaSuccess; ++i)
        s = stage(h, (float)kRK4A[i % 5], (float)kRK4B[i % 5], dt);
      if (s == BBW_OK && e == cudaSuccess) e = cudaEventRecord(e1, h->stream);
      if (s == BBW_OK && e == cudaSuccess) e = cudaEventSynchronize(e1);
      if (s == BBW_OK && e != cudaSuccess) s = set_cuda_error(e, "bbw_curved_autotune: timing");
      float ms = 0.f;
      if (s == BBW_OK) cudaEventElapsedTime(&ms, e0, e1);
      if (s == BBW_OK && (best < 0 || ms < best_ms)) best = code, best_ms = ms;
    }
  // the state and residual as they were, the fastest variant kept
  h->cur = cur0;
  e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->side);
  if (e == cudaSuccess)
    e = cudaMemcpy(h->Q[cur0], saveQ, n * sizeof(float), cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(h->res, saveR, n * sizeof(float), cudaMemcpyDeviceToDevice);
  cleanup();
  if (s != BBW_OK) return s;
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_autotune: restore");
  if (best < 0) return set_error(BBW_ERR_UNSUPPORTED, "bbw_curved_autotune: no variant fits");
  if ((s = bbw_set_config(h->aff, best)) != BBW_OK) return s;
  if (config) *config = best;
  return BBW_OK;
}
