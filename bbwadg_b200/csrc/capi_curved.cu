// Curvilinear WADG solver handle: device copies of the curved path's arrays
// and the reference's stage RK_step_WADG (cpp/src/WaveOKL3d.cpp:2111-2185):
//   skew-form volume + surface kernels on the curved elements,
//   J-weighted volume + surface kernels on the planar elements,
//   rk_update_WADG (all four fields weighted by 1/J, c^2 on p) on all.
// bbw_curved_steps runs the LSRK45 loop of Wave_RK (useWADG = 2,
// cpp/src/WaveOKL3d.cpp:2014-2079) as one CUDA graph per step.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "bbwadg.h"
#include "ctx.h"
#include "device_common.cuh"

namespace bbw {
bbw_status curved_volume(int N, int K, const int *Klist, int Nq, const float *vgeoq,
                         const float *Jq, const float *Vq, const float *Vrq, const float *Vsq,
                         const float *Vtq, const float *Pq, const float *Prq, const float *Psq,
                         const float *Ptq, const float *Q, float *rhsQ, cudaStream_t st);
bbw_status curved_surface(int N, int K, const int *Klist, int Nfq, const float *fgeoq,
                          const float *VfqFace, const float *Pfq, const int *Fmask,
                          const int *vmapP, const float *Q, float *rhsQ, cudaStream_t st);
bbw_status planar_volume(int N, int K, const int *Klist, const float *vgeo, const float *J,
                         const float *Dr, const float *Ds, const float *Dt, const float *Q,
                         float *rhsQ, cudaStream_t st);
bbw_status planar_surface(int N, int K, const int *Klist, const float *fgeo, const float *J,
                          const int *Fmask, const int *vmapP, const float *LIFT, const float *Q,
                          float *rhsQ, cudaStream_t st);
}  // namespace bbw

using namespace bbw;

struct bbw_curved {
  int N = 0, K = 0, Nq = 0, Nfq = 0, Nq_red = 0, KC = 0, KP = 0, Np = 0, device = 0;
  cudaStream_t stream = nullptr;
  float *Q = nullptr, *res = nullptr, *rhs = nullptr;
  int *KlistC = nullptr, *KlistP = nullptr, *Fmask = nullptr, *vmapP = nullptr;
  float *vgeo = nullptr, *fgeo = nullptr, *Jplanar = nullptr, *vgeoq = nullptr, *Jq = nullptr,
        *fgeoq = nullptr, *Jq_red = nullptr, *c2q = nullptr;
  float *op[16] = {};  // Dr Ds Dt LIFT Vq Vrq Vsq Vtq Pq Prq Psq Ptq VfqFace Pfq Vq_red Pq_red
  cudaGraphExec_t graph = nullptr;
  uint32_t graph_dt_bits = 0;
  std::vector<void *> owned;
};

namespace {

enum { kDr, kDs, kDt, kLIFT, kVq, kVrq, kVsq, kVtq, kPq, kPrq, kPsq, kPtq, kVfqFace, kPfq,
       kVqRed, kPqRed };

template <class T>
bbw_status own_upload(bbw_curved *h, T **dst, const T *src, size_t n, const char *what) {
  bbw_status s = upload(dst, src, n, what);
  if (s == BBW_OK) h->owned.push_back(*dst);
  return s;
}

void release(bbw_curved *h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (void *p : h->owned) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

bbw_status stage(bbw_curved *h, float fa, float fb, float fdt) {
  const int N = h->N;
  float **o = h->op;
  bbw_status s = curved_volume(N, h->KC, h->KlistC, h->Nq, h->vgeoq, h->Jq, o[kVq], o[kVrq],
                               o[kVsq], o[kVtq], o[kPq], o[kPrq], o[kPsq], o[kPtq], h->Q, h->rhs,
                               h->stream);
  if (s == BBW_OK)
    s = curved_surface(N, h->KC, h->KlistC, h->Nfq, h->fgeoq, o[kVfqFace], o[kPfq], h->Fmask,
                       h->vmapP, h->Q, h->rhs, h->stream);
  if (s == BBW_OK)
    s = planar_volume(N, h->KP, h->KlistP, h->vgeo, h->Jplanar, o[kDr], o[kDs], o[kDt], h->Q,
                      h->rhs, h->stream);
  if (s == BBW_OK)
    s = planar_surface(N, h->KP, h->KlistP, h->fgeo, h->Jplanar, h->Fmask, h->vmapP, o[kLIFT],
                       h->Q, h->rhs, h->stream);
  if (s == BBW_OK)
    s = bbw_rk_update_wadg(N, h->K, h->Nq_red, o[kVqRed], o[kPqRed], h->Jq_red, h->c2q, fa, fb,
                           fdt, h->rhs, h->res, h->Q, h->stream);
  return s;
}

}  // namespace

extern "C" bbw_status bbw_curved_create(const bbw_curved_desc *d, int device, bbw_curved **out) {
  if (!out || !d) return set_error(BBW_ERR_ARG, "bbw_curved_create: NULL argument");
  *out = nullptr;
  const int N = d->N, K = d->K;
  if (N < 1 || N > BBW_MAX_N) return set_error(BBW_ERR_UNSUPPORTED, "bbw_curved_create: N");
  const int Np = NP(N), NF = 4 * NFP(N);
  if (K < 1 || d->Nq < Np || d->Nfq < 1 || d->Nq_reduced < 1 || d->KCurved < 0 ||
      d->KPlanar < 0 || d->KCurved + d->KPlanar != K ||
      (long long)K * 4 * Np >= (1LL << 31))
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
  // every element in exactly one list; traces inside the mesh
  std::vector<char> seen(K, 0);
  for (int pass = 0; pass < 2; ++pass) {
    const int n = pass ? d->KPlanar : d->KCurved;
    const int *L = pass ? d->KlistPlanar : d->KlistCurved;
    for (int i = 0; i < n; ++i) {
      if (L[i] < 0 || L[i] >= K || seen[L[i]])
        return set_error(BBW_ERR_ARG, "bbw_curved_create: element lists must partition 0..K-1");
      seen[L[i]] = 1;
    }
  }
  for (int i = 0; i < NF; ++i)
    if (d->Fmask[i] < 0 || d->Fmask[i] >= Np)
      return set_error(BBW_ERR_ARG, "bbw_curved_create: Fmask entry out of range");
  for (size_t i = 0; i < (size_t)K * NF; ++i) {
    const int v = d->vmapP[i];
    if (v < 0 || v >= K * 4 * Np || v % (4 * Np) >= Np)
      return set_error(BBW_ERR_ARG, "bbw_curved_create: vmapP entry out of range");
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_create: device");
  bbw_curved *h = new bbw_curved;
  h->N = N, h->K = K, h->Nq = d->Nq, h->Nfq = d->Nfq, h->Nq_red = d->Nq_reduced;
  h->KC = d->KCurved, h->KP = d->KPlanar, h->Np = Np, h->device = device;
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    release(h);
    return set_cuda_error(e, "bbw_curved_create: stream");
  }
  const size_t ns = (size_t)K * 4 * Np, Nq = d->Nq, Nfq = d->Nfq, Nr = d->Nq_reduced;
  const int KC = std::max(d->KCurved, 1), KP = std::max(d->KPlanar, 1);
  std::vector<int> zeros(1, 0);
  struct OpSpec { const float *src; size_t n; };
  const OpSpec ops[16] = {
      {d->Dr, (size_t)Np * Np}, {d->Ds, (size_t)Np * Np}, {d->Dt, (size_t)Np * Np},
      {d->LIFT, (size_t)Np * NF}, {d->Vq, Nq * Np}, {d->Vrq, Nq * Np}, {d->Vsq, Nq * Np},
      {d->Vtq, Nq * Np}, {d->Pq, Np * Nq}, {d->Prq, Np * Nq}, {d->Psq, Np * Nq},
      {d->Ptq, Np * Nq}, {d->VfqFace, Nfq * NFP(N)}, {d->Pfq, Np * 4 * Nfq},
      {d->Vq_reduced, Nr * Np}, {d->Pq_reduced, Np * Nr}};
  bbw_status s = BBW_OK;
  const bool curved = d->KCurved > 0;
#define UP(dst, src, n) \
  if (s == BBW_OK) s = own_upload(h, dst, src, n, "bbw_curved_create: upload")
  UP(&h->Q, (const float *)nullptr, ns);
  UP(&h->res, (const float *)nullptr, ns);
  UP(&h->rhs, (const float *)nullptr, ns);
  UP(&h->KlistC, curved ? d->KlistCurved : zeros.data(), (size_t)KC);
  UP(&h->KlistP, d->KPlanar ? d->KlistPlanar : zeros.data(), (size_t)KP);
  UP(&h->Fmask, d->Fmask, (size_t)NF);
  UP(&h->vmapP, d->vmapP, (size_t)K * NF);
  UP(&h->vgeo, d->vgeo, (size_t)K * 9);
  UP(&h->fgeo, d->fgeo, (size_t)K * 16);
  UP(&h->Jplanar, d->Jplanar, (size_t)K);
  UP(&h->Jq_red, d->Jq_reduced, (size_t)K * Nr);
  UP(&h->c2q, d->c2q, (size_t)K * Nr);
  if (curved) {
    UP(&h->vgeoq, d->vgeoq, (size_t)K * 9 * Nq);
    UP(&h->Jq, d->Jq, (size_t)K * Nq);
    UP(&h->fgeoq, d->fgeoq, (size_t)K * 16 * Nfq);
  }
  for (int i = 0; i < 16; ++i)
    if (ops[i].src) UP(&h->op[i], ops[i].src, ops[i].n);
#undef UP
  // one stage on the zero state (it stays zero) sets the kernels' launch
  // attributes outside any later graph capture
  if (s == BBW_OK) s = stage(h, 0.f, 0.f, 0.f);
  if (s == BBW_OK) s = set_cuda_error(cudaStreamSynchronize(h->stream), "bbw_curved_create");
  if (s != BBW_OK) {
    release(h);
    return s;
  }
  *out = h;
  return BBW_OK;
}

extern "C" bbw_status bbw_curved_destroy(bbw_curved *h) {
  if (!h) return BBW_OK;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  release(h);
  return BBW_OK;
}

static bbw_status copy_state(bbw_curved *h, float *dev, const float *src, float *dst,
                             const char *what) {
  if (!h || (!src && !dst)) return set_error(BBW_ERR_ARG, what);
  const size_t n = (size_t)h->K * 4 * h->Np * sizeof(float);
  cudaError_t e = src ? cudaMemcpyAsync(dev, src, n, cudaMemcpyHostToDevice, h->stream)
                      : cudaMemcpyAsync(dst, dev, n, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return set_cuda_error(e, what);
}

extern "C" bbw_status bbw_curved_set_state(bbw_curved *h, const float *Q) {
  bbw_status s = copy_state(h, h ? h->Q : nullptr, Q, nullptr, "bbw_curved_set_state");
  if (s != BBW_OK) return s;
  const size_t n = (size_t)h->K * 4 * h->Np * sizeof(float);
  return set_cuda_error(cudaMemsetAsync(h->res, 0, n, h->stream), "bbw_curved_set_state");
}

extern "C" bbw_status bbw_curved_get_state(bbw_curved *h, float *Q) {
  return copy_state(h, h ? h->Q : nullptr, nullptr, Q, "bbw_curved_get_state");
}

extern "C" bbw_status bbw_curved_get_residual(bbw_curved *h, float *r) {
  return copy_state(h, h ? h->res : nullptr, nullptr, r, "bbw_curved_get_residual");
}

extern "C" bbw_status bbw_curved_stage(bbw_curved *h, float fa, float fb, float fdt) {
  if (!h) return set_error(BBW_ERR_ARG, "bbw_curved_stage: NULL handle");
  return stage(h, fa, fb, fdt);
}

extern "C" bbw_status bbw_curved_steps(bbw_curved *h, float dt, int nsteps) {
  if (!h || nsteps < 0) return set_error(BBW_ERR_ARG, "bbw_curved_steps: bad argument");
  uint32_t bits;
  std::memcpy(&bits, &dt, 4);
  if (!h->graph || h->graph_dt_bits != bits) {
    if (h->graph) cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_steps: capture");
    bbw_status s = BBW_OK;
    for (int i = 0; i < 5 && s == BBW_OK; ++i)
      s = stage(h, (float)kRK4A[i], (float)kRK4B[i], dt);
    e = cudaStreamEndCapture(h->stream, &g);
    if (s != BBW_OK) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return s;
    }
    if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_steps: end capture");
    e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_steps: instantiate");
    h->graph_dt_bits = bits;
  }
  for (int step = 0; step < nsteps; ++step) {
    cudaError_t e = cudaGraphLaunch(h->graph, h->stream);
    if (e != cudaSuccess) return set_cuda_error(e, "bbw_curved_steps: launch");
  }
  return BBW_OK;
}

extern "C" bbw_status bbw_curved_sync(bbw_curved *h) {
  if (!h) return set_error(BBW_ERR_ARG, "bbw_curved_sync: NULL handle");
  return set_cuda_error(cudaStreamSynchronize(h->stream), "bbw_curved_sync");
}

extern "C" void *bbw_curved_stream(bbw_curved *h) { return h ? (void *)h->stream : nullptr; }
