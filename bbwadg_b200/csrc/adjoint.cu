// Forward / backward pair of the discrete adjoint (receiver-misfit
// gradient with respect to c^2 at the cubature points).
//
// bbw_forward advances the context like bbw_steps (same fused stage, traces
// recorded by the receivers).  Its tape keeps either the pre-c^2 cubature
// values of every stage (when the device has room: on a B200 the 400-step,
// 8-shot N = 4 workload on 24 576 elements takes 90 GB), which is all the
// reverse sweep needs, or the state at every `checkpoint_every`-th step
// start, from which bbw_backward recomputes each segment forward once with
// the same stage kernel.  The stages are reversed with the adjoint kernels
// of kernels_adj.cu.  The c^2 gradient is accumulated in
// FP64.  There is no reference counterpart; the forward operators are the
// reference's rk_volume / rk_surface / rk_update_WADG
// (cpp/okl/WaveKernels.okl:44-260, cpp/okl/WaveKernelsWADG.okl:1760-1887).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "bbwadg.h"
#include "ctx.h"
#include "internal.h"

using namespace bbw;

struct bbw_tape {
  int nsteps = 0, every = 1, step0 = 0;
  float dt = 0.f;
  double t0 = 0.0;
  size_t state = 0;           // floats per state (all shots)
  std::vector<float *> ck;    // step-start states at steps 0, every, 2 every, ...
  float *vq_all = nullptr;    // or: cubature values of every stage, [step][stage][S][Nq][K]
};

namespace bbw {

void adj_release(bbw_ctx *c) {
  AdjOps &a = c->adj;
  for (int d = 0; d < 3; ++d) cudaFree(a.D[d]), cudaFree(a.DT[d]);
  cudaFree(a.LIFT), cudaFree(a.Vq), cudaFree(a.Pq);
  cudaFree(a.Fmask), cudaFree(a.vmapP), cudaFree(a.fidx), cudaFree(a.mapP);
  cudaFree(a.PqT), cudaFree(a.VqT), cudaFree(a.DTp), cudaFree(a.LTp);
  a = AdjOps();
}

}  // namespace bbw

namespace {

// face-node pairing in face-node space from vmapP (vmapP is an involution on
// the face nodes of a conforming mesh)
bbw_status build_maps(const bbw_ctx *c, std::vector<int> &fidx, std::vector<int> &mapP) {
  const int K = c->K, Np = c->Np, Nfp = c->Nfp, NF = 4 * Nfp;
  const int *Fm = c->hFmask.data(), *vm = c->hvmapP.data();
  fidx.assign((size_t)4 * Np, -1);
  for (int f = 0; f < 4; ++f)
    for (int i = 0; i < Nfp; ++i) fidx[(size_t)f * Np + Fm[f * Nfp + i]] = i;
  mapP.assign((size_t)K * NF, -1);
  std::vector<int> inv(Np);
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 4; ++f) {
      const int *v = vm + (size_t)k * NF + f * Nfp;
      const int k2 = v[0] / (4 * Np);
      bool boundary = k2 == k;
      for (int i = 0; i < Nfp && boundary; ++i) boundary = v[i] % (4 * Np) == Fm[f * Nfp + i];
      if (boundary) continue;
      // the face of k2 whose traces point back into k
      int f2 = -1;
      for (int g = 0; g < 4 && f2 < 0; ++g)
        if (vm[(size_t)k2 * NF + g * Nfp] / (4 * Np) == k) f2 = g;
      if (f2 < 0) return set_error(BBW_ERR_MESH, "adjoint: vmapP is not symmetric");
      std::fill(inv.begin(), inv.end(), -1);
      for (int j = 0; j < Nfp; ++j) inv[Fm[f2 * Nfp + j]] = j;
      for (int i = 0; i < Nfp; ++i) {
        const int j = inv[v[i] % (4 * Np)];
        if (j < 0 || vm[(size_t)k2 * NF + f2 * Nfp + j] != k * 4 * Np + Fm[f * Nfp + i])
          return set_error(BBW_ERR_MESH, "adjoint: vmapP is not symmetric");
        mapP[(size_t)k * NF + f * Nfp + i] = k2 * NF + f2 * Nfp + j;
      }
    }
  return BBW_OK;
}

bbw_status adj_setup(bbw_ctx *c) {
  AdjOps &a = c->adj;
  if (a.ready) return BBW_OK;
  const int Np = c->Np, NF = 4 * c->Nfp;
  std::vector<int> fidx, mapP;
  bbw_status s = build_maps(c, fidx, mapP);
  if (s != BBW_OK) return s;
  for (int d = 0; d < 3; ++d) {
    std::vector<float> t((size_t)Np * Np);
    for (int n = 0; n < Np; ++n)
      for (int m = 0; m < Np; ++m) t[n + (size_t)m * Np] = c->hD[d][m + (size_t)n * Np];
    if ((s = upload(&a.D[d], c->hD[d].data(), c->hD[d].size(), "adjoint: D")) != BBW_OK ||
        (s = upload(&a.DT[d], t.data(), t.size(), "adjoint: D^T")) != BBW_OK)
      return s;
  }
  if ((s = upload(&a.LIFT, c->hLIFT.data(), c->hLIFT.size(), "adjoint: LIFT")) != BBW_OK ||
      (s = upload(&a.Vq, c->hVq.data(), c->hVq.size(), "adjoint: Vq")) != BBW_OK ||
      (s = upload(&a.Pq, c->hPq.data(), c->hPq.size(), "adjoint: Pq")) != BBW_OK ||
      (s = upload(&a.Fmask, c->hFmask.data(), c->hFmask.size(), "adjoint: Fmask")) != BBW_OK ||
      (s = upload(&a.vmapP, c->hvmapP.data(), c->hvmapP.size(), "adjoint: vmapP")) != BBW_OK ||
      (s = upload(&a.fidx, fidx.data(), fidx.size(), "adjoint: face index")) != BBW_OK ||
      (s = upload(&a.mapP, mapP.data(), mapP.size(), "adjoint: mapP")) != BBW_OK)
    return s;
  // padded layouts of the reverse-stage kernels (see AdjOps)
  const int Nq = c->Nq, Nfp = c->Nfp;
  const int ldq = (Nq + 3) & ~3, ldp = (Np + 3) & ~3, ldf = (Nfp + 3) & ~3;
  std::vector<float> pt((size_t)Np * ldq, 0.f), vt((size_t)Nq * ldp, 0.f),
      dt((size_t)3 * Np * ldp, 0.f), lt((size_t)4 * Np * ldf, 0.f);
  for (int n = 0; n < Np; ++n)
    for (int q = 0; q < Nq; ++q) {
      pt[(size_t)n * ldq + q] = c->hPq[n + (size_t)q * Np];  // Pq: Np x Nq column-major
      vt[(size_t)q * ldp + n] = c->hVq[q + (size_t)n * Nq];  // Vq: Nq x Np column-major
    }
  for (int d = 0; d < 3; ++d)  // D^T column m, row n = D[m][n]
    for (int m = 0; m < Np; ++m)
      for (int n = 0; n < Np; ++n)
        dt[((size_t)d * Np + m) * ldp + n] = c->hD[d][m + (size_t)n * Np];
  for (int f = 0; f < 4; ++f)
    for (int n = 0; n < Np; ++n)
      for (int j = 0; j < Nfp; ++j)
        lt[((size_t)f * Np + n) * ldf + j] = c->hLIFT[n + (size_t)(f * Nfp + j) * Np];
  if ((s = upload(&a.PqT, pt.data(), pt.size(), "adjoint: Pq^T")) != BBW_OK ||
      (s = upload(&a.VqT, vt.data(), vt.size(), "adjoint: Vq^T")) != BBW_OK ||
      (s = upload(&a.DTp, dt.data(), dt.size(), "adjoint: D^T")) != BBW_OK ||
      (s = upload(&a.LTp, lt.data(), lt.size(), "adjoint: LIFT^T")) != BBW_OK)
    return s;
  (void)NF;
  a.ready = true;
  return BBW_OK;
}

struct DevBuf {  // freed on scope exit
  std::vector<void *> p;
  ~DevBuf() {
    for (void *x : p) cudaFree(x);
  }
  template <class T>
  bbw_status get(T **out, size_t n, const char *what) {
    bbw_status s = upload<T>(out, nullptr, n, what);
    if (s == BBW_OK) p.push_back(*out);
    return s;
  }
};

}  // namespace

extern "C" bbw_status bbw_set_c2q(bbw_ctx *c, const float *c2q) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !c2q) return set_error(BBW_ERR_ARG, "bbw_set_c2q: NULL");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->c2q, c2q, (size_t)c->K * c->Nq * sizeof(float), cudaMemcpyHostToDevice);
  return set_cuda_error(e, "bbw_set_c2q");
}

extern "C" bbw_status bbw_tape_free(bbw_tape *t) {
  if (!t) return BBW_OK;
  for (float *p : t->ck) cudaFree(p);
  cudaFree(t->vq_all);
  delete t;
  return BBW_OK;
}

extern "C" int bbw_tape_kind(const bbw_tape *t) { return t && t->vq_all ? 1 : 0; }

extern "C" bbw_status bbw_forward(bbw_ctx *c, float dt, int nsteps, int checkpoint_every,
                                  bbw_tape **out) {
  return bbw_forward_ex(c, dt, nsteps, checkpoint_every, BBW_TAPE_CUBATURE, out);
}

extern "C" bbw_status bbw_forward_ex(bbw_ctx *c, float dt, int nsteps, int checkpoint_every,
                                     int keep, bbw_tape **out) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !out || nsteps < 1 || checkpoint_every < 1 || !(dt > 0.f) ||
      (keep != BBW_TAPE_CHECKPOINTS && keep != BBW_TAPE_CUBATURE))
    return set_error(BBW_ERR_ARG, "bbw_forward: bad argument");
  *out = nullptr;
  if (c->R <= 0) return set_error(BBW_ERR_STATE, "bbw_forward: no receivers set");
  if (c->gs)
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_forward: no adjoint in the GEMM precision form");
  if (c->plan.Kc > 0 && c->plan.Kc < c->K)
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_forward: the adjoint needs the whole mesh (no halo)");
  bbw_status s = adj_setup(c);
  if (s != BBW_OK) return s;
  double t0 = 0;
  int st0 = 0;
  if ((s = bbw_get_time(c, &t0, &st0)) != BBW_OK) return s;
  if (st0 + nsteps > c->max_steps)
    return set_error(BBW_ERR_ARG, "bbw_forward: receiver capacity (max_steps) too small");
  bbw_tape *t = new bbw_tape;
  t->nsteps = nsteps, t->every = checkpoint_every, t->step0 = st0, t->dt = dt, t->t0 = t0;
  t->state = (size_t)c->S * c->K * 4 * c->Np;
  const size_t vqn = (size_t)c->S * c->Nq * c->K;  // cubature values per stage
  if (keep == BBW_TAPE_CUBATURE) {
    size_t fr = 0, tot = 0;
    const size_t need = (size_t)nsteps * 5 * vqn * sizeof(float);
    void *p = nullptr;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && need + ((size_t)4 << 30) < fr &&
        cudaMalloc(&p, need) == cudaSuccess)
      t->vq_all = static_cast<float *>(p);  // every entry is written by the forward stages
    cudaGetLastError();  // no room after all: checkpoints
  }
  if (t->vq_all) {
    for (int n = 0; n < nsteps; ++n)
      if ((s = step_storing_cubature(c, dt, t->vq_all + (size_t)n * 5 * vqn, vqn)) != BBW_OK) {
        bbw_tape_free(t);
        return s;
      }
    *out = t;
    return BBW_OK;
  }
  const int nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
  for (int i = 0; i < nck; ++i) {
    float *p = nullptr;
    if ((s = upload<float>(&p, nullptr, t->state, "bbw_forward: checkpoint")) != BBW_OK) {
      bbw_tape_free(t);
      return s;
    }
    t->ck.push_back(p);
  }
  for (int n = 0; n < nsteps; ++n) {
    if (n % checkpoint_every == 0) {
      float *Q = nullptr;
      bbw_device_state(c, &Q, nullptr, nullptr);
      cudaError_t e = cudaMemcpyAsync(t->ck[n / checkpoint_every], Q, t->state * sizeof(float),
                                      cudaMemcpyDeviceToDevice, c->stream);
      if (e != cudaSuccess) {
        bbw_tape_free(t);
        return set_cuda_error(e, "bbw_forward: checkpoint");
      }
    }
    if ((s = bbw_steps(c, dt, 1)) != BBW_OK) {
      bbw_tape_free(t);
      return s;
    }
  }
  *out = t;
  return BBW_OK;
}

extern "C" bbw_status bbw_backward(bbw_ctx *c, bbw_tape *t, const float *dL_dtraces,
                                   double *dL_dc2q, float *dL_dQ0) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !t || !dL_dtraces || !dL_dc2q) return set_error(BBW_ERR_ARG, "bbw_backward: NULL");
  if (t->state != (size_t)c->S * c->K * 4 * c->Np)
    return set_error(BBW_ERR_STATE, "bbw_backward: tape does not match the context");
  bbw_status s = adj_setup(c);
  if (s != BBW_OK) return s;
  const int N = c->N, K = c->K, Np = c->Np, Nq = c->Nq, NF = 4 * c->Nfp, S = c->S, R = c->R;
  const int nsteps = t->nsteps, every = t->every;
  const float dt = t->dt;
  cudaStream_t st = c->stream;
  const AdjOps &a = c->adj;
  DevBuf buf;
  float *lamQ, *lamR, *z, *rhs, *sigma, *res, *g, *seg = nullptr, *stq = nullptr, *vq = nullptr;
  double *grad, *tdev;
  const int seglen = std::min(every, nsteps);
  const bool full = t->vq_all != nullptr;  // the tape holds every stage's cubature values
  if ((s = buf.get(&lamQ, t->state, "bbw_backward")) != BBW_OK ||
      (s = buf.get(&lamR, t->state, "bbw_backward")) != BBW_OK ||
      (s = buf.get(&z, t->state, "bbw_backward")) != BBW_OK ||
      (s = buf.get(&rhs, t->state, "bbw_backward")) != BBW_OK ||
      (s = buf.get(&sigma, (size_t)S * K * NF, "bbw_backward")) != BBW_OK ||
      (s = buf.get(&res, t->state, "bbw_backward")) != BBW_OK ||
      (s = buf.get(&g, (size_t)S * R * nsteps, "bbw_backward")) != BBW_OK ||
      (s = buf.get(&grad, (size_t)K * Nq, "bbw_backward")) != BBW_OK ||
      (s = buf.get(&tdev, 1, "bbw_backward")) != BBW_OK)
    return s;
  if (!full &&
      ((s = buf.get(&seg, (size_t)seglen * t->state, "bbw_backward: segment states")) != BBW_OK ||
       (s = buf.get(&stq, (size_t)5 * t->state, "bbw_backward: stage states")) != BBW_OK ||
       (s = buf.get(&vq, (size_t)5 * S * Nq * K, "bbw_backward: cubature values")) != BBW_OK))
    return s;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess)
    e = cudaMemcpy(g, dL_dtraces, (size_t)S * R * nsteps * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_backward: upload");

  FusedPlan pl = c->plan;
  pl.time = tdev;
  TcPlan tpl = c->tc;
  tpl.time = tdev;
  // one forward stage of the recomputation in the context's own form (FP32
  // fused or tensor-core stage, bit-identical to the forward pass),
  // optionally storing Vq S(Q)_p at the cubature points
  auto launch = [&](int i, const float *in, float *outq, float *vqo) {
    const float cs = c->src_stage_times ? (float)kRK4C[i] : 0.f;
    if (c->precision != BBW_PREC_FP32) {
      TcPlan tp = tpl;
      tp.vq_out = vqo;
      return tc_launch(tp, in, outq, res, (float)kRK4A[i], (float)kRK4B[i], dt, cs, st);
    }
    FusedPlan p = pl;
    p.vq_out = vqo;
    return fused_launch(p, in, outq, res, (float)kRK4A[i], (float)kRK4B[i], dt, cs, st);
  };
  // step-start times exactly as the device clock accumulated them
  std::vector<double> tn(nsteps + 1);
  tn[0] = t->t0;
  for (int n = 0; n < nsteps; ++n) tn[n + 1] = tn[n] + (double)dt;
  auto stage = [&](int i, const float *in, float *outq) { return launch(i, in, outq, nullptr); };
  const size_t vqn = (size_t)S * Nq * K;  // per stage
  auto stage_v = [&](int i, const float *in, float *outq) {  // also storing Vq S(Q)_p
    return launch(i, in, outq, vq + (size_t)i * vqn);
  };
  auto step_fwd = [&](int n, const float *in, float *outq) {  // stage outputs in stq[1..4]
    bbw_status r = set_device_double(tdev, tn[n], st);
    const float *q = in;
    for (int i = 0; i < 5 && r == BBW_OK; ++i) {
      float *o = i < 4 ? stq + (size_t)(i + 1) * t->state : outq;
      r = stage(i, q, o);
      q = o;
    }
    return r;
  };

  // Segment store: when the device has room, one forward pass per segment
  // keeps the cubature values of every stage of the segment (vq_all), so the
  // reverse sweep needs no second recomputation (the adjoint stages need only
  // those values, not the forward states).
  float *vq_all = nullptr;
  if (!full) {
    size_t fr = 0, tot = 0;
    const size_t need = (size_t)seglen * 5 * vqn * sizeof(float);
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && need + ((size_t)2 << 30) < fr &&
        buf.get(&vq_all, (size_t)seglen * 5 * vqn, "bbw_backward") != BBW_OK)
      vq_all = nullptr;  // fall back to recomputing each step again in the sweep
  }
  const int nseg = (nsteps + every - 1) / every;
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int n0 = sg * every, len = std::min(every, nsteps - n0);
    if (full) {
      // nothing to recompute
    } else if (vq_all) {
      // forward over the segment; stage outputs chain through stq[1..4] and
      // the step outputs alternate between z and seg
      const float *q = t->ck[sg];
      for (int j = 0; j < len; ++j) {
        if ((s = set_device_double(tdev, tn[n0 + j], st)) != BBW_OK) return s;
        float *out = (j & 1) ? seg : z;
        const float *qi = q;
        for (int i = 0; i < 5; ++i) {
          float *o = i < 4 ? stq + (size_t)(i + 1) * t->state : out;
          if ((s = launch(i, qi, o, vq_all + ((size_t)j * 5 + i) * vqn)) != BBW_OK) return s;
          qi = o;
        }
        q = out;
      }
    } else {
      e = cudaMemcpyAsync(seg, t->ck[sg], t->state * sizeof(float), cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return set_cuda_error(e, "bbw_backward: segment");
      for (int j = 1; j < len; ++j)
        if ((s = step_fwd(n0 + j - 1, seg + (size_t)(j - 1) * t->state,
                          seg + (size_t)j * t->state)) != BBW_OK)
          return s;
    }
    for (int j = len - 1; j >= 0; --j) {
      const int n = n0 + j;
      if ((s = adj_receivers(S, K, Np, R, c->rec_elem, c->rec_w, g, nsteps, n, lamQ, st)) !=
          BBW_OK)
        return s;
      const float *vqs = vq;
      if (full) {
        vqs = t->vq_all + (size_t)n * 5 * vqn;
      } else if (vq_all) {
        vqs = vq_all + (size_t)j * 5 * vqn;
      } else {
        // the step's five stages again from its start state (bit-identical
        // to the forward), keeping each stage's Vq S(Q)_p; the step's output
        // goes to z (scratch until the adjoint stages below overwrite it)
        if ((s = set_device_double(tdev, tn[n], st)) != BBW_OK) return s;
        const float *q = seg + (size_t)j * t->state;
        for (int i = 0; i < 5 && s == BBW_OK; ++i) {
          float *o = i < 4 ? stq + (size_t)(i + 1) * t->state : z;
          s = stage_v(i, q, o);
          q = o;
        }
        if (s != BBW_OK) return s;
      }
      for (int i = 4; i >= 0; --i) {
        const float ai = (float)kRK4A[i], bi = (float)kRK4B[i];
        if ((s = adj_wadg(N, S, K, Nq, a.PqT, a.VqT, pl.c2q, lamQ, lamR, ai, bi, dt,
                          vqs + (size_t)i * vqn, z, grad, st)) != BBW_OK ||
            (s = adj_volume(N, S, K, c->vgeo, a.DTp, z, rhs, st)) != BBW_OK ||
            (s = adj_sigma(N, S, K, c->fgeo, a.LTp, z, sigma, st)) != BBW_OK ||
            (s = adj_gather(N, S, K, c->bc, dt, c->fgeo, a.fidx, a.mapP, sigma, rhs, lamQ, st)) !=
                BBW_OK)
          return s;
      }
    }
  }
  e = cudaStreamSynchronize(st);
  std::vector<double> gq((size_t)K * Nq);  // device layout [Nq][K]
  if (e == cudaSuccess)
    e = cudaMemcpy(gq.data(), grad, gq.size() * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    for (int k = 0; k < K; ++k)
      for (int q = 0; q < Nq; ++q) dL_dc2q[(size_t)k * Nq + q] = gq[(size_t)q * K + k];
  if (e == cudaSuccess && dL_dQ0)
    e = cudaMemcpy(dL_dQ0, lamQ, t->state * sizeof(float), cudaMemcpyDeviceToHost);
  return set_cuda_error(e, "bbw_backward: download");
}
