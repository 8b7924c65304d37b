// Solver context of the C ABI: device-resident mesh, operators and state,
// fused stage launches and CUDA-graph-captured LSRK45 steps.
//
// Replaces the module-level OCCA buffers and host driver of the reference
// (cpp/src/WaveOKL3d.cpp:12-135 globals, WaveInitOCCA3d :1400-1680,
// InitWADG_subelem :419-915, RK_step_WADG_subelem :2084-2109,
// Wave_RK :2014-2081, WaveSetData3d / WaveGetData3d :2527-2558).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "bbwadg.h"
#include "device_common.cuh"
#include "fused.h"
#include "ctx.h"
#include "internal.h"

namespace bbw {

// LSRK45 coefficients (Carpenter-Kennedy), cpp/src/StartUp3d.cpp:517-529
const double kRK4A[5] = {0.0, -567301805773.0 / 1357537059087.0,
                                -2404267990393.0 / 2016746695238.0,
                                -3550918686646.0 / 2091501179385.0,
                                -1275806237668.0 / 842570457699.0};
const double kRK4B[5] = {1432997174477.0 / 9575080441755.0,
                                5161836677717.0 / 13612068292357.0,
                                1720146321549.0 / 2090206949498.0,
                                3134564353537.0 / 4481467310338.0,
                                2277821191437.0 / 14882151754819.0};
// stage times t + rk4c[s] dt, cpp/src/StartUp3d.cpp:531-537
const double kRK4C[5] = {0.0, 1432997174477.0 / 9575080441755.0,
                                2526269341429.0 / 6820363962896.0,
                                2006345519317.0 / 3224310063776.0,
                                2802321613138.0 / 2924317926251.0};

static int round4i(int x) { return (x + 3) & ~3; }
static int cdivi(int a, int b) { return (a + b - 1) / b; }

}  // namespace bbw

using namespace bbw;

namespace {

void release(bbw_ctx *c) {
  if (!c) return;
  if (c->gs) {
    gemm_stage_release(*c->gs);
    delete c->gs;
    c->gs = nullptr;
  }
  for (int i = 0; i < 2; ++i)
    if (c->step_graph[i]) cudaGraphExecDestroy(c->step_graph[i]);
  cudaFree(c->Q[0]);
  cudaFree(c->Q[1]);
  cudaFree(c->res);
  cudaFree(c->vgeo);
  cudaFree(c->fgeo);
  cudaFree(c->c2q);
  cudaFree(c->ops);
  cudaFree(c->nbr);
  cudaFree(c->tables);
  cudaFree(c->d_time);
  cudaFree(c->d_step);
  cudaFree(c->src_off);
  cudaFree(c->src_elem);
  cudaFree(c->src_tile);
  cudaFree(c->src_vec);
  cudaFree(c->rec_elem);
  cudaFree(c->rec_w);
  cudaFree(c->traces);
  cudaFree(c->geo_tc);
  cudaFree(c->ops_tc);
  cudaFree(c->err);
  adj_release(c);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // namespace

namespace bbw {

// Operators packed per thread group for the fused kernel with W thread
// groups (row blocks) per CTA:
//   vol  [W][Np(m)][P3R]  rows in pairs p = i/2: Dr, Ds, Dt of row r0+i at
//                         6p + (i%2) + {0, 2, 4}                      (nodal)
//   lift [W][NF(m)][PR]   LIFT[r0+i][m]                           (nodal)
//   pq   [W][Nq(q)][PR]   Pq[r0+i][q]
//   vq   [W][Np(n)][PRQ]  Vq[q0+i][n]
// rows r0 = w R, R = ceil(Np / W); cubature rows q0 = w RQ, RQ = ceil(Nq / W).
void pack_fused_ops(int N, int Nq, int W, bool bb, const float *Dr, const float *Ds,
                    const float *Dt, const float *LIFT, const float *Vq, const float *Pq,
                    FusedOps &out) {
  const int Np = np_of(N), NF = 4 * nfp_of(N);
  const int R = cdivi(Np, W), PR = round4i(R), P3R = round4i(6 * cdivi(R, 2));
  const int RQ = cdivi(Nq, W), QB = fused_vq_block(W), PRQ = cdivi(RQ, QB) * QB;
  std::vector<float> &ops = out.ops;
  ops.clear();
  if (!bb) {
    std::vector<float> vol((size_t)W * Np * P3R, 0.f), lift((size_t)W * NF * PR, 0.f);
    for (int w = 0; w < W; ++w)
      for (int i = 0; i < R; ++i) {
        const int r = w * R + i;
        if (r >= Np) continue;
        for (int mm = 0; mm < Np; ++mm) {  // row pairs: (Dr, Dr', Ds, Ds', Dt, Dt')
          float *d = &vol[((size_t)w * Np + mm) * P3R + 6 * (i / 2) + (i % 2)];
          d[0] = Dr[r + mm * Np], d[2] = Ds[r + mm * Np], d[4] = Dt[r + mm * Np];
        }
        for (int mm = 0; mm < NF; ++mm) lift[((size_t)w * NF + mm) * PR + i] = LIFT[r + mm * Np];
      }
    ops.insert(ops.end(), vol.begin(), vol.end());
    out.off_lift = (int)ops.size();
    ops.insert(ops.end(), lift.begin(), lift.end());
  } else {
    out.off_lift = 0;
  }
  out.off_pq = (int)ops.size();
  std::vector<float> pq((size_t)W * Nq * PR, 0.f), vq((size_t)W * Np * PRQ, 0.f);
  for (int w = 0; w < W; ++w) {
    for (int i = 0; i < R; ++i) {
      const int r = w * R + i;
      if (r < Np)
        for (int q = 0; q < Nq; ++q) pq[((size_t)w * Nq + q) * PR + i] = Pq[r + q * Np];
    }
    for (int i = 0; i < RQ; ++i) {
      const int q = w * RQ + i;
      if (q < Nq)
        for (int n = 0; n < Np; ++n) vq[((size_t)w * Np + n) * PRQ + i] = Vq[q + n * Nq];
    }
  }
  ops.insert(ops.end(), pq.begin(), pq.end());
  out.off_vq = (int)ops.size();
  ops.insert(ops.end(), vq.begin(), vq.end());
  out.RQ = RQ, out.PRQ = PRQ;
}

}  // namespace bbw

namespace {

// Dense operators of the context's basis, kept on the host for the adjoint.
// Nodal: the given Dr, Ds, Dt, LIFT.  BB: the same linear maps assembled
// from the sparse forms the BB kernels apply (cpp/okl/WaveKernels.okl:
// 428-467 derivative, :576-644 L0 then EEL lift).
void dense_operators(int N, int Nq, const bbw_ops_desc *o, bool bb, bbw_ctx *c) {
  const int Np = np_of(N), Nfp = nfp_of(N), NF = 4 * Nfp;
  for (int d = 0; d < 3; ++d) c->hD[d].assign((size_t)Np * Np, 0.f);
  c->hLIFT.assign((size_t)Np * NF, 0.f);
  c->hVq.assign(o->Vq, o->Vq + (size_t)Nq * Np);
  c->hPq.assign(o->Pq, o->Pq + (size_t)Np * Nq);
  if (!bb) {
    const float *Dd[3] = {o->Dr, o->Ds, o->Dt};
    for (int d = 0; d < 3; ++d) c->hD[d].assign(Dd[d], Dd[d] + (size_t)Np * Np);
    c->hLIFT.assign(o->LIFT, o->LIFT + (size_t)Np * NF);
    return;
  }
  // dpdr = .5 (p2 - p1), dpds = .5 (p3 - p1), dpdt = .5 (p4 - p1) with
  // p_c = sum_j Dvals[n].j p[Dj_ids[n].c]; column-major D[n + col Np]
  const int *Dp[4] = {o->D_ids1, o->D_ids2, o->D_ids3, o->D_ids4};
  std::vector<double> acc[3];
  for (int d = 0; d < 3; ++d) acc[d].assign((size_t)Np * Np, 0.0);
  for (int n = 0; n < Np; ++n)
    for (int j = 0; j < 4; ++j) {
      const double v = o->Dvals4[4 * n + j];
      const int *id = Dp[j] + 4 * n;
      for (int d = 0; d < 3; ++d) {
        acc[d][n + (size_t)id[d + 1] * Np] += .5 * v;
        acc[d][n + (size_t)id[0] * Np] -= .5 * v;
      }
    }
  for (int d = 0; d < 3; ++d)
    for (size_t i = 0; i < acc[d].size(); ++i) c->hD[d][i] = (float)acc[d][i];
  // LIFT[n][f Nfp + i] = sum over EEL entries (n, f Nfp + i') of EEL * L0[i'][i]
  const int L0 = o->L0_nnz;
  std::vector<double> lift((size_t)Np * NF, 0.0);
  for (int n = 0; n < Np; ++n)
    for (int j = 0; j < o->EEL_nnz; ++j) {
      const int col = o->EEL_ids[n + j * Np];
      const double ev = o->EEL_vals[n + j * Np];
      if (ev == 0.0 || col < 0 || col >= NF) continue;
      const int f = col / Nfp, ip = col - f * Nfp;
      for (int l = 0; l < L0; ++l) {
        const int i = o->L0_ids[ip + l * Nfp];
        if (i < 0 || i >= Nfp) continue;
        lift[n + (size_t)(f * Nfp + i) * Np] += ev * o->L0_vals[ip + l * Nfp];
      }
    }
  for (size_t i = 0; i < lift.size(); ++i) c->hLIFT[i] = (float)lift[i];
}

// vmapP -> per face (neighbour << 8 | permutation id), permutation table
bbw_status compress_connectivity(int N, int K, const int *Fmask, const int *vmapP,
                                 std::vector<int> &nbr, std::vector<int> &pats, int &npat) {
  const int Np = np_of(N), Nfp = nfp_of(N), NF = 4 * Nfp;
  nbr.assign((size_t)K * 4, 0);
  pats.clear();
  npat = 0;
  std::map<std::vector<int>, int> index;
  std::vector<int> p(Nfp);
  for (int k = 0; k < K; ++k)
    for (int f = 0; f < 4; ++f) {
      const int *v = vmapP + (size_t)k * NF + f * Nfp;
      const long long k2 = v[0] / (4 * Np);
      bool boundary = true;
      for (int j = 0; j < Nfp; ++j) {
        if (v[j] < 0 || v[j] / (4 * Np) != k2 || v[j] % (4 * Np) >= Np)
          return set_error(BBW_ERR_MESH, "vmapP: trace index outside the p field of one element");
        p[j] = v[j] % (4 * Np);
        boundary = boundary && k2 == k && p[j] == Fmask[f * Nfp + j];
      }
      if (k2 >= K) return set_error(BBW_ERR_MESH, "vmapP: neighbour out of range");
      if (boundary) {
        nbr[4 * (size_t)k + f] = (int)(k << 8) | 255;
        continue;
      }
      if (k2 == k)
        return set_error(BBW_ERR_MESH, "vmapP: face maps partly onto its own element");
      auto it = index.find(p);
      int id;
      if (it == index.end()) {
        if (npat >= 255) return set_error(BBW_ERR_MESH, "vmapP: too many face permutations");
        id = npat++;
        index[p] = id;
        pats.insert(pats.end(), p.begin(), p.end());
      } else {
        id = it->second;
      }
      nbr[4 * (size_t)k + f] = (int)(k2 << 8) | id;
    }
  return BBW_OK;
}

}  // namespace

extern "C" bbw_status bbw_create(const bbw_mesh_desc *m, const bbw_ops_desc *o, int variant,
                                 int bc, bbw_ctx **out) {
  return bbw_create_ex(m, o, variant, bc, BBW_PREC_FP32, out);
}

extern "C" bbw_status bbw_create_ex(const bbw_mesh_desc *m, const bbw_ops_desc *o, int variant,
                                    int bc, int precision, bbw_ctx **out) {
  if (!out) return set_error(BBW_ERR_ARG, "bbw_create: out is NULL");
  *out = nullptr;
  if (!m || !o || (variant != BBW_NODAL && variant != BBW_BB) || (bc != 0 && bc != 1) ||
      (precision != BBW_PREC_FP32 && precision != BBW_PREC_F16X3 &&
       precision != BBW_PREC_BF16X3 && precision != BBW_PREC_TF32))
    return set_error(BBW_ERR_ARG, "bbw_create: bad argument");
  // split pairs on the fused tensor-core stage where it fits; TF32, and
  // split pairs beyond it, on the GEMM form (gemm_stage.cu)
  const bool split = precision == BBW_PREC_F16X3 || precision == BBW_PREC_BF16X3;
  const bool gemm = precision == BBW_PREC_TF32 || (split && !tc_supported(m->N, m->Nq));
  const bool tcp = split && !gemm;
  const int N = m->N, K = m->K, Nq = m->Nq;
  if (N < 1 || N > BBW_MAX_N) return set_error(BBW_ERR_UNSUPPORTED, "bbw_create: N out of range");
  if (K <= 0 || K >= (1 << 23) || Nq <= 0)
    return set_error(BBW_ERR_ARG, "bbw_create: K must be in [1, 2^23), Nq > 0");
  if (!m->vgeo || !m->fgeo || !m->Fmask || !m->vmapP || !m->c2q || !o->Vq || !o->Pq)
    return set_error(BBW_ERR_ARG, "bbw_create: missing mesh or WADG array");
  const bool bb = variant == BBW_BB;
  if (!bb && (!o->Dr || !o->Ds || !o->Dt || !o->LIFT))
    return set_error(BBW_ERR_ARG, "bbw_create: nodal operators missing");
  if (bb && (!o->D_ids1 || !o->D_ids2 || !o->D_ids3 || !o->D_ids4 || !o->Dvals4 ||
             !o->EEL_ids || !o->EEL_vals || !o->L0_ids || !o->L0_vals || o->EEL_nnz <= 0 ||
             o->L0_nnz <= 0))
    return set_error(BBW_ERR_ARG, "bbw_create: BB operators missing");
  const int Np = np_of(N), Nfp = nfp_of(N), NF = 4 * Nfp;
  // the fused stage skips the velocity rows of the WADG update (Pq*Vq = I),
  // which requires Jq = 1 (affine elements)
  std::vector<float> c2J((size_t)K * Nq);
  for (size_t i = 0; i < c2J.size(); ++i) {
    const float J = m->Jq ? m->Jq[i] : 1.f;
    if (J != 1.f)
      return set_error(BBW_ERR_UNSUPPORTED,
                       "bbw_create: fused stage needs Jq = 1 (affine elements); use the "
                       "kernel-level entry points for curved Jacobians");
    c2J[i] = m->c2q[i];
  }
  std::vector<int> nbr, pats;
  int npat = 0;
  bbw_status s = compress_connectivity(N, K, m->Fmask, m->vmapP, nbr, pats, npat);
  if (s != BBW_OK) return s;

  // ---- pack operators in the per-warp layouts of the fused kernel
  for (int i = 0; i < NF; ++i)
    if (m->Fmask[i] < 0 || m->Fmask[i] >= Np)
      return set_error(BBW_ERR_ARG, "bbw_create: Fmask entry out of range");
  const int W = fused_default_warps(N), E = fused_default_tile(N);
  FusedOps fo;
  pack_fused_ops(N, Nq, fused_groups(W, E), bb, o->Dr, o->Ds, o->Dt, o->LIFT, o->Vq, o->Pq, fo);
  const std::vector<float> &ops = fo.ops;
  const int off_lift = fo.off_lift, off_pq = fo.off_pq, off_vq = fo.off_vq;
  const int RQ = fo.RQ, PRQ = fo.PRQ;
  // ---- integer tables: Fmask | patterns | BB tables
  std::vector<int> tab(m->Fmask, m->Fmask + NF);
  tab.resize(round4i((int)tab.size()), 0);
  const int pat_off = (int)tab.size();
  tab.insert(tab.end(), pats.begin(), pats.end());
  // the fused stage zero-fills the neighbour codes past the last element of
  // a ragged tile (neighbour 0, permutation 0) and reads their traces too;
  // with no interior face (a single element) permutation 0 would not exist,
  // so give it one row of valid node ids
  if (npat == 0) tab.insert(tab.end(), (size_t)Nfp, 0);
  tab.resize(round4i((int)tab.size()), 0);
  const int bb_off = (int)tab.size();
  if (bb) {
    const int *Dp[4] = {o->D_ids1, o->D_ids2, o->D_ids3, o->D_ids4};
    for (int d = 0; d < 4; ++d) tab.insert(tab.end(), Dp[d], Dp[d] + 4 * Np);
    for (int i = 0; i < 4 * Np; ++i) {
      int bits;
      std::memcpy(&bits, &o->Dvals4[i], 4);
      tab.push_back(bits);
    }
    // header, L0 and EEL as (face-node row, value bits) pairs
    const int L0 = o->L0_nnz;
    auto bits = [](float v) {
      int b;
      std::memcpy(&b, &v, 4);
      return b;
    };
    // EEL as CSR with the nonzeros of each row bucketed by face
    std::vector<int> ptr((size_t)Np * 5);
    std::vector<int> pairs;
    for (int n = 0; n < Np; ++n)
      for (int f = 0; f < 4; ++f) {
        ptr[(size_t)n * 5 + f] = (int)pairs.size() / 2;
        for (int j = 0; j < o->EEL_nnz; ++j) {
          const int c = o->EEL_ids[n + j * Np];
          const float v = o->EEL_vals[n + j * Np];
          if (c < 0 || c >= NF) return set_error(BBW_ERR_ARG, "bbw_create: EEL id out of range");
          if (v != 0.f && c / Nfp == f) pairs.push_back(c), pairs.push_back(bits(v));
        }
        if (f == 3) ptr[(size_t)n * 5 + 4] = (int)pairs.size() / 2;
      }
    tab.push_back(L0);
    tab.push_back((int)pairs.size() / 2);
    tab.push_back(0);
    tab.push_back(0);
    for (int nt = 0; nt < Nfp; ++nt)
      for (int j = 0; j < L0; ++j) {
        tab.push_back(o->L0_ids[nt + j * Nfp]);
        tab.push_back(bits(o->L0_vals[nt + j * Nfp]));
      }
    tab.insert(tab.end(), ptr.begin(), ptr.end());
    if (tab.size() % 2) tab.push_back(0);
    tab.insert(tab.end(), pairs.begin(), pairs.end());
    for (int i = 0; i < Np; ++i)
      for (int d = 0; d < 4; ++d)
        for (int c = 0; c < 4; ++c) {
          const int id = Dp[d][4 * i + c];
          if (id < 0 || id >= Np) return set_error(BBW_ERR_ARG, "bbw_create: D id out of range");
        }
    for (int i = 0; i < Nfp * L0; ++i)
      if (o->L0_ids[i] < 0 || o->L0_ids[i] >= Nfp)
        return set_error(BBW_ERR_ARG, "bbw_create: L0 id out of range");
  }
  tab.resize(round4i((int)tab.size()), 0);

  bbw_ctx *c = new bbw_ctx;
  c->N = N, c->K = K, c->Nq = Nq, c->Np = Np, c->Nfp = Nfp, c->variant = variant, c->bc = bc;
  dense_operators(N, Nq, o, bb, c);
  c->hFmask.assign(m->Fmask, m->Fmask + NF);
  c->hvmapP.assign(m->vmapP, m->vmapP + (size_t)K * NF);
  cudaGetDevice(&c->device);
  const size_t nstate = (size_t)K * 4 * Np;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return set_cuda_error(e, "bbw_create: stream");
  }
  if ((s = upload<float>(&c->Q[0], nullptr, nstate, "bbw_create: Q")) != BBW_OK ||
      (s = upload<float>(&c->Q[1], nullptr, nstate, "bbw_create: Q")) != BBW_OK ||
      (s = upload<float>(&c->res, nullptr, nstate, "bbw_create: res")) != BBW_OK ||
      (s = upload(&c->vgeo, m->vgeo, (size_t)K * 9, "bbw_create: vgeo")) != BBW_OK ||
      (s = upload(&c->fgeo, m->fgeo, (size_t)K * 16, "bbw_create: fgeo")) != BBW_OK ||
      (s = upload(&c->c2q, c2J.data(), c2J.size(), "bbw_create: c2q")) != BBW_OK ||
      (s = upload(&c->nbr, nbr.data(), nbr.size(), "bbw_create: connectivity")) != BBW_OK ||
      (s = upload(&c->ops, ops.data(), ops.size(), "bbw_create: operators")) != BBW_OK ||
      (s = upload(&c->tables, tab.data(), tab.size(), "bbw_create: tables")) != BBW_OK ||
      (s = upload<double>(&c->d_time, nullptr, 1, "bbw_create: clock")) != BBW_OK ||
      (s = upload<int>(&c->d_step, nullptr, 1, "bbw_create: clock")) != BBW_OK) {
    release(c);
    return s;
  }
  FusedPlan &pl = c->plan;
  pl.N = N, pl.K = K, pl.Nq = Nq, pl.RQ = RQ, pl.PRQ = PRQ, pl.bc = bc, pl.npat = npat;
  pl.bb = bb;
  pl.vgeo = c->vgeo, pl.fgeo = c->fgeo, pl.c2q = c->c2q, pl.nbr = c->nbr;
  pl.ops = c->ops, pl.ops_floats = (int)ops.size();
  pl.off_lift = off_lift, pl.off_pq = off_pq, pl.off_vq = off_vq;
  pl.tables = c->tables, pl.table_ints = (int)tab.size(), pl.pat_off = pat_off, pl.bb_off = bb_off;
  pl.S = 1, pl.time = c->d_time, pl.W = W, pl.E = E;
  if ((s = fused_prepare(pl)) != BBW_OK) {
    release(c);
    return s;
  }
  c->precision = precision;
  if (gemm) {
    c->gs = new GemmStage;
    if ((s = gemm_stage_create(*c->gs, N, K, Nq, bc, precision, c->hD, c->hLIFT, c->hVq,
                               c->hPq)) != BBW_OK) {
      release(c);
      return s;
    }
  }
  if (tcp) {
    // geometry records, split-FP16 / split-BF16 operators in the canonical
    // K-major layout
    TcPlan &tp = c->tc;
    tp.N = N, tp.K = K, tp.Nq = Nq, tp.bc = bc, tp.bf = precision == BBW_PREC_BF16X3;
    // Fmask and the face permutations only: the BB tables after them serve
    // the FP32 stage (the tensor-core stage applies dense BB operators)
    tp.table_ints = bb_off, tp.pat_off = pat_off;
    tp.L = tc_layout(N, Nq, tp.table_ints);
    const TcLayout &TL = tp.L;
    std::vector<float> geo((size_t)K * TC_GEO, 0.f);
    for (int k = 0; k < K; ++k) {
      std::memcpy(&geo[(size_t)k * TC_GEO], m->fgeo + (size_t)k * 16, 16 * sizeof(float));
      std::memcpy(&geo[(size_t)k * TC_GEO + 16], m->vgeo + (size_t)k * 9, 9 * sizeof(float));
    }
    // operator planes with MR (MRQ) stored rows, see tc_layout.  The dense
    // operators of the context's basis: for BB the dense equivalents of the
    // sparse derivative and of the L0 + degree-elevation lift
    // (dense_operators), applied to BB coefficients as the reference's
    // rk_volume_bern / rk_surface_bern do (cpp/okl/WaveKernels.okl:344-647)
    std::vector<uint16_t> h(TL.ops_halfs);
    const int MR = TL.MR, MRQ = TL.MRQ;
    for (int d = 0; d < 3; ++d)
      tc_pack_operator(c->hD[d].data(), Np, Np, 1, Np, MR, TL.KV, &h[TL.oD + 2 * d * MR * TL.KV],
                       &h[TL.oD + (2 * d + 1) * MR * TL.KV], tp.bf);
    for (int f = 0; f < 4; ++f)
      tc_pack_operator(c->hLIFT.data() + (size_t)f * Nfp * Np, Np, Nfp, 1, Np, MR, TL.KF,
                       &h[TL.oL + 2 * f * MR * TL.KF], &h[TL.oL + (2 * f + 1) * MR * TL.KF],
                       tp.bf);
    tc_pack_operator(c->hPq.data(), Np, Nq, 1, Np, MR, TL.KQ, &h[TL.oPq], &h[TL.oPq + MR * TL.KQ],
                     tp.bf);
    tc_pack_operator(c->hVq.data(), Nq, Np, 1, Nq, MRQ, TL.KV, &h[TL.oVq],
                     &h[TL.oVq + MRQ * TL.KV], tp.bf);
    uint16_t *dops = nullptr;
    if ((s = upload(&c->geo_tc, geo.data(), geo.size(), "bbw_create: geometry")) != BBW_OK ||
        (s = upload(&dops, h.data(), h.size(), "bbw_create: tensor-core operators")) != BBW_OK ||
        (s = upload<int>(&c->err, nullptr, 1, "bbw_create: status")) != BBW_OK) {
      c->ops_tc = dops;
      release(c);
      return s;
    }
    c->ops_tc = dops;
    tp.geo = c->geo_tc, tp.c2q = c->c2q, tp.nbr = c->nbr, tp.tables = c->tables;
    tp.ops = c->ops_tc, tp.err = c->err, tp.time = c->d_time;
    if ((s = tc_prepare(tp)) != BBW_OK) {
      release(c);
      return s;
    }
  }
  *out = c;
  return BBW_OK;
}

extern "C" bbw_status bbw_check(bbw_ctx *c) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return set_error(BBW_ERR_ARG, "bbw_check: ctx is NULL");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_check");
  if (!c->err) return BBW_OK;
  int h = 0;
  e = cudaMemcpy(&h, c->err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_check");
  return h ? set_error(BBW_ERR_TIMEOUT, "a bounded device wait gave up; state is invalid")
           : BBW_OK;
}

extern "C" bbw_status bbw_destroy(bbw_ctx *c) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return BBW_OK;
  cudaStreamSynchronize(c->stream);
  release(c);
  return BBW_OK;
}

static bbw_status copy_state(bbw_ctx *c, float *dev, const float *src, float *dst) {
  if (!c) return set_error(BBW_ERR_ARG, "bbw: ctx is NULL");
  const size_t bytes = (size_t)c->S * c->K * 4 * c->Np * sizeof(float);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw: sync");
  if (src) e = cudaMemcpy(dev, src, bytes, cudaMemcpyHostToDevice);
  else e = cudaMemcpy(dst, dev, bytes, cudaMemcpyDeviceToHost);
  return set_cuda_error(e, "bbw: state copy");
}

extern "C" bbw_status bbw_set_state(bbw_ctx *c, const float *Q) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !Q) return set_error(BBW_ERR_ARG, "bbw_set_state: NULL");
  return copy_state(c, c->Q[c->cur], Q, nullptr);
}
extern "C" bbw_status bbw_get_state(bbw_ctx *c, float *Q) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !Q) return set_error(BBW_ERR_ARG, "bbw_get_state: NULL");
  return copy_state(c, c->Q[c->cur], nullptr, Q);
}
extern "C" bbw_status bbw_set_residual(bbw_ctx *c, const float *r) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !r) return set_error(BBW_ERR_ARG, "bbw_set_residual: NULL");
  return copy_state(c, c->res, r, nullptr);
}
extern "C" bbw_status bbw_get_residual(bbw_ctx *c, float *r) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !r) return set_error(BBW_ERR_ARG, "bbw_get_residual: NULL");
  return copy_state(c, c->res, nullptr, r);
}

static void drop_graphs(bbw_ctx *c) {
  for (int i = 0; i < 2; ++i) {
    if (c->step_graph[i]) cudaGraphExecDestroy(c->step_graph[i]);
    c->step_graph[i] = nullptr;
  }
}

extern "C" bbw_status bbw_stage_ex(bbw_ctx *c, float fa, float fb, float fdt, float cstage) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return set_error(BBW_ERR_ARG, "bbw_stage: ctx is NULL");
  bbw_status s;
  if (c->gs) {
    const GemmInputs in = {c->vgeo, c->fgeo, c->c2q, c->nbr, c->tables, c->plan.pat_off};
    s = gemm_stage_launch(*c->gs, in, c->Q[c->cur], c->Q[c->cur ^ 1], c->res, fa, fb, fdt,
                          c->stream);
  } else {
    s = c->precision != BBW_PREC_FP32
            ? tc_launch(c->tc, c->Q[c->cur], c->Q[c->cur ^ 1], c->res, fa, fb, fdt, cstage,
                        c->stream)
            : fused_launch(c->plan, c->Q[c->cur], c->Q[c->cur ^ 1], c->res, fa, fb, fdt, cstage,
                           c->stream);
  }
  if (s == BBW_OK) c->cur ^= 1;
  return s;
}

extern "C" bbw_status bbw_stage(bbw_ctx *c, float fa, float fb, float fdt) {
  DeviceGuard dg(c ? c->device : -1);
  return bbw_stage_ex(c, fa, fb, fdt, 0.f);
}

// one LSRK45 step: five fused stages at times t + rk4c[s] dt, then the
// receivers and the clock
static bbw_status one_step(bbw_ctx *c, float dt) {
  bbw_status s = BBW_OK;
  for (int i = 0; i < 5 && s == BBW_OK; ++i)
    s = bbw_stage_ex(c, (float)kRK4A[i], (float)kRK4B[i], dt,
                     c->src_stage_times ? (float)kRK4C[i] : 0.f);
  if (s != BBW_OK) return s;
  return record_and_advance(c->N, c->K, c->S, c->Q[c->cur], c->R, c->rec_elem, c->rec_w,
                            c->traces, c->max_steps, c->d_time, c->d_step, dt, c->stream);
}

// one LSRK45 step launched stage by stage (no graph), as one_step, storing
// each stage's pre-c^2 cubature values at vq + i * vqn (the adjoint tape)
bbw_status step_storing_cubature(bbw_ctx *c, float dt, float *vq, size_t vqn) {
  float *keep_f = c->plan.vq_out, *keep_t = c->tc.vq_out;
  bbw_status s = BBW_OK;
  for (int i = 0; i < 5 && s == BBW_OK; ++i) {
    c->plan.vq_out = c->tc.vq_out = vq + (size_t)i * vqn;
    s = bbw_stage_ex(c, (float)kRK4A[i], (float)kRK4B[i], dt,
                     c->src_stage_times ? (float)kRK4C[i] : 0.f);
  }
  c->plan.vq_out = keep_f, c->tc.vq_out = keep_t;
  if (s != BBW_OK) return s;
  return record_and_advance(c->N, c->K, c->S, c->Q[c->cur], c->R, c->rec_elem, c->rec_w,
                            c->traces, c->max_steps, c->d_time, c->d_step, dt, c->stream);
}

extern "C" bbw_status bbw_steps(bbw_ctx *c, float dt, int nsteps) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || nsteps < 0) return set_error(BBW_ERR_ARG, "bbw_steps: bad argument");
  uint32_t bits;
  std::memcpy(&bits, &dt, 4);
  for (int step = 0; step < nsteps; ++step) {
    const int par = c->cur;
    if (!c->step_graph[par] || c->graph_dt_bits[par] != bits) {
      if (c->step_graph[par]) cudaGraphExecDestroy(c->step_graph[par]);
      c->step_graph[par] = nullptr;
      cudaGraph_t g;
      cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return set_cuda_error(e, "bbw_steps: capture");
      bbw_status s = one_step(c, dt);
      e = cudaStreamEndCapture(c->stream, &g);
      c->cur = par;  // capture recorded the launches without running them
      if (s != BBW_OK) return s;
      if (e != cudaSuccess) return set_cuda_error(e, "bbw_steps: end capture");
      e = cudaGraphInstantiate(&c->step_graph[par], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return set_cuda_error(e, "bbw_steps: instantiate");
      c->graph_dt_bits[par] = bits;
    }
    cudaError_t e = cudaGraphLaunch(c->step_graph[par], c->stream);
    if (e != cudaSuccess) return set_cuda_error(e, "bbw_steps: launch");
    c->cur ^= 1;  // five stages swap the buffers an odd number of times
  }
  return BBW_OK;
}

// plan of the fused stage with W warps, E-element tiles and the requested
// placement; the packed operators are uploaded to *ops_buf (owned by the
// caller)
static bbw_status make_variant(bbw_ctx *c, int W, int E, int want_ops, int want_pipe,
                               FusedPlan &p, float **ops_buf) {
  FusedOps fo;
  pack_fused_ops(c->N, c->Nq, fused_groups(W, E), c->variant == BBW_BB, c->hD[0].data(), c->hD[1].data(),
                 c->hD[2].data(), c->hLIFT.data(), c->hVq.data(), c->hPq.data(), fo);
  bbw_status s = upload(ops_buf, fo.ops.data(), fo.ops.size(), "fused stage: operators");
  if (s != BBW_OK) return s;
  p = c->plan;
  p.W = W, p.E = E;
  p.ops = *ops_buf, p.ops_floats = (int)fo.ops.size();
  p.off_lift = fo.off_lift, p.off_pq = fo.off_pq, p.off_vq = fo.off_vq;
  p.RQ = fo.RQ, p.PRQ = fo.PRQ;
  p.want_ops = want_ops, p.want_pipe = want_pipe;
  return fused_prepare(p);
}

static int config_code(const FusedPlan &p) {
  return p.W | (p.ops_smem > 0 ? 1 << 8 : 0) | (p.pipe ? 1 << 9 : 0) | (p.E == 16 ? 1 << 10 : 0);
}

extern "C" bbw_status bbw_set_config(bbw_ctx *c, int config) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return set_error(BBW_ERR_ARG, "bbw_set_config: ctx is NULL");
  const int W = config & 255;
  if ((W != 8 && W != 16) || (config >> 11) != 0)
    return set_error(BBW_ERR_ARG, "bbw_set_config: W must be 8 or 16, flags bits 8-10");
  if (c->precision != BBW_PREC_FP32) return BBW_OK;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_set_config");
  FusedPlan p;
  float *buf = nullptr;
  bbw_status s = make_variant(c, W, (config >> 10 & 1) ? 16 : 32, config >> 8 & 1, config >> 9 & 1, p,
                              &buf);
  if (s != BBW_OK) {
    cudaFree(buf);
    return s;
  }
  cudaFree(c->ops);
  c->ops = buf;
  c->plan = p;
  drop_graphs(c);
  return BBW_OK;
}

extern "C" bbw_status bbw_autotune(bbw_ctx *c, float dt, int stages, int *config) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !(dt > 0.f) || stages < 1) return set_error(BBW_ERR_ARG, "bbw_autotune: bad argument");
  if (c->precision != BBW_PREC_FP32) {  // nothing to choose for the tensor-core stage
    if (config) *config = 0;
    return BBW_OK;
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_autotune");
  const size_t n = (size_t)c->S * c->K * 4 * c->Np;
  float *q[2] = {nullptr, nullptr}, *r = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto cleanup = [&]() {
    cudaFree(q[0]), cudaFree(q[1]), cudaFree(r);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  bbw_status s;
  if ((s = upload<float>(&q[0], nullptr, n, "bbw_autotune")) != BBW_OK ||
      (s = upload<float>(&q[1], nullptr, n, "bbw_autotune")) != BBW_OK ||
      (s = upload<float>(&r, nullptr, n, "bbw_autotune")) != BBW_OK) {
    cleanup();
    return s;
  }
  cudaMemcpy(q[0], c->Q[c->cur], n * sizeof(float), cudaMemcpyDeviceToDevice);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int Ws[2] = {8, 16}, Es[2] = {32, 16};
  float best_ms = 0.f;
  int best = -1;
  for (int ei = 0; ei < 2; ++ei)
  for (int wi = 0; wi < 2; ++wi)
    for (int v = 0; v < 4; ++v) {
      FusedPlan p;
      float *buf = nullptr;
      if (make_variant(c, Ws[wi], Es[ei], v < 2 ? 1 : 0, v % 2 == 0 ? 1 : 0, p, &buf) != BBW_OK) {
        cudaFree(buf);  // does not fit
        continue;
      }
      int cur = 0;
      for (int i = 0; i < 2; ++i, cur ^= 1)  // warm-up
        fused_launch(p, q[cur], q[cur ^ 1], r, 0.f, (float)kRK4B[0], dt, 0.f, c->stream);
      cudaEventRecord(e0, c->stream);
      for (int i = 0; i < stages; ++i, cur ^= 1)
        fused_launch(p, q[cur], q[cur ^ 1], r, (float)kRK4A[i % 5], (float)kRK4B[i % 5], dt, 0.f,
                     c->stream);
      cudaEventRecord(e1, c->stream);
      e = cudaEventSynchronize(e1);
      cudaFree(buf);
      if (e != cudaSuccess) {
        cleanup();
        return set_cuda_error(e, "bbw_autotune: timing");
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (best < 0 || ms < best_ms) best = config_code(p), best_ms = ms;
    }
  cleanup();
  if (best < 0) return set_error(BBW_ERR_UNSUPPORTED, "bbw_autotune: no variant fits");
  bbw_status s2 = bbw_set_config(c, best);
  if (s2 != BBW_OK) return s2;
  if (config) *config = config_code(c->plan);
  return BBW_OK;
}

extern "C" bbw_status bbw_set_grid_limit(bbw_ctx *c, int max_ctas) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || max_ctas < 0) return set_error(BBW_ERR_ARG, "bbw_set_grid_limit: bad argument");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_set_grid_limit");
  c->plan.max_ctas = max_ctas;
  c->tc.max_ctas = max_ctas;
  drop_graphs(c);
  return BBW_OK;
}

extern "C" bbw_status bbw_set_compute_range(bbw_ctx *c, int Kc) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || Kc < 1 || Kc > c->K) return set_error(BBW_ERR_ARG, "bbw_set_compute_range: bad Kc");
  if (Kc < c->K && c->precision != BBW_PREC_FP32)
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_set_compute_range: halo elements need BBW_PREC_FP32");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_set_compute_range");
  c->plan.Kc = Kc;
  drop_graphs(c);
  return BBW_OK;
}

static bbw_status check_element_list(bbw_ctx *c, int n, const int *idx, const void *buf,
                                     const char *who) {
  if (!c || n < 0 || (n > 0 && (!idx || !buf))) return set_error(BBW_ERR_ARG, who);
  return BBW_OK;
}

extern "C" bbw_status bbw_gather_elements(bbw_ctx *c, int n, const int *idx, float *buf) {
  DeviceGuard dg(c ? c->device : -1);
  bbw_status s = check_element_list(c, n, idx, buf, "bbw_gather_elements: bad argument");
  if (s != BBW_OK) return s;
  return gather_elements(c->Np, c->K, c->S, c->Q[c->cur], n, idx, buf, c->stream);
}

extern "C" bbw_status bbw_stage_part(bbw_ctx *c, float fa, float fb, float fdt, int K0, int K1) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || K0 < 0 || K1 > c->K || K0 >= K1)
    return set_error(BBW_ERR_ARG, "bbw_stage_part: need 0 <= K0 < K1 <= K");
  if (c->precision != BBW_PREC_FP32)
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_stage_part: FP32 stage only");
  FusedPlan p = c->plan;
  p.K0 = K0, p.Kc = K1;
  return fused_launch(p, c->Q[c->cur], c->Q[c->cur ^ 1], c->res, fa, fb, fdt, 0.f, c->stream);
}

extern "C" bbw_status bbw_stage_commit(bbw_ctx *c) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return set_error(BBW_ERR_ARG, "bbw_stage_commit: ctx is NULL");
  c->cur ^= 1;
  return BBW_OK;
}

extern "C" bbw_status bbw_move_elements(bbw_ctx *c, int which, int dir, int n, const int *idx,
                                        float *buf, void *stream) {
  DeviceGuard dg(c ? c->device : -1);
  bbw_status s = check_element_list(c, n, idx, buf, "bbw_move_elements: bad argument");
  if (s != BBW_OK) return s;
  if ((which != 0 && which != 1) || (dir != 0 && dir != 1))
    return set_error(BBW_ERR_ARG, "bbw_move_elements: which and dir must be 0 or 1");
  float *Q = c->Q[c->cur ^ which];
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  return dir == 0 ? gather_elements(c->Np, c->K, c->S, Q, n, idx, buf, st)
                  : scatter_elements(c->Np, c->K, c->S, Q, n, idx, buf, st);
}

extern "C" bbw_status bbw_scatter_elements(bbw_ctx *c, int n, const int *idx, const float *buf) {
  DeviceGuard dg(c ? c->device : -1);
  bbw_status s = check_element_list(c, n, idx, buf, "bbw_scatter_elements: bad argument");
  if (s != BBW_OK) return s;
  return scatter_elements(c->Np, c->K, c->S, c->Q[c->cur], n, idx, buf, c->stream);
}

extern "C" bbw_status bbw_set_shots(bbw_ctx *c, int S) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || S < 1) return set_error(BBW_ERR_ARG, "bbw_set_shots: bad argument");
  if (c->gs && S != 1)
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_set_shots: one shot in the GEMM precision form");
  cudaStreamSynchronize(c->stream);
  const size_t n = (size_t)S * c->K * 4 * c->Np;
  if ((size_t)S * c->K * 4 * c->Np > ((size_t)1 << 40))
    return set_error(BBW_ERR_ARG, "bbw_set_shots: too large");
  float *q0 = nullptr, *q1 = nullptr, *r = nullptr;
  bbw_status s;
  if ((s = upload<float>(&q0, nullptr, n, "bbw_set_shots")) != BBW_OK ||
      (s = upload<float>(&q1, nullptr, n, "bbw_set_shots")) != BBW_OK ||
      (s = upload<float>(&r, nullptr, n, "bbw_set_shots")) != BBW_OK) {
    cudaFree(q0);
    cudaFree(q1);
    cudaFree(r);
    return s;
  }
  cudaFree(c->Q[0]);
  cudaFree(c->Q[1]);
  cudaFree(c->res);
  c->Q[0] = q0, c->Q[1] = q1, c->res = r, c->cur = 0;
  c->S = S;
  c->plan.S = S;
  c->tc.S = S;
  if (c->src_off) {  // source table is per shot: drop it
    cudaFree(c->src_off), cudaFree(c->src_elem), cudaFree(c->src_vec), cudaFree(c->src_tile);
    c->src_off = c->src_elem = c->src_tile = nullptr, c->src_vec = nullptr;
    c->plan.src_off = c->plan.src_elem = nullptr, c->plan.src_vec = nullptr;
    c->tc.src_tile = c->tc.src_elem = nullptr, c->tc.src_vec = nullptr;
  }
  if (c->traces) {
    cudaFree(c->traces);
    c->traces = nullptr;
    if (c->R > 0 &&
        (s = upload<float>(&c->traces, nullptr, (size_t)S * c->R * c->max_steps,
                           "bbw_set_shots: traces")) != BBW_OK)
      return s;
  }
  drop_graphs(c);
  return BBW_OK;
}

extern "C" bbw_status bbw_set_sources(bbw_ctx *c, int nent, const int *shot, const int *elem,
                                      const float *vec, float f0, float t_delay, float amplitude,
                                      int stage_times) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || nent < 0 || (nent > 0 && (!shot || !elem || !vec)))
    return set_error(BBW_ERR_ARG, "bbw_set_sources: bad argument");
  if (c->gs && nent > 0)
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_set_sources: no sources in the GEMM precision form");
  cudaStreamSynchronize(c->stream);
  cudaFree(c->src_off), cudaFree(c->src_elem), cudaFree(c->src_vec), cudaFree(c->src_tile);
  c->src_off = c->src_elem = c->src_tile = nullptr, c->src_vec = nullptr;
  c->plan.src_off = c->plan.src_elem = nullptr, c->plan.src_vec = nullptr;
  c->tc.src_tile = c->tc.src_elem = nullptr, c->tc.src_vec = nullptr;
  drop_graphs(c);
  if (nent == 0) return BBW_OK;
  const int Np = c->Np;
  std::vector<int> off(c->S + 1, 0), order(nent), el(nent);
  for (int j = 0; j < nent; ++j) {
    if (shot[j] < 0 || shot[j] >= c->S || elem[j] < 0 || elem[j] >= c->K)
      return set_error(BBW_ERR_ARG, "bbw_set_sources: shot or element out of range");
    off[shot[j] + 1] += 1;
  }
  for (int i = 0; i < c->S; ++i) off[i + 1] += off[i];
  // order by (shot, element); the kernel bisects a shot's entries by element
  for (int j = 0; j < nent; ++j) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return shot[a] != shot[b] ? shot[a] < shot[b] : elem[a] < elem[b];
  });
  std::vector<float> v((size_t)nent * Np);
  // the tensor-core stage's table: entries of work item (shot, 32-element
  // tile) vt are [tile[vt], tile[vt + 1]) in the sorted order
  const int ntiles = (c->K + 31) / 32;
  std::vector<int> tile((size_t)c->S * ntiles + 1, 0);
  for (int at = 0; at < nent; ++at) {
    const int j = order[at];
    el[at] = elem[j];
    std::memcpy(&v[(size_t)at * Np], vec + (size_t)j * Np, Np * sizeof(float));
    tile[(size_t)shot[j] * ntiles + elem[j] / 32 + 1] += 1;
  }
  for (size_t i = 1; i < tile.size(); ++i) tile[i] += tile[i - 1];
  bbw_status s;
  if ((s = upload(&c->src_off, off.data(), off.size(), "bbw_set_sources")) != BBW_OK ||
      (s = upload(&c->src_elem, el.data(), el.size(), "bbw_set_sources")) != BBW_OK ||
      (s = upload(&c->src_vec, v.data(), v.size(), "bbw_set_sources")) != BBW_OK ||
      (s = upload(&c->src_tile, tile.data(), tile.size(), "bbw_set_sources")) != BBW_OK)
    return s;
  c->plan.src_off = c->src_off, c->plan.src_elem = c->src_elem, c->plan.src_vec = c->src_vec;
  c->plan.f0 = f0, c->plan.tR = t_delay, c->plan.samp = amplitude;
  c->tc.src_tile = c->src_tile, c->tc.src_elem = c->src_elem, c->tc.src_vec = c->src_vec;
  c->tc.f0 = f0, c->tc.tR = t_delay, c->tc.samp = amplitude;
  c->src_stage_times = stage_times != 0;
  return BBW_OK;
}

extern "C" bbw_status bbw_set_receivers(bbw_ctx *c, int R, const int *elem, const float *w,
                                        int max_steps) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || R < 0 || max_steps < 0 || (R > 0 && (!elem || !w)))
    return set_error(BBW_ERR_ARG, "bbw_set_receivers: bad argument");
  cudaStreamSynchronize(c->stream);
  cudaFree(c->rec_elem), cudaFree(c->rec_w), cudaFree(c->traces);
  c->rec_elem = nullptr, c->rec_w = nullptr, c->traces = nullptr;
  c->R = 0, c->max_steps = 0;
  drop_graphs(c);
  if (R == 0) return BBW_OK;
  for (int r = 0; r < R; ++r)
    if (elem[r] < 0 || elem[r] >= c->K)
      return set_error(BBW_ERR_ARG, "bbw_set_receivers: element out of range");
  bbw_status s;
  if ((s = upload(&c->rec_elem, elem, (size_t)R, "bbw_set_receivers")) != BBW_OK ||
      (s = upload(&c->rec_w, w, (size_t)R * c->Np, "bbw_set_receivers")) != BBW_OK ||
      (s = upload<float>(&c->traces, nullptr, (size_t)c->S * R * std::max(max_steps, 1),
                         "bbw_set_receivers")) != BBW_OK)
    return s;
  c->R = R, c->max_steps = max_steps;
  return BBW_OK;
}

extern "C" bbw_status bbw_get_traces(bbw_ctx *c, float *out, int *nsteps) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !out) return set_error(BBW_ERR_ARG, "bbw_get_traces: bad argument");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_get_traces");
  int st = 0;
  e = cudaMemcpy(&st, c->d_step, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_cuda_error(e, "bbw_get_traces");
  if (nsteps) *nsteps = std::min(st, c->max_steps);
  if (c->R == 0) return BBW_OK;
  e = cudaMemcpy(out, c->traces, (size_t)c->S * c->R * c->max_steps * sizeof(float),
                 cudaMemcpyDeviceToHost);
  return set_cuda_error(e, "bbw_get_traces");
}

extern "C" bbw_status bbw_set_time(bbw_ctx *c, double t) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return set_error(BBW_ERR_ARG, "bbw_set_time: ctx is NULL");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_time, &t, sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->d_step, 0, sizeof(int));
  return set_cuda_error(e, "bbw_set_time");
}

extern "C" bbw_status bbw_get_time(bbw_ctx *c, double *t, int *step) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return set_error(BBW_ERR_ARG, "bbw_get_time: ctx is NULL");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess && t) e = cudaMemcpy(t, c->d_time, sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && step) e = cudaMemcpy(step, c->d_step, sizeof(int), cudaMemcpyDeviceToHost);
  return set_cuda_error(e, "bbw_get_time");
}

extern "C" bbw_status bbw_run(bbw_ctx *c, double final_time, float dt) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c || !(dt > 0.f) || final_time < 0) return set_error(BBW_ERR_ARG, "bbw_run: bad argument");
  double time = 0;
  while (time < final_time) {
    if (time + dt > final_time) dt = (float)(final_time - time);  // WaveOKL3d.cpp:2048
    bbw_status s = bbw_steps(c, dt, 1);
    if (s != BBW_OK) return s;
    time += dt;
  }
  return BBW_OK;
}

extern "C" bbw_status bbw_sync(bbw_ctx *c) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return set_error(BBW_ERR_ARG, "bbw_sync: ctx is NULL");
  return set_cuda_error(cudaStreamSynchronize(c->stream), "bbw_sync");
}

extern "C" bbw_status bbw_device_state(bbw_ctx *c, float **Q, float **res, void **stream) {
  DeviceGuard dg(c ? c->device : -1);
  if (!c) return set_error(BBW_ERR_ARG, "bbw_device_state: ctx is NULL");
  if (Q) *Q = c->Q[c->cur];
  if (res) *res = c->res;
  if (stream) *stream = (void *)c->stream;
  return BBW_OK;
}
