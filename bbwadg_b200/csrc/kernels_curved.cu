// Kernel-level replacements of the reference's curvilinear WADG kernels
// (sm_100a): the skew-symmetric volume and surface kernels of the curved
// elements and the J-weighted volume and surface kernels of the planar ones.
//
// Each kernel keeps its OKL counterpart's argument list, array layouts and
// per-output summation order, so results agree with the reference to FP32
// rounding.  A CTA handles EB elements of the kernel's element list (thread
// = element x point); element data and the per-point intermediates live in
// shared memory, operators are read through the read-only data cache, and
// the per-point geometric factors ([K][9][Nq], [K][4][4][Nfq]) are read with
// consecutive threads on consecutive points.
#include <cuda_runtime.h>

#include <algorithm>

#include "bbwadg.h"
#include "curved.h"
#include "device_common.cuh"

namespace bbw {

constexpr int kCurvedThreads = 256;
constexpr size_t kCurvedSmemMax = 200 * 1024;

// elements per CTA: enough threads for the widest phase, shared memory bounded
inline int curved_eb(int width, size_t smem_per_elem) {
  int eb = std::max(1, kCurvedThreads / std::max(width, 1));
  while (eb > 1 && eb * smem_per_elem > 48 * 1024) --eb;
  return eb;
}

// ----------------------------------------------- rk_volume_WADG_skew_combine
// cpp/okl/WaveKernelsWADG.okl:514-682
template <int N>
__global__ void __launch_bounds__(kCurvedThreads) k_volume_skew(
    int K, const int *__restrict__ Klist, int Nq, int EB, const float *__restrict__ vgeoq,
    const float *__restrict__ Jq, const float *__restrict__ Vq, const float *__restrict__ Vrq,
    const float *__restrict__ Vsq, const float *__restrict__ Vtq, const float *__restrict__ Pq,
    const float *__restrict__ Prq, const float *__restrict__ Psq, const float *__restrict__ Ptq,
    const float *__restrict__ Q, float *__restrict__ rhsQ) {
  constexpr int Np = NP(N);
  extern __shared__ float smem[];
  const int per = 4 * Np + 6 * Nq;
  const int k0 = blockIdx.x * EB;
  const int ne = min(EB, K - k0);
  for (int i = threadIdx.x; i < ne * 4 * Np; i += blockDim.x) {
    const int e = i / (4 * Np), j = i % (4 * Np);
    smem[e * per + j] = Q[(size_t)Klist[k0 + e] * 4 * Np + j];
  }
  __syncthreads();
  // interpolate u, v, w and the reference gradient of p to the cubature
  for (int i = threadIdx.x; i < ne * Nq; i += blockDim.x) {
    const int e = i / Nq, n = i % Nq, k = Klist[k0 + e];
    const float *sq = smem + e * per;
    float dpdr = 0.f, dpds = 0.f, dpdt = 0.f, uq = 0.f, vq = 0.f, wq = 0.f;
    for (int m = 0; m < Np; ++m) {
      const float pm = sq[m], um = sq[Np + m], vm = sq[2 * Np + m], wm = sq[3 * Np + m];
      const float V = __ldg(Vq + n + m * Nq);
      uq += V * um;
      vq += V * vm;
      wq += V * wm;
      dpdr += __ldg(Vrq + n + m * Nq) * pm;
      dpds += __ldg(Vsq + n + m * Nq) * pm;
      dpdt += __ldg(Vtq + n + m * Nq) * pm;
    }
    const float *g = vgeoq + (size_t)k * 9 * Nq + n;
    const float rx = g[0], sx = g[Nq], tx = g[2 * Nq], ry = g[3 * Nq], sy = g[4 * Nq],
                ty = g[5 * Nq], rz = g[6 * Nq], sz = g[7 * Nq], tz = g[8 * Nq];
    const float J = Jq[n + (size_t)k * Nq];
    float *t = smem + e * per + 4 * Np;
    t[n] = (rx * dpdr + sx * dpds + tx * dpdt) * J;
    t[Nq + n] = (ry * dpdr + sy * dpds + ty * dpdt) * J;
    t[2 * Nq + n] = (rz * dpdr + sz * dpds + tz * dpdt) * J;
    t[3 * Nq + n] = -((uq * rx + vq * ry + wq * rz) * J);
    t[4 * Nq + n] = -((uq * sx + vq * sy + wq * sz) * J);
    t[5 * Nq + n] = -((uq * tx + vq * ty + wq * tz) * J);
  }
  __syncthreads();
  // project: grad p with Pq, div U weakly with Prq / Psq / Ptq
  for (int i = threadIdx.x; i < ne * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = Klist[k0 + e];
    const float *t = smem + e * per + 4 * Np;
    float divU = 0.f, dpdx = 0.f, dpdy = 0.f, dpdz = 0.f;
    for (int m = 0; m < Nq; ++m) {
      const float P = __ldg(Pq + n + m * Np);
      dpdx += P * t[m];
      dpdy += P * t[Nq + m];
      dpdz += P * t[2 * Nq + m];
      divU += __ldg(Prq + n + m * Np) * t[3 * Nq + m];
      divU += __ldg(Psq + n + m * Np) * t[4 * Nq + m];
      divU += __ldg(Ptq + n + m * Np) * t[5 * Nq + m];
    }
    const size_t id = n + (size_t)k * 4 * Np;
    rhsQ[id] = -divU;
    rhsQ[id + Np] = -dpdx;
    rhsQ[id + 2 * Np] = -dpdy;
    rhsQ[id + 3 * Np] = -dpdz;
  }
}

// ---------------------------------------------- rk_surface_WADG_skew_combine
// cpp/okl/WaveKernelsWADG.okl:3024-3195
template <int N>
__global__ void __launch_bounds__(kCurvedThreads) k_surface_skew(
    int K, const int *__restrict__ Klist, int Nfq, int EB, const float *__restrict__ fgeoq,
    const float *__restrict__ VfqFace, const float *__restrict__ Pfq,
    const int *__restrict__ Fmask, const int *__restrict__ vmapP, const float *__restrict__ Q,
    float *__restrict__ rhsQ) {
  constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N);
  extern __shared__ float smem[];
  const int per = 7 * NF + 16 * Nfq;
  const int k0 = blockIdx.x * EB;
  const int ne = min(EB, K - k0);
  // jumps and averages at the face nodes; on the boundary dp = -2 pM, du = 0
  // and the "average" is the interior value
  for (int i = threadIdx.x; i < ne * NF; i += blockDim.x) {
    const int e = i / NF, m = i % NF, k = Klist[k0 + e];
    const int idM = Fmask[m] + k * Np * 4, idP = vmapP[m + (size_t)k * NF];
    const bool bnd = idM == idP;
    const float pM = Q[idM], uM = Q[idM + Np], vM = Q[idM + 2 * Np], wM = Q[idM + 3 * Np];
    const float pP = Q[idP], uP = Q[idP + Np], vP = Q[idP + 2 * Np], wP = Q[idP + 3 * Np];
    float *s = smem + e * per;
    s[m] = bnd ? -2.f * pM : pP - pM;
    s[NF + m] = bnd ? 0.f : uP - uM;
    s[2 * NF + m] = bnd ? 0.f : vP - vM;
    s[3 * NF + m] = bnd ? 0.f : wP - wM;
    s[4 * NF + m] = bnd ? uM : .5f * (uP + uM);
    s[5 * NF + m] = bnd ? vM : .5f * (vP + vM);
    s[6 * NF + m] = bnd ? wP : .5f * (wP + wM);
  }
  __syncthreads();
  // interpolate to the face cubature and form the fluxes
  for (int i = threadIdx.x; i < ne * 4 * Nfq; i += blockDim.x) {
    const int e = i / (4 * Nfq), fq = i % (4 * Nfq), f = fq / Nfq, n = fq % Nfq;
    const int k = Klist[k0 + e];
    const float *s = smem + e * per + f * Nfp;
    float dp = 0.f, du = 0.f, dv = 0.f, dw = 0.f, au = 0.f, av = 0.f, aw = 0.f;
    for (int j = 0; j < Nfp; ++j) {
      const float V = __ldg(VfqFace + n + j * Nfq);
      dp += V * s[j];
      du += V * s[NF + j];
      dv += V * s[2 * NF + j];
      dw += V * s[3 * NF + j];
      au += V * s[4 * NF + j];
      av += V * s[5 * NF + j];
      aw += V * s[6 * NF + j];
    }
    const float *g = fgeoq + ((size_t)k * 4 + f) * 4 * Nfq + n;
    const float nx = g[0], ny = g[Nfq], nz = g[2 * Nfq], sJ = g[3 * Nfq];
    const float Unjump = du * nx + dv * ny + dw * nz;
    const float Unavg = au * nx + av * ny + aw * nz;
    const float pflux = -(Unavg - .5f * dp) * sJ;
    const float Uflux = -.5f * (dp - Unjump) * sJ;
    float *fl = smem + e * per + 7 * NF;
    fl[fq] = pflux;
    fl[4 * Nfq + fq] = Uflux * nx;
    fl[8 * Nfq + fq] = Uflux * ny;
    fl[12 * Nfq + fq] = Uflux * nz;
  }
  __syncthreads();
  // lift with the face-cubature projection, added to the volume rhs
  for (int i = threadIdx.x; i < ne * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = Klist[k0 + e];
    const float *fl = smem + e * per + 7 * NF;
    const size_t id = n + (size_t)k * 4 * Np;
    float rp = rhsQ[id], ru = rhsQ[id + Np], rv = rhsQ[id + 2 * Np], rw = rhsQ[id + 3 * Np];
    for (int m = 0; m < 4 * Nfq; ++m) {
      const float P = __ldg(Pfq + n + (size_t)m * Np);
      rp += P * fl[m];
      ru += P * fl[4 * Nfq + m];
      rv += P * fl[8 * Nfq + m];
      rw += P * fl[12 * Nfq + m];
    }
    rhsQ[id] = rp;
    rhsQ[id + Np] = ru;
    rhsQ[id + 2 * Np] = rv;
    rhsQ[id + 3 * Np] = rw;
  }
}

// ---------------------------------------------------------- rk_volume_planar
// cpp/okl/WaveKernelsWADG.okl:2203-2318
template <int N>
__global__ void __launch_bounds__(kCurvedThreads) k_volume_planar(
    int K, const int *__restrict__ Klist, const float *__restrict__ vgeo,
    const float *__restrict__ J, const float *__restrict__ Dr, const float *__restrict__ Ds,
    const float *__restrict__ Dt, const float *__restrict__ Q, float *__restrict__ rhsQ) {
  constexpr int Np = NP(N), EB = VOL_EB(N) > 8 ? 8 : VOL_EB(N);
  __shared__ float sp[EB][Np], sUr[EB][Np], sUs[EB][Np], sUt[EB][Np], sG[EB][9];
  const int k0 = blockIdx.x * EB;
  for (int i = threadIdx.x; i < EB * 9; i += blockDim.x) {
    const int e = i / 9;
    if (k0 + e < K) sG[e][i % 9] = vgeo[(size_t)Klist[k0 + e] * 9 + i % 9];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np;
    if (k0 + e >= K) continue;
    const size_t id = n + (size_t)Klist[k0 + e] * Np * 4;
    sp[e][n] = Q[id];
    const float un = Q[id + Np], vn = Q[id + 2 * Np], wn = Q[id + 3 * Np];
    sUr[e][n] = un * sG[e][0] + vn * sG[e][1] + wn * sG[e][2];
    sUs[e][n] = un * sG[e][3] + vn * sG[e][4] + wn * sG[e][5];
    sUt[e][n] = un * sG[e][6] + vn * sG[e][7] + wn * sG[e][8];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np;
    if (k0 + e >= K) continue;
    const int k = Klist[k0 + e];
    float dpdr = 0, dpds = 0, dpdt = 0, divU = 0;
#pragma unroll 8
    for (int m = 0; m < Np; ++m) {
      const float Drm = __ldg(Dr + n + m * Np), Dsm = __ldg(Ds + n + m * Np),
                  Dtm = __ldg(Dt + n + m * Np);
      const float pm = sp[e][m];
      dpdr += Drm * pm;
      dpds += Dsm * pm;
      dpdt += Dtm * pm;
      divU += Drm * sUr[e][m];
      divU += Dsm * sUs[e][m];
      divU += Dtm * sUt[e][m];
    }
    const float *G = sG[e];
    const float Jk = J[k];
    const size_t id = n + (size_t)k * 4 * Np;
    rhsQ[id] = -divU * Jk;
    rhsQ[id + Np] = -(G[0] * dpdr + G[3] * dpds + G[6] * dpdt) * Jk;
    rhsQ[id + 2 * Np] = -(G[1] * dpdr + G[4] * dpds + G[7] * dpdt) * Jk;
    rhsQ[id + 3 * Np] = -(G[2] * dpdr + G[5] * dpds + G[8] * dpdt) * Jk;
  }
}

// --------------------------------------------------------- rk_surface_planar
// cpp/okl/WaveKernelsWADG.okl:2320-2441 (pressure-release wall)
template <int N>
__global__ void __launch_bounds__(kCurvedThreads) k_surface_planar(
    int K, const int *__restrict__ Klist, const float *__restrict__ fgeo,
    const float *__restrict__ J, const int *__restrict__ Fmask, const int *__restrict__ vmapP,
    const float *__restrict__ LIFT, const float *__restrict__ Q, float *__restrict__ rhsQ) {
  constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N), EB = SURF_EB(N) > 8 ? 8 : SURF_EB(N);
  __shared__ float s_pflux[EB][NF], s_Uflux[EB][NF], s_nxyz[EB][12];
  const int k0 = blockIdx.x * EB;
  for (int i = threadIdx.x; i < EB * NF; i += blockDim.x) {
    const int e = i / NF, n = i % NF;
    if (k0 + e >= K) continue;
    const int k = Klist[k0 + e], f = n / Nfp;
    const float *fg = fgeo + (size_t)k * 16 + 4 * f;
    const float Fscale = fg[0] * J[k], nx = fg[1], ny = fg[2], nz = fg[3];
    if (n % Nfp == 0) s_nxyz[e][3 * f] = nx, s_nxyz[e][3 * f + 1] = ny, s_nxyz[e][3 * f + 2] = nz;
    const int idM = Fmask[n] + k * Np * 4, idP = vmapP[n + (size_t)k * NF];
    const float pM = Q[idM], uM = Q[idM + Np], vM = Q[idM + 2 * Np], wM = Q[idM + 3 * Np];
    const float pP = Q[idP], uP = Q[idP + Np], vP = Q[idP + 2 * Np], wP = Q[idP + 3 * Np];
    float pjump = pP - pM;
    float Unjump = (uP - uM) * nx + (vP - vM) * ny + (wP - wM) * nz;
    if (idM == idP) pjump = -2.f * pM, Unjump = 0.f;
    s_pflux[e][n] = .5f * (pjump - Unjump) * Fscale;
    s_Uflux[e][n] = .5f * (Unjump - pjump) * Fscale;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np;
    if (k0 + e >= K) continue;
    float v1 = 0, v2 = 0, v3 = 0, v4 = 0;
#pragma unroll 4
    for (int m = 0; m < NF; ++m) {
      const float Lnm = __ldg(LIFT + n + m * Np);
      const int fm = m / Nfp;
      const float dfm = s_Uflux[e][m];
      v1 += Lnm * s_pflux[e][m];
      v2 += Lnm * dfm * s_nxyz[e][3 * fm];
      v3 += Lnm * dfm * s_nxyz[e][1 + 3 * fm];
      v4 += Lnm * dfm * s_nxyz[e][2 + 3 * fm];
    }
    const size_t id = n + (size_t)Klist[k0 + e] * 4 * Np;
    rhsQ[id] += v1;
    rhsQ[id + Np] += v2;
    rhsQ[id + 2 * Np] += v3;
    rhsQ[id + 3 * Np] += v4;
  }
}

// -------------------------------------------------- fused curved-element stage
// One LSRK stage of the curved elements k = k_off + i, i < KC, in one pass:
// the skew volume terms, the skew surface terms (added in the order of
// rk_surface_WADG_skew_combine), rk_update_WADG's projection with 1/J and c^2
// on p, and the LSRK update.  Reads the old state Qold (own element and
// neighbour traces), writes Qnew and res of these elements only, so it runs
// beside the planar elements' stage on the same double-buffered state.
// Geometry rows are compact: row i of vgeoq / Jq / fgeoq / Jr / c2q
// (CurvedStageArgs, curved.h).
//
// The kernel is latency-bound (dependent operator loads, barriers between
// phases), so every contraction is split into one work item per element x
// output field x point: 6 Nq items for the volume interpolation, 4 Np for
// the rhs, 4 Nr and 4 Np for the update, each a single dot product.  Per
// field the summation order is the one of the reference's kernels.
template <int N>
__global__ void __launch_bounds__(kCurvedThreads, 6) k_curved_stage(CurvedStageArgs A,
                                                                 const float *__restrict__ Qold,
                                                                 float *__restrict__ Qnew,
                                                                 float *__restrict__ res) {
  constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N);
  extern __shared__ float smem[];
  const int Nq = A.Nq, Nfq = A.Nfq, Nr = A.Nr;
  // per element: q[4Np] | raw[6Nq] | t[6Nq] | s[7NF] | fl[16Nfq] | r[4Np] | u[4Nr]
  const int o_raw = 4 * Np, o_t = o_raw + 6 * Nq, o_s = o_t + 6 * Nq, o_f = o_s + 7 * NF,
            o_r = o_f + 16 * Nfq, o_u = o_r + 4 * Np, per = o_u + 4 * Nr;
  const int i0 = blockIdx.x * A.EB;
  const int ne = min(A.EB, A.KC - i0);
  const int T = blockDim.x;
  for (int i = threadIdx.x; i < ne * 4 * Np; i += T) {
    const int e = i / (4 * Np), j = i % (4 * Np);
    smem[e * per + j] = Qold[(size_t)(A.k_off + i0 + e) * 4 * Np + j];
  }
  __syncthreads();
  // volume interpolation (rk_volume_WADG_skew_combine): c = 0..2 u v w with
  // Vq, c = 3..5 dp/dr, dp/ds, dp/dt with Vrq / Vsq / Vtq
  for (int i = threadIdx.x; i < ne * 6 * Nq; i += T) {
    const int n = i % Nq, c = (i / Nq) % 6, e = i / (6 * Nq);
    const float *op = c < 3 ? A.Vq : c == 3 ? A.Vrq : c == 4 ? A.Vsq : A.Vtq;
    const float *x = smem + e * per + (c < 3 ? (c + 1) * Np : 0);
    float acc = 0.f;
#pragma unroll
    for (int m = 0; m < Np; ++m) acc += __ldg(op + n + m * Nq) * x[m];
    smem[e * per + o_raw + c * Nq + n] = acc;
  }
  // surface: jumps and averages at the face nodes (rk_surface_WADG_skew_combine)
  for (int i = threadIdx.x; i < ne * NF; i += T) {
    const int e = i / NF, m = i % NF, k = A.k_off + i0 + e;
    const int idM = A.Fmask[m] + k * Np * 4, idP = A.vmapP[m + (size_t)k * NF];
    const bool bnd = idM == idP;
    const float pM = Qold[idM], uM = Qold[idM + Np], vM = Qold[idM + 2 * Np],
                wM = Qold[idM + 3 * Np];
    const float pP = Qold[idP], uP = Qold[idP + Np], vP = Qold[idP + 2 * Np],
                wP = Qold[idP + 3 * Np];
    float *sv = smem + e * per + o_s;
    sv[m] = bnd ? -2.f * pM : pP - pM;
    sv[NF + m] = bnd ? 0.f : uP - uM;
    sv[2 * NF + m] = bnd ? 0.f : vP - vM;
    sv[3 * NF + m] = bnd ? 0.f : wP - wM;
    sv[4 * NF + m] = bnd ? uM : .5f * (uP + uM);
    sv[5 * NF + m] = bnd ? vM : .5f * (vP + vM);
    sv[6 * NF + m] = bnd ? wP : .5f * (wP + wM);
  }
  __syncthreads();
  // geometric factors at the cubature: J grad p and -J (rst-contravariant U)
  for (int i = threadIdx.x; i < ne * Nq; i += T) {
    const int e = i / Nq, n = i % Nq, row = i0 + e;
    const float *raw = smem + e * per + o_raw;
    const float uq = raw[n], vq = raw[Nq + n], wq = raw[2 * Nq + n];
    const float dpdr = raw[3 * Nq + n], dpds = raw[4 * Nq + n], dpdt = raw[5 * Nq + n];
    const float *g = A.vgeoq + (size_t)row * 9 * Nq + n;
    const float rx = g[0], sx = g[Nq], tx = g[2 * Nq], ry = g[3 * Nq], sy = g[4 * Nq],
                ty = g[5 * Nq], rz = g[6 * Nq], sz = g[7 * Nq], tz = g[8 * Nq];
    const float J = A.Jq[n + (size_t)row * Nq];
    float *t = smem + e * per + o_t;
    t[n] = (rx * dpdr + sx * dpds + tx * dpdt) * J;
    t[Nq + n] = (ry * dpdr + sy * dpds + ty * dpdt) * J;
    t[2 * Nq + n] = (rz * dpdr + sz * dpds + tz * dpdt) * J;
    t[3 * Nq + n] = -((uq * rx + vq * ry + wq * rz) * J);
    t[4 * Nq + n] = -((uq * sx + vq * sy + wq * sz) * J);
    t[5 * Nq + n] = -((uq * tx + vq * ty + wq * tz) * J);
  }
  // face cubature: interpolate jumps / averages, upwind fluxes
  for (int i = threadIdx.x; i < ne * 4 * Nfq; i += T) {
    const int e = i / (4 * Nfq), fq = i % (4 * Nfq), f = fq / Nfq, n = fq % Nfq, row = i0 + e;
    const float *sv = smem + e * per + o_s + f * Nfp;
    float dp = 0.f, du = 0.f, dv = 0.f, dw = 0.f, au = 0.f, av = 0.f, aw = 0.f;
#pragma unroll
    for (int j = 0; j < Nfp; ++j) {
      const float V = __ldg(A.VfqFace + n + j * Nfq);
      dp += V * sv[j];
      du += V * sv[NF + j];
      dv += V * sv[2 * NF + j];
      dw += V * sv[3 * NF + j];
      au += V * sv[4 * NF + j];
      av += V * sv[5 * NF + j];
      aw += V * sv[6 * NF + j];
    }
    const float *g = A.fgeoq + ((size_t)row * 4 + f) * 4 * Nfq + n;
    const float nx = g[0], ny = g[Nfq], nz = g[2 * Nfq], sJ = g[3 * Nfq];
    const float Unjump = du * nx + dv * ny + dw * nz;
    const float Unavg = au * nx + av * ny + aw * nz;
    const float pflux = -(Unavg - .5f * dp) * sJ;
    const float Uflux = -.5f * (dp - Unjump) * sJ;
    float *fl = smem + e * per + o_f;
    fl[fq] = pflux;
    fl[4 * Nfq + fq] = Uflux * nx;
    fl[8 * Nfq + fq] = Uflux * ny;
    fl[12 * Nfq + fq] = Uflux * nz;
  }
  __syncthreads();
  // rhs of field c: volume projection (div U weakly for p, Pq grad p for
  // u, v, w), then the lifted fluxes
  for (int i = threadIdx.x; i < ne * 4 * Np; i += T) {
    const int n = i % Np, c = (i / Np) % 4, e = i / (4 * Np);
    const float *t = smem + e * per + o_t;
    const float *fl = smem + e * per + o_f + c * 4 * Nfq;
    float acc = 0.f;
    if (c == 0) {
#pragma unroll 4
      for (int m = 0; m < Nq; ++m) {
        acc += __ldg(A.Prq + n + m * Np) * t[3 * Nq + m];
        acc += __ldg(A.Psq + n + m * Np) * t[4 * Nq + m];
        acc += __ldg(A.Ptq + n + m * Np) * t[5 * Nq + m];
      }
    } else {
      const float *tc = t + (c - 1) * Nq;
#pragma unroll 8
      for (int m = 0; m < Nq; ++m) acc += __ldg(A.Pq + n + m * Np) * tc[m];
    }
    float r = -acc;
#pragma unroll 8
    for (int m = 0; m < 4 * Nfq; ++m) r += __ldg(A.Pfq + n + (size_t)m * Np) * fl[m];
    smem[e * per + o_r + c * Np + n] = r;
  }
  __syncthreads();
  // rk_update_WADG: interpolate field c, weight with 1/J (and c^2 on p)
  for (int i = threadIdx.x; i < ne * 4 * Nr; i += T) {
    const int n = i % Nr, c = (i / Nr) % 4, e = i / (4 * Nr), row = i0 + e;
    const float *r = smem + e * per + o_r + c * Np;
    float a = 0.f;
#pragma unroll
    for (int j = 0; j < Np; ++j) a += __ldg(A.Vqr + n + j * Nr) * r[j];
    const float invJ = 1.f / A.Jr[n + (size_t)row * Nr];
    a *= invJ;
    if (c == 0) a *= A.c2q[n + (size_t)row * Nr];
    smem[e * per + o_u + c * Nr + n] = a;
  }
  __syncthreads();
  // project and advance: res = fa res + dt r, Q = Q + fb res
  for (int i = threadIdx.x; i < ne * 4 * Np; i += T) {
    const int n = i % Np, c = (i / Np) % 4, e = i / (4 * Np), k = A.k_off + i0 + e;
    const float *u = smem + e * per + o_u + c * Nr;
    float acc = 0.f;
#pragma unroll 8
    for (int j = 0; j < Nr; ++j) acc += __ldg(A.Pqr + n + j * Np) * u[j];
    const size_t id = n + c * Np + (size_t)k * 4 * Np;
    const float rs = A.fa * res[id] + A.fdt * acc;
    res[id] = rs;
    Qnew[id] = smem[e * per + c * Np + n] + A.fb * rs;
  }
}

template <int N>
bbw_status launch_curved_stage(CurvedStageArgs A, const float *Qold, float *Qnew, float *res,
                               cudaStream_t st) {
  constexpr int Np = NP(N), NF = 4 * NFP(N);
  const size_t per = sizeof(float) * (8 * Np + 12 * (size_t)A.Nq + 7 * NF +
                                      16 * (size_t)A.Nfq + 4 * (size_t)A.Nr);
  // a few work items per thread in the widest phase, shared memory bounded
  const int width = std::max(std::max(A.Nq, A.Nr), std::max(4 * A.Nfq, 4 * Np));
  A.EB = curved_eb(width, per);
  if (A.EB * per > kCurvedSmemMax)
    return set_error(BBW_ERR_UNSUPPORTED, "curved stage: cubature too large for shared memory");
  bbw_status s =
      ensure_smem_limit(k_curved_stage<N>, (int)kCurvedSmemMax, "curved stage attribute");
  if (s != BBW_OK) return s;
  k_curved_stage<N><<<(A.KC + A.EB - 1) / A.EB, kCurvedThreads, A.EB * per, st>>>(A, Qold, Qnew,
                                                                                   res);
  return check_launch("curved stage");
}

// ----------------------------------------------------------------- launches
template <int N>
bbw_status launch_volume_skew(int K, const int *Klist, int Nq, const float *vgeoq,
                              const float *Jq, const float *Vq, const float *Vrq,
                              const float *Vsq, const float *Vtq, const float *Pq,
                              const float *Prq, const float *Psq, const float *Ptq,
                              const float *Q, float *rhsQ, cudaStream_t st) {
  constexpr int Np = NP(N);
  const size_t per = sizeof(float) * (4 * Np + 6 * (size_t)Nq);
  const int eb = curved_eb(std::max(Nq, Np), per);
  if (eb * per > kCurvedSmemMax)
    return set_error(BBW_ERR_UNSUPPORTED, "rk_volume_WADG_skew_combine: Nq too large");
  bbw_status s = ensure_smem_limit(k_volume_skew<N>, (int)kCurvedSmemMax,
                                   "rk_volume_WADG_skew_combine attribute");
  if (s != BBW_OK) return s;
  k_volume_skew<N><<<(K + eb - 1) / eb, kCurvedThreads, eb * per, st>>>(
      K, Klist, Nq, eb, vgeoq, Jq, Vq, Vrq, Vsq, Vtq, Pq, Prq, Psq, Ptq, Q, rhsQ);
  return check_launch("rk_volume_WADG_skew_combine");
}

template <int N>
bbw_status launch_surface_skew(int K, const int *Klist, int Nfq, const float *fgeoq,
                               const float *VfqFace, const float *Pfq, const int *Fmask,
                               const int *vmapP, const float *Q, float *rhsQ, cudaStream_t st) {
  constexpr int NF = 4 * NFP(N);
  const size_t per = sizeof(float) * (7 * NF + 16 * (size_t)Nfq);
  const int eb = curved_eb(std::max(4 * Nfq, NF), per);
  if (eb * per > kCurvedSmemMax)
    return set_error(BBW_ERR_UNSUPPORTED, "rk_surface_WADG_skew_combine: Nfq too large");
  bbw_status s = ensure_smem_limit(k_surface_skew<N>, (int)kCurvedSmemMax,
                                   "rk_surface_WADG_skew_combine attribute");
  if (s != BBW_OK) return s;
  k_surface_skew<N><<<(K + eb - 1) / eb, kCurvedThreads, eb * per, st>>>(
      K, Klist, Nfq, eb, fgeoq, VfqFace, Pfq, Fmask, vmapP, Q, rhsQ);
  return check_launch("rk_surface_WADG_skew_combine");
}

template <int N>
bbw_status launch_volume_planar(int K, const int *Klist, const float *vgeo, const float *J,
                                const float *Dr, const float *Ds, const float *Dt,
                                const float *Q, float *rhsQ, cudaStream_t st) {
  constexpr int EB = VOL_EB(N) > 8 ? 8 : VOL_EB(N);
  k_volume_planar<N><<<(K + EB - 1) / EB, kCurvedThreads, 0, st>>>(K, Klist, vgeo, J, Dr, Ds,
                                                                   Dt, Q, rhsQ);
  return check_launch("rk_volume_planar");
}

template <int N>
bbw_status launch_surface_planar(int K, const int *Klist, const float *fgeo, const float *J,
                                 const int *Fmask, const int *vmapP, const float *LIFT,
                                 const float *Q, float *rhsQ, cudaStream_t st) {
  constexpr int EB = SURF_EB(N) > 8 ? 8 : SURF_EB(N);
  k_surface_planar<N><<<(K + EB - 1) / EB, kCurvedThreads, 0, st>>>(K, Klist, fgeo, J, Fmask,
                                                                    vmapP, LIFT, Q, rhsQ);
  return check_launch("rk_surface_planar");
}

#define BBW_CURVED_DISPATCH(CALL, what)                                  \
  switch (N) {                                                           \
    case 1: return CALL(1);                                              \
    case 2: return CALL(2);                                              \
    case 3: return CALL(3);                                              \
    case 4: return CALL(4);                                              \
    case 5: return CALL(5);                                              \
    case 6: return CALL(6);                                              \
    case 7: return CALL(7);                                              \
    case 8: return CALL(8);                                              \
  }                                                                      \
  return set_error(BBW_ERR_UNSUPPORTED, what ": N out of range");

bbw_status curved_volume(int N, int K, const int *Klist, int Nq, const float *vgeoq,
                         const float *Jq, const float *Vq, const float *Vrq, const float *Vsq,
                         const float *Vtq, const float *Pq, const float *Prq, const float *Psq,
                         const float *Ptq, const float *Q, float *rhsQ, cudaStream_t st) {
  if (K == 0) return BBW_OK;
#define CALL(n) \
  launch_volume_skew<n>(K, Klist, Nq, vgeoq, Jq, Vq, Vrq, Vsq, Vtq, Pq, Prq, Psq, Ptq, Q, rhsQ, st)
  BBW_CURVED_DISPATCH(CALL, "rk_volume_WADG_skew_combine")
#undef CALL
}

bbw_status curved_surface(int N, int K, const int *Klist, int Nfq, const float *fgeoq,
                          const float *VfqFace, const float *Pfq, const int *Fmask,
                          const int *vmapP, const float *Q, float *rhsQ, cudaStream_t st) {
  if (K == 0) return BBW_OK;
#define CALL(n) launch_surface_skew<n>(K, Klist, Nfq, fgeoq, VfqFace, Pfq, Fmask, vmapP, Q, rhsQ, st)
  BBW_CURVED_DISPATCH(CALL, "rk_surface_WADG_skew_combine")
#undef CALL
}

bbw_status planar_volume(int N, int K, const int *Klist, const float *vgeo, const float *J,
                         const float *Dr, const float *Ds, const float *Dt, const float *Q,
                         float *rhsQ, cudaStream_t st) {
  if (K == 0) return BBW_OK;
#define CALL(n) launch_volume_planar<n>(K, Klist, vgeo, J, Dr, Ds, Dt, Q, rhsQ, st)
  BBW_CURVED_DISPATCH(CALL, "rk_volume_planar")
#undef CALL
}

bbw_status planar_surface(int N, int K, const int *Klist, const float *fgeo, const float *J,
                          const int *Fmask, const int *vmapP, const float *LIFT, const float *Q,
                          float *rhsQ, cudaStream_t st) {
  if (K == 0) return BBW_OK;
#define CALL(n) launch_surface_planar<n>(K, Klist, fgeo, J, Fmask, vmapP, LIFT, Q, rhsQ, st)
  BBW_CURVED_DISPATCH(CALL, "rk_surface_planar")
#undef CALL
}

bbw_status curved_stage(int N, const CurvedStageArgs &A, const float *Qold, float *Qnew,
                        float *res, cudaStream_t st) {
  if (A.KC == 0) return BBW_OK;
#define CALL(n) launch_curved_stage<n>(A, Qold, Qnew, res, st)
  BBW_CURVED_DISPATCH(CALL, "curved stage")
#undef CALL
}

}  // namespace bbw

using namespace bbw;

extern "C" bbw_status bbw_rk_volume_wadg_skew_combine(
    int N, int Nq, int K, const int *Klist, const float *vgeoq, const float *Jq, const float *Vq,
    const float *Vrq, const float *Vsq, const float *Vtq, const float *Pq, const float *Prq,
    const float *Psq, const float *Ptq, const float *Vskew, const float *Pskew, const float *Q,
    float *rhsQ, void *stream) {
  (void)Vskew, (void)Pskew;  // accepted and not read, as in the reference kernel
  if (K < 0 || Nq < NP(std::max(N, 1)) ||
      (K > 0 && (!Klist || !vgeoq || !Jq || !Vq || !Vrq || !Vsq || !Vtq || !Pq || !Prq || !Psq ||
                 !Ptq || !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_volume_wadg_skew_combine: bad argument");
  return curved_volume(N, K, Klist, Nq, vgeoq, Jq, Vq, Vrq, Vsq, Vtq, Pq, Prq, Psq, Ptq, Q, rhsQ,
                       (cudaStream_t)stream);
}

extern "C" bbw_status bbw_rk_surface_wadg_skew_combine(int N, int Nfq, int K, const int *Klist,
                                                       const float *fgeo, const float *fgeoq,
                                                       const float *VfqFace, const float *Pfq,
                                                       const int *Fmask, const int *vmapP,
                                                       const float *Q, float *rhsQ,
                                                       void *stream) {
  (void)fgeo;  // accepted and not read, as in the reference kernel
  if (K < 0 || Nfq < 1 ||
      (K > 0 && (!Klist || !fgeoq || !VfqFace || !Pfq || !Fmask || !vmapP || !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_surface_wadg_skew_combine: bad argument");
  return curved_surface(N, K, Klist, Nfq, fgeoq, VfqFace, Pfq, Fmask, vmapP, Q, rhsQ,
                        (cudaStream_t)stream);
}

extern "C" bbw_status bbw_rk_volume_planar(int N, int K, const int *Klist, const float *vgeo,
                                           const float *J, const float *Dr, const float *Ds,
                                           const float *Dt, const float *Q, float *rhsQ,
                                           void *stream) {
  if (K < 0 || (K > 0 && (!Klist || !vgeo || !J || !Dr || !Ds || !Dt || !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_volume_planar: bad argument");
  return planar_volume(N, K, Klist, vgeo, J, Dr, Ds, Dt, Q, rhsQ, (cudaStream_t)stream);
}

extern "C" bbw_status bbw_rk_surface_planar(int N, int K, const int *Klist, const float *fgeo,
                                            const float *J, const int *Fmask, const int *vmapP,
                                            const float *LIFT, const float *Q, float *rhsQ,
                                            void *stream) {
  if (K < 0 || (K > 0 && (!Klist || !fgeo || !J || !Fmask || !vmapP || !LIFT || !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_surface_planar: bad argument");
  return planar_surface(N, K, Klist, fgeo, J, Fmask, vmapP, LIFT, Q, rhsQ, (cudaStream_t)stream);
}
