// Discrete-adjoint kernels of the LSRK45 WADG step (sm_100a).
//
// One forward stage maps (Q, res) -> (Q', res'):
//     res' = a res + dt A(c2) Q,     Q' = Q + b res',
// with A = W(c2) S: S the DG operator (volume + surface, rk_volume /
// rk_surface, cpp/okl/WaveKernels.okl:44-260) and W the WADG projection of
// the pressure row, Pq diag(c2/J) Vq (rk_update_WADG,
// cpp/okl/WaveKernelsWADG.okl:1760-1887; J = 1, so the velocity rows are the
// identity).  Given the adjoint state (lamQ, lamR) of (Q', res') the stage
// is reversed as
//     mu = lamR + b lamQ
//     z  = W^T mu = (Vq^T diag(c2) Pq^T mu_p, mu_u, mu_v, mu_w)
//     dL/dc2q[k][q] += dt (Pq^T mu_p)_q (Vq S(Q)_p)_q        (FP64)
//     lamQ += dt S^T z,  lamR = a mu.
// S^T z = volume^T z + surface^T z.  The volume part has the forward
// volume's form with Dr, Ds, Dt replaced by their transposes (k_adj_volume).  The surface part: with
//     sigma[k][f][i] = .5 Fscale LIFT_f^T (z_p - n_f . z_U)   (per face node)
// the pressure and velocity adjoints of each face node collect
//     p: -sigma_k + sigma_k2,   U: n_k sigma_k - n_k2 sigma_k2
// from the element's own face and the matching face node of the neighbour
// k2, and -2 sigma (p = 0 wall) or 2 n sigma (rigid wall) on the boundary.
#include <cuda_runtime.h>

#include "bbwadg.h"
#include "device_common.cuh"

namespace bbw {

constexpr int AE = 32;   // elements per CTA (lane = element)
constexpr int AW = 8;    // warps per CTA
constexpr int AS = AE + 1;  // shared row stride

// Operators come in padded layouts built once on the host (AdjOps): the
// contraction index outer and four consecutive output rows contiguous (row
// stride padded to 4), so one warp-uniform 16-byte load feeds four rows of
// the warp's register block, each applied to the element values of the 32
// lanes.  A CTA copies them into shared memory when they fit beside its
// tiles (stage != 0), else reads them from global memory (L1-cached).
__device__ __forceinline__ int pad4(int x) { return (x + 3) & ~3; }

__device__ __forceinline__ void fma4(float (&acc)[4], const float4 a, float x) {
  acc[0] = fmaf(a.x, x, acc[0]);
  acc[1] = fmaf(a.y, x, acc[1]);
  acc[2] = fmaf(a.z, x, acc[2]);
  acc[3] = fmaf(a.w, x, acc[3]);
}

// mu = lamR + b lamQ; lamR <- a mu; z <- W^T mu; grad[q][k] += dt t_q v_q with
// t = Pq^T mu_p and v = Vq S(Q)_p stored by the forward recomputation
// ([shot][Nq][K]).  Lane = element, warps own quads of rows.  The shots of a
// tile are done in turn, so every gradient entry is accumulated by one
// thread in shot order.
template <int N>
__global__ void __launch_bounds__(AE * AW) k_adj_wadg(int S, int K, int Nq, int stage,
                                                     const float *__restrict__ PqT,
                                                     const float *__restrict__ VqT,
                                                     const float *__restrict__ c2q,
                                                     const float *__restrict__ lamQ,
                                                     float *__restrict__ lamR, float a, float b,
                                                     float dt, const float *__restrict__ vq,
                                                     float *__restrict__ z,
                                                     double *__restrict__ grad) {
  constexpr int Np = NP(N), ldp = (NP(N) + 3) & ~3;
  extern __shared__ float smem[];
  const int ldq = pad4(Nq);
  const int nops = stage ? Np * ldq + Nq * ldp : 0;
  float *sMu = smem + nops;         // [Np][AS]
  float *sT = sMu + Np * AS;        // [Nq][AS]
  float *sC = sT + Nq * AS;         // [Nq][AS] c2/J
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k0 = blockIdx.x * AE, ne = min(AE, K - k0);
  const float *sPt = PqT, *sVt = VqT;  // [Np][ldq] Pq^T, [Nq][ldp] Vq^T
  if (stage) {
    for (int i = tid; i < Np * ldq / 4; i += AE * AW)
      reinterpret_cast<float4 *>(smem)[i] = __ldg(reinterpret_cast<const float4 *>(PqT) + i);
    for (int i = tid; i < Nq * ldp / 4; i += AE * AW)
      reinterpret_cast<float4 *>(smem + Np * ldq)[i] =
          __ldg(reinterpret_cast<const float4 *>(VqT) + i);
    sPt = smem, sVt = smem + Np * ldq;
  }
  for (int i = tid; i < ne * Nq; i += AE * AW) sC[(i % Nq) * AS + i / Nq] = c2q[(size_t)k0 * Nq + i];
  const int nqq = (Nq + 3) >> 2, npq = (Np + 3) >> 2;
  for (int sh = 0; sh < S; ++sh) {
    const size_t so = (size_t)sh * K * 4 * Np + (size_t)k0 * 4 * Np;
    __syncthreads();
    for (int i = tid; i < ne * 4 * Np; i += AE * AW) {
      const int e = i / (4 * Np), fn = i - e * 4 * Np;
      const float mu = lamR[so + i] + b * lamQ[so + i];
      lamR[so + i] = a * mu;
      if (fn < Np) sMu[fn * AS + e] = mu;
      else z[so + i] = mu;  // velocity rows: Pq Vq = I (J = 1)
    }
    for (int i = tid; i < (AE - ne) * Np; i += AE * AW)  // idle lanes of a partial tile
      sMu[(i % Np) * AS + ne + i / Np] = 0.f;
    __syncthreads();
    for (int qq = warp; qq < nqq; qq += AW) {  // t = Pq^T mu_p, rows 4qq..4qq+3
      float t[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 5
      for (int n = 0; n < Np; ++n)
        fma4(t, reinterpret_cast<const float4 *>(sPt + n * ldq)[qq], sMu[n * AS + lane]);
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int q = 4 * qq + r;
        if (q < Nq && lane < ne) {
          if (vq)
            grad[(size_t)q * K + k0 + lane] +=
                (double)dt * (double)t[r] * (double)vq[((size_t)sh * Nq + q) * K + k0 + lane];
          sT[q * AS + lane] = sC[q * AS + lane] * t[r];
        } else if (q < Nq) {
          sT[q * AS + lane] = 0.f;
        }
      }
    }
    __syncthreads();
    for (int nq = warp; nq < npq; nq += AW) {  // z_p = Vq^T (c2 t), rows 4nq..4nq+3
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
      for (int q = 0; q < Nq; ++q)
        fma4(acc, reinterpret_cast<const float4 *>(sVt + q * ldp)[nq], sT[q * AS + lane]);
#pragma unroll
      for (int r = 0; r < 4; ++r) {  // mu_p is dead: its rows take z_p
        const int n = 4 * nq + r;
        if (n < Np) sMu[n * AS + lane] = acc[r];
      }
    }
    __syncthreads();
    for (int i = tid; i < ne * Np; i += AE * AW) {
      const int e = i / Np, n = i - e * Np;
      z[so + (size_t)e * 4 * Np + n] = sMu[n * AS + e];
    }
  }
}

// sigma[k][m] = .5 Fscale_f sum_n LIFT[n + m Np] (z_p[n] - n_f . z_U[n]) for the
// S*K elements of all shots (geometry row k % Kg); lane = element.  The face
// combinations w_f = z_p - n_f . z_U are formed once per face, then each warp
// takes quads of one face's rows.
template <int N>
__global__ void __launch_bounds__(AE * AW) k_adj_sigma(int K, int Kg, int stage,
                                                      const float *__restrict__ fgeo,
                                                      const float *__restrict__ LTp,
                                                      const float *__restrict__ z,
                                                      float *__restrict__ sigma) {
  constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N), ldf = (NFP(N) + 3) & ~3;
  extern __shared__ float smem[];
  const int nops = stage ? 4 * Np * ldf : 0;
  float *sZ = smem + nops;          // [4Np][AS]
  float *sW = sZ + 4 * Np * AS;     // [4][Np][AS]
  float *sO = sW + 4 * Np * AS;     // [NF][AS]
  float *sG = sO + NF * AS;         // [AE][16]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k0 = blockIdx.x * AE, ne = min(AE, K - k0);
  const float *sL = LTp;  // [4][Np][ldf]: LIFT^T per face
  if (stage) {
    for (int i = tid; i < nops / 4; i += AE * AW)
      reinterpret_cast<float4 *>(smem)[i] = __ldg(reinterpret_cast<const float4 *>(LTp) + i);
    sL = smem;
  }
  for (int i = tid; i < ne * 4 * Np; i += AE * AW)
    sZ[(i % (4 * Np)) * AS + i / (4 * Np)] = z[(size_t)k0 * 4 * Np + i];
  for (int i = tid; i < ne * 16; i += AE * AW)
    sG[i] = fgeo[(size_t)((k0 + i / 16) % Kg) * 16 + i % 16];
  __syncthreads();
  const int e = lane < ne ? lane : 0;
  for (int i = warp; i < 4 * Np; i += AW) {  // w_f[n] per lane
    const int f = i / Np, n = i - f * Np;
    const float nx = sG[e * 16 + 4 * f + 1], ny = sG[e * 16 + 4 * f + 2],
                nz = sG[e * 16 + 4 * f + 3];
    sW[i * AS + lane] = lane < ne ? sZ[n * AS + lane] - (nx * sZ[(Np + n) * AS + lane] +
                                                         ny * sZ[(2 * Np + n) * AS + lane] +
                                                         nz * sZ[(3 * Np + n) * AS + lane])
                                  : 0.f;
  }
  __syncthreads();
  constexpr int nfq = (Nfp + 3) >> 2;
  for (int u = warp; u < 4 * nfq; u += AW) {
    const int f = u / nfq, jq = u - f * nfq;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    const float *L = sL + f * Np * ldf;
    const float *w = sW + f * Np * AS;
#pragma unroll 5
    for (int n = 0; n < Np; ++n)
      fma4(acc, reinterpret_cast<const float4 *>(L + n * ldf)[jq], w[n * AS + lane]);
    const float Fs = sG[e * 16 + 4 * f];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int j = 4 * jq + r;
      if (j < Nfp) sO[(f * Nfp + j) * AS + lane] = .5f * Fs * acc[r];
    }
  }
  __syncthreads();
  for (int i = tid; i < ne * NF; i += AE * AW) sigma[(size_t)k0 * NF + i] = sO[(i % NF) * AS + i / NF];
}

// Volume part of S^T z: the forward volume form (rk_volume,
// cpp/okl/WaveKernels.okl:44-153) with the transposes of Dr, Ds, Dt (padded
// layout DTp), for the S*K elements of all shots (geometry row
// k % Kg).  Lane = element; each warp takes quads of output rows with the
// four gradient / divergence sums in registers; per-output summation order
// as in the forward kernel.
template <int N>
__global__ void __launch_bounds__(AE * AW) k_adj_volume(int K, int Kg, int stage,
                                                       const float *__restrict__ vgeo,
                                                       const float *__restrict__ DTp,
                                                       const float *__restrict__ z,
                                                       float *__restrict__ vol) {
  constexpr int Np = NP(N), ldp = (NP(N) + 3) & ~3, npq = (NP(N) + 3) >> 2;
  extern __shared__ float smem[];
  const int nops = stage ? 3 * Np * ldp : 0;
  float *sX = smem + nops;            // [4Np][AS]: p, then U in the rst directions
  float *sO = sX + 4 * Np * AS;       // [4Np][AS]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k0 = blockIdx.x * AE, ne = min(AE, K - k0);
  const float *sD = DTp;  // [3][Np][ldp]: column m of operator d at (d*Np + m)*ldp
  if (stage) {
    for (int i = tid; i < nops / 4; i += AE * AW)
      reinterpret_cast<float4 *>(smem)[i] = __ldg(reinterpret_cast<const float4 *>(DTp) + i);
    sD = smem;
  }
  for (int i = tid; i < AE * 4 * Np; i += AE * AW) {
    const int e = i / (4 * Np), j = i - e * 4 * Np;
    sX[j * AS + e] = e < ne ? z[(size_t)k0 * 4 * Np + i] : 0.f;
  }
  float G[9];
  const int kg = (k0 + (lane < ne ? lane : 0)) % Kg;
#pragma unroll
  for (int c = 0; c < 9; ++c) G[c] = __ldg(vgeo + (size_t)kg * 9 + c);
  __syncthreads();
  for (int n = warp; n < Np; n += AW) {  // u, v, w -> contravariant components, in place
    const float un = sX[(Np + n) * AS + lane], vn = sX[(2 * Np + n) * AS + lane],
                wn = sX[(3 * Np + n) * AS + lane];
    sX[(Np + n) * AS + lane] = un * G[0] + vn * G[1] + wn * G[2];
    sX[(2 * Np + n) * AS + lane] = un * G[3] + vn * G[4] + wn * G[5];
    sX[(3 * Np + n) * AS + lane] = un * G[6] + vn * G[7] + wn * G[8];
  }
  __syncthreads();
  for (int nq = warp; nq < npq; nq += AW) {
    float dr[4] = {0.f, 0.f, 0.f, 0.f}, ds[4] = {0.f, 0.f, 0.f, 0.f};
    float dt[4] = {0.f, 0.f, 0.f, 0.f}, dv[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 5
    for (int m = 0; m < Np; ++m) {
      const float4 a = reinterpret_cast<const float4 *>(sD + m * ldp)[nq];
      const float4 b = reinterpret_cast<const float4 *>(sD + (Np + m) * ldp)[nq];
      const float4 c = reinterpret_cast<const float4 *>(sD + (2 * Np + m) * ldp)[nq];
      const float p = sX[m * AS + lane], ur = sX[(Np + m) * AS + lane],
                  us = sX[(2 * Np + m) * AS + lane], ut = sX[(3 * Np + m) * AS + lane];
      fma4(dr, a, p);
      fma4(ds, b, p);
      fma4(dt, c, p);
      fma4(dv, a, ur);
      fma4(dv, b, us);
      fma4(dv, c, ut);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int n = 4 * nq + r;
      if (n >= Np) continue;
      sO[n * AS + lane] = -dv[r];
      sO[(Np + n) * AS + lane] = -(G[0] * dr[r] + G[3] * ds[r] + G[6] * dt[r]);
      sO[(2 * Np + n) * AS + lane] = -(G[1] * dr[r] + G[4] * ds[r] + G[7] * dt[r]);
      sO[(3 * Np + n) * AS + lane] = -(G[2] * dr[r] + G[5] * ds[r] + G[8] * dt[r]);
    }
  }
  __syncthreads();
  for (int i = tid; i < ne * 4 * Np; i += AE * AW) {
    const int e = i / (4 * Np), j = i - e * 4 * Np;
    vol[(size_t)k0 * 4 * Np + i] = sO[j * AS + e];
  }
}

// lamQ[k][.][n] += dt (vol[k][.][n] + surface adjoint at node n)
template <int N>
__global__ void __launch_bounds__(256) k_adj_gather(int K, int Kg, int bc, float dt,
                                                    const float *__restrict__ fgeo,
                                                    const int *__restrict__ fidx,
                                                    const int *__restrict__ mapP,
                                                    const float *__restrict__ sigma,
                                                    const float *__restrict__ vol,
                                                    float *__restrict__ lamQ) {
  constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)K * Np) return;
  const int k = (int)(i / Np), n = (int)(i - (long long)k * Np);
  const int kg = k % Kg;                    // mesh row (shots share the mesh)
  const size_t sbase = (size_t)(k - kg) * NF;  // sigma offset of the shot
  float dp = 0.f, du = 0.f, dv = 0.f, dw = 0.f;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const int fi = __ldg(fidx + f * Np + n);
    if (fi < 0) continue;
    const int m = f * Nfp + fi;
    const float s = sigma[(size_t)k * NF + m];
    const float *fg = fgeo + (size_t)kg * 16 + 4 * f;
    const float nx = fg[1], ny = fg[2], nz = fg[3];
    const int code = __ldg(mapP + (size_t)kg * NF + m);
    if (code < 0) {
      if (bc == BBW_BC_PRESSURE_RELEASE) {
        dp -= 2.f * s;
      } else {
        du += 2.f * nx * s, dv += 2.f * ny * s, dw += 2.f * nz * s;
      }
    } else {
      const int k2 = code / NF, f2 = (code - k2 * NF) / Nfp;
      const float s2 = sigma[sbase + code];
      const float *g2 = fgeo + (size_t)k2 * 16 + 4 * f2;
      dp += s2 - s;
      du += nx * s - g2[1] * s2;
      dv += ny * s - g2[2] * s2;
      dw += nz * s - g2[3] * s2;
    }
  }
  const size_t id = (size_t)k * 4 * Np + n;
  lamQ[id] += dt * (vol[id] + dp);
  lamQ[id + Np] += dt * (vol[id + Np] + du);
  lamQ[id + 2 * Np] += dt * (vol[id + 2 * Np] + dv);
  lamQ[id + 3 * Np] += dt * (vol[id + 3 * Np] + dw);
}

// trace[s][r][n] = w_r . Q_p(elem_r) after step n  =>  lamQ_p(elem_r) += g w_r.
// One warp per shot, receivers in order (deterministic when receivers share
// an element).
__global__ void k_adj_receivers(int S, int K, int Np, int R, const int *__restrict__ rec_elem,
                                const float *__restrict__ rec_w, const float *__restrict__ g,
                                int nsteps, int n, float *__restrict__ lamQ) {
  const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (s >= S) return;
  for (int r = 0; r < R; ++r) {
    const float gr = g[((size_t)s * R + r) * nsteps + n];
    float *q = lamQ + ((size_t)s * K + rec_elem[r]) * 4 * Np;
    for (int j = lane; j < Np; j += 32) q[j] += gr * rec_w[(size_t)r * Np + j];
    __syncwarp();
  }
}

__global__ void k_set_double(double *p, double v) { *p = v; }

// ------------------------------------------------------------- host side
// shared memory of a launch: tiles, plus the staged operators when they fit
static size_t stage_smem(size_t tiles, size_t ops, int *stage) {
  *stage = tiles + ops <= 200 * 1024 ? 1 : 0;
  return tiles + (*stage ? ops : 0);
}

template <int N>
static bbw_status launch_adj_n(int S, int K, int Nq, const float *PqT, const float *VqT,
                               const float *c2q, const float *lamQ, float *lamR, float a, float b,
                               float dt, const float *vq, float *z, double *grad,
                               cudaStream_t st) {
  constexpr int Np = NP(N);
  const int ldq = (Nq + 3) & ~3, ldp = (Np + 3) & ~3;
  int stage = 0;
  const size_t sm = stage_smem(
      sizeof(float) * (size_t)AS * (Np + 2 * Nq),
      sizeof(float) * ((size_t)Np * ldq + (size_t)Nq * ldp), &stage);
  if (sm > 200 * 1024) return set_error(BBW_ERR_UNSUPPORTED, "adjoint WADG: Nq too large");
  bbw_status s = ensure_smem_limit(k_adj_wadg<N>, 200 * 1024, "adjoint WADG attribute");
  if (s != BBW_OK) return s;
  k_adj_wadg<N><<<(K + AE - 1) / AE, AE * AW, sm, st>>>(S, K, Nq, stage, PqT, VqT, c2q, lamQ,
                                                        lamR, a, b, dt, vq, z, grad);
  return check_launch("adjoint WADG");
}

template <int N>
static bbw_status launch_sigma_n(int S, int K, const float *fgeo, const float *LTp,
                                 const float *z, float *sigma, cudaStream_t st) {
  constexpr int Np = NP(N), NF = 4 * NFP(N), ldf = (NFP(N) + 3) & ~3;
  int stage = 0;
  const size_t sm = stage_smem(sizeof(float) * ((size_t)AS * (8 * Np + NF) + AE * 16),
                               sizeof(float) * (size_t)4 * Np * ldf, &stage);
  if (sm > 200 * 1024) return set_error(BBW_ERR_UNSUPPORTED, "adjoint lift: N too large");
  bbw_status s = ensure_smem_limit(k_adj_sigma<N>, 200 * 1024, "adjoint lift attribute");
  if (s != BBW_OK) return s;
  k_adj_sigma<N><<<(S * K + AE - 1) / AE, AE * AW, sm, st>>>(S * K, K, stage, fgeo, LTp, z,
                                                               sigma);
  return check_launch("adjoint lift");
}

template <int N>
static bbw_status launch_volume_n(int S, int K, const float *vgeo, const float *DTp,
                                  const float *z, float *vol, cudaStream_t st) {
  constexpr int Np = NP(N), ldp = (NP(N) + 3) & ~3;
  int stage = 0;
  const size_t sm = stage_smem(sizeof(float) * (size_t)8 * Np * AS,
                               sizeof(float) * (size_t)3 * Np * ldp, &stage);
  if (sm > 200 * 1024) return set_error(BBW_ERR_UNSUPPORTED, "adjoint volume: N too large");
  bbw_status s = ensure_smem_limit(k_adj_volume<N>, 200 * 1024, "adjoint volume attribute");
  if (s != BBW_OK) return s;
  k_adj_volume<N><<<(S * K + AE - 1) / AE, AE * AW, sm, st>>>(S * K, K, stage, vgeo, DTp, z, vol);
  return check_launch("adjoint volume");
}

template <int N>
static bbw_status launch_gather_n(int S, int K, int bc, float dt, const float *fgeo,
                                  const int *fidx, const int *mapP, const float *sigma,
                                  const float *vol, float *lamQ, cudaStream_t st) {
  const long long n = (long long)S * K * NP(N);
  k_adj_gather<N><<<(int)((n + 255) / 256), 256, 0, st>>>(S * K, K, bc, dt, fgeo, fidx, mapP,
                                                           sigma, vol, lamQ);
  return check_launch("adjoint face gather");
}

#define BBW_N_SWITCH(CALL)                    \
  switch (N) {                                \
    case 1: return CALL(1);                   \
    case 2: return CALL(2);                   \
    case 3: return CALL(3);                   \
    case 4: return CALL(4);                   \
    case 5: return CALL(5);                   \
    case 6: return CALL(6);                   \
    case 7: return CALL(7);                   \
    case 8: return CALL(8);                   \
  }                                           \
  return set_error(BBW_ERR_UNSUPPORTED, "adjoint: N out of range");

bbw_status adj_wadg(int N, int S, int K, int Nq, const float *PqT, const float *VqT, const float *c2q,
                    const float *lamQ, float *lamR, float a, float b, float dt, const float *vq,
                    float *z, double *grad, cudaStream_t st) {
#define CALL(n) launch_adj_n<n>(S, K, Nq, PqT, VqT, c2q, lamQ, lamR, a, b, dt, vq, z, grad, st)
  BBW_N_SWITCH(CALL)
#undef CALL
}

bbw_status adj_sigma(int N, int S, int K, const float *fgeo, const float *LTp, const float *z,
                     float *sigma, cudaStream_t st) {
#define CALL(n) launch_sigma_n<n>(S, K, fgeo, LTp, z, sigma, st)
  BBW_N_SWITCH(CALL)
#undef CALL
}

bbw_status adj_volume(int N, int S, int K, const float *vgeo, const float *DTp, const float *z,
                      float *vol, cudaStream_t st) {
#define CALL(n) launch_volume_n<n>(S, K, vgeo, DTp, z, vol, st)
  BBW_N_SWITCH(CALL)
#undef CALL
}

bbw_status adj_gather(int N, int S, int K, int bc, float dt, const float *fgeo, const int *fidx,
                      const int *mapP, const float *sigma, const float *vol, float *lamQ,
                      cudaStream_t st) {
#define CALL(n) launch_gather_n<n>(S, K, bc, dt, fgeo, fidx, mapP, sigma, vol, lamQ, st)
  BBW_N_SWITCH(CALL)
#undef CALL
}

bbw_status adj_receivers(int S, int K, int Np, int R, const int *rec_elem, const float *rec_w,
                         const float *g, int nsteps, int n, float *lamQ, cudaStream_t st) {
  if (R <= 0) return BBW_OK;
  const int wpb = 4;
  k_adj_receivers<<<(S + wpb - 1) / wpb, 32 * wpb, 0, st>>>(S, K, Np, R, rec_elem, rec_w, g,
                                                            nsteps, n, lamQ);
  return check_launch("adjoint receivers");
}

bbw_status set_device_double(double *p, double v, cudaStream_t st) {
  k_set_double<<<1, 1, 0, st>>>(p, v);
  return check_launch("device clock");
}

}  // namespace bbw
