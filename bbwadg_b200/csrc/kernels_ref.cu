// Kernel-level replacements of the reference's OKL kernels (sm_100a).
//
// Each kernel keeps its OKL counterpart's argument list, array layouts and
// per-output summation order, so results agree with the reference to FP32
// rounding; they are the drop-in entry points (bbw_rk_*) and the parity
// baseline of the fused stage kernel.  A CTA handles EB elements; operators
// are read through the read-only data cache, element data is staged in
// shared memory, global traffic is coalesced over the element block.
#include <cuda_runtime.h>

#include <algorithm>

#include "bbwadg.h"
#include "device_common.cuh"

namespace bbw {

// ---------------------------------------------------------------- rk_volume
// cpp/okl/WaveKernels.okl:44-153
template <int N>
__global__ void __launch_bounds__(256) k_rk_volume(int K, int Kg, const float *__restrict__ vgeo,
                                                    const float *__restrict__ Dr,
                                                    const float *__restrict__ Ds,
                                                    const float *__restrict__ Dt,
                                                    const float *__restrict__ Q,
                                                    float *__restrict__ rhsQ) {
  constexpr int Np = NP(N), EB = VOL_EB(N);
  __shared__ float sp[EB][Np], sUr[EB][Np], sUs[EB][Np], sUt[EB][Np];
  __shared__ float sG[EB][9];
  const int k0 = blockIdx.x * EB;
  for (int i = threadIdx.x; i < EB * 9; i += blockDim.x) {
    const int e = i / 9;  // geometry of element k is row k % Kg (shots share the mesh)
    if (k0 + e < K) sG[e][i % 9] = vgeo[(size_t)((k0 + e) % Kg) * 9 + i % 9];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = k0 + e;
    if (k < K) {
      const size_t id = n + (size_t)k * Np * 4;
      sp[e][n] = Q[id];
      const float un = Q[id + Np], vn = Q[id + 2 * Np], wn = Q[id + 3 * Np];
      sUr[e][n] = un * sG[e][0] + vn * sG[e][1] + wn * sG[e][2];
      sUs[e][n] = un * sG[e][3] + vn * sG[e][4] + wn * sG[e][5];
      sUt[e][n] = un * sG[e][6] + vn * sG[e][7] + wn * sG[e][8];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = k0 + e;
    if (k >= K) continue;
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
    const size_t id = n + (size_t)k * 4 * Np;
    rhsQ[id] = -divU;
    rhsQ[id + Np] = -(G[0] * dpdr + G[3] * dpds + G[6] * dpdt);
    rhsQ[id + 2 * Np] = -(G[1] * dpdr + G[4] * dpds + G[7] * dpdt);
    rhsQ[id + 3 * Np] = -(G[2] * dpdr + G[5] * dpds + G[8] * dpdt);
  }
}

// ------------------------------------------------------------- face fluxes
// cpp/okl/WaveKernels.okl:180-216 (rk_surface) / :535-569 (rk_surface_bern)
__device__ __forceinline__ void upwind_flux(const float *__restrict__ Q, int idM, int idP, int Np,
                                            float Fscale, float nx, float ny, float nz, int bc,
                                            float &pflux, float &Uflux) {
  const bool isBoundary = idM == idP;
  const float pM = Q[idM], uM = Q[idM + Np], vM = Q[idM + 2 * Np], wM = Q[idM + 3 * Np];
  const float pP = Q[idP], uP = Q[idP + Np], vP = Q[idP + 2 * Np], wP = Q[idP + 3 * Np];
  float pjump = pP - pM;
  float Unjump = (uP - uM) * nx + (vP - vM) * ny + (wP - wM) * nz;
  if (isBoundary) {
    if (bc == BBW_BC_PRESSURE_RELEASE) {
      pjump = -2.f * pM;
      Unjump = 0.f;
    } else {
      pjump = 0.f;
      Unjump = -2.f * (uM * nx + vM * ny + wM * nz);
    }
  }
  pflux = .5f * (pjump - Unjump) * Fscale;
  Uflux = .5f * (Unjump - pjump) * Fscale;
}

// --------------------------------------------------------------- rk_surface
// cpp/okl/WaveKernels.okl:156-260
template <int N>
__global__ void __launch_bounds__(256) k_rk_surface(int K, int Kg, int bc,
                                                     const float *__restrict__ fgeo,
                                                     const int *__restrict__ Fmask,
                                                     const int *__restrict__ vmapP,
                                                     const float *__restrict__ LIFT,
                                                     const float *__restrict__ Q,
                                                     float *__restrict__ rhsQ) {
  constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N), EB = SURF_EB(N);
  __shared__ float s_pflux[EB][NF], s_Uflux[EB][NF], s_nxyz[EB][12];
  const int k0 = blockIdx.x * EB;
  for (int i = threadIdx.x; i < EB * NF; i += blockDim.x) {
    const int e = i / NF, n = i % NF, k = k0 + e;
    if (k >= K) continue;
    // mesh row of element k and its shot's first element (shots share the mesh)
    const int kg = k % Kg, kb = k - kg;
    const int f = n / Nfp;
    const float *fg = fgeo + (size_t)kg * 16 + 4 * f;
    const float Fscale = fg[0], nx = fg[1], ny = fg[2], nz = fg[3];
    if (n % Nfp == 0) {
      s_nxyz[e][3 * f] = nx, s_nxyz[e][3 * f + 1] = ny, s_nxyz[e][3 * f + 2] = nz;
    }
    upwind_flux(Q, Fmask[n] + k * Np * 4, vmapP[n + (size_t)kg * NF] + kb * Np * 4, Np, Fscale, nx,
                ny, nz, bc, s_pflux[e][n], s_Uflux[e][n]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = k0 + e;
    if (k >= K) continue;
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
    const size_t id = n + (size_t)k * 4 * Np;
    rhsQ[id] += v1;
    rhsQ[id + Np] += v2;
    rhsQ[id + 2 * Np] += v3;
    rhsQ[id + 3 * Np] += v4;
  }
}

// ---------------------------------------------------------------- rk_update
// cpp/okl/WaveKernels.okl:262-313 (element-wise, vectorised)
__global__ void k_rk_update(long long n4, float fa, float fb, float fdt,
                            const float4 *__restrict__ rhsQ, float4 *__restrict__ resQ,
                            float4 *__restrict__ Q) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4;
       i += (long long)gridDim.x * blockDim.x) {
    const float4 r = rhsQ[i];
    float4 s = resQ[i], q = Q[i];
    s.x = fa * s.x + fdt * r.x;
    s.y = fa * s.y + fdt * r.y;
    s.z = fa * s.z + fdt * r.z;
    s.w = fa * s.w + fdt * r.w;
    q.x += fb * s.x;
    q.y += fb * s.y;
    q.z += fb * s.z;
    q.w += fb * s.w;
    resQ[i] = s;
    Q[i] = q;
  }
}

// ----------------------------------------------------------- rk_update_WADG
// cpp/okl/WaveKernelsWADG.okl:1760-1887
template <int N>
__global__ void __launch_bounds__(256) k_rk_update_wadg(int K, int Nq, const float *__restrict__ Vq,
                                                         const float *__restrict__ Pq,
                                                         const float *__restrict__ Jq,
                                                         const float *__restrict__ c2q, float fa,
                                                         float fb, float fdt,
                                                         const float *__restrict__ rhsQ,
                                                         float *__restrict__ resQ,
                                                         float *__restrict__ Q) {
  constexpr int Np = NP(N), EB = UPD_EB(N);
  extern __shared__ float smem[];
  float *s_r = smem;                 // [EB][4][Np]
  float *s_q = smem + EB * 4 * Np;   // [EB][4][Nq]
  const int k0 = blockIdx.x * EB;
  for (int i = threadIdx.x; i < EB * 4 * Np; i += blockDim.x) {
    const int e = i / (4 * Np);
    if (k0 + e < K) s_r[i] = rhsQ[(size_t)k0 * 4 * Np + i];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Nq; i += blockDim.x) {
    const int e = i / Nq, n = i % Nq, k = k0 + e;
    if (k >= K) continue;
    const float *r = s_r + e * 4 * Np;
    float a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (int j = 0; j < Np; ++j) {
      const float V = __ldg(Vq + n + j * Nq);
      a0 += V * r[j];
      a1 += V * r[j + Np];
      a2 += V * r[j + 2 * Np];
      a3 += V * r[j + 3 * Np];
    }
    const float c2 = c2q[n + (size_t)k * Nq];
    const float invJ = 1.f / Jq[n + (size_t)k * Nq];
    float *q = s_q + e * 4 * Nq;
    q[n] = a0 * invJ * c2;
    q[n + Nq] = a1 * invJ;
    q[n + 2 * Nq] = a2 * invJ;
    q[n + 3 * Nq] = a3 * invJ;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = k0 + e;
    if (k >= K) continue;
    const float *q = s_q + e * 4 * Nq;
    float rp = 0, ru = 0, rv = 0, rw = 0;
    for (int j = 0; j < Nq; ++j) {
      const float P = __ldg(Pq + n + j * Np);
      rp += P * q[j];
      ru += P * q[j + Nq];
      rv += P * q[j + 2 * Nq];
      rw += P * q[j + 3 * Nq];
    }
    const float rr[4] = {rp, ru, rv, rw};
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const size_t id = n + f * Np + (size_t)k * 4 * Np;
      const float res = fa * resQ[id] + fdt * rr[f];
      resQ[id] = res;
      Q[id] += fb * res;
    }
  }
}

// ----------------------------------------------------------- rk_volume_bern
// cpp/okl/WaveKernels.okl:344-474
template <int N>
__global__ void __launch_bounds__(256) k_rk_volume_bern(
    int K, const float *__restrict__ vgeo, const int4 *__restrict__ D1, const int4 *__restrict__ D2,
    const int4 *__restrict__ D3, const int4 *__restrict__ D4, const float4 *__restrict__ Dvals,
    const float *__restrict__ Q, float *__restrict__ rhsQ) {
  constexpr int Np = NP(N), EB = VOL_EB(N);
  __shared__ float sp[EB][Np], sUr[EB][Np], sUs[EB][Np], sUt[EB][Np];
  __shared__ float sG[EB][9];
  const int k0 = blockIdx.x * EB;
  for (int i = threadIdx.x; i < EB * 9; i += blockDim.x) {
    const int e = i / 9;
    if (k0 + e < K) sG[e][i % 9] = vgeo[(size_t)(k0 + e) * 9 + i % 9];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = k0 + e;
    if (k < K) {
      const size_t id = n + (size_t)k * Np * 4;
      sp[e][n] = Q[id];
      const float un = Q[id + Np], vn = Q[id + 2 * Np], wn = Q[id + 3 * Np];
      sUr[e][n] = un * sG[e][0] + vn * sG[e][1] + wn * sG[e][2];
      sUs[e][n] = un * sG[e][3] + vn * sG[e][4] + wn * sG[e][5];
      sUt[e][n] = un * sG[e][6] + vn * sG[e][7] + wn * sG[e][8];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = k0 + e;
    if (k >= K) continue;
    const float4 dv = __ldg(Dvals + n);
    const int4 a = __ldg(D1 + n), b = __ldg(D2 + n), c = __ldg(D3 + n), d = __ldg(D4 + n);
    const float *p = sp[e], *ur = sUr[e], *us = sUs[e], *ut = sUt[e];
    const float p1 = dv.x * p[a.x] + dv.y * p[b.x] + dv.z * p[c.x] + dv.w * p[d.x];
    const float p2 = dv.x * p[a.y] + dv.y * p[b.y] + dv.z * p[c.y] + dv.w * p[d.y];
    const float p3 = dv.x * p[a.z] + dv.y * p[b.z] + dv.z * p[c.z] + dv.w * p[d.z];
    const float p4 = dv.x * p[a.w] + dv.y * p[b.w] + dv.z * p[c.w] + dv.w * p[d.w];
    float dU1 = dv.x * (ur[a.y] + us[a.z] + ut[a.w]);
    dU1 += dv.y * (ur[b.y] + us[b.z] + ut[b.w]);
    dU1 += dv.z * (ur[c.y] + us[c.z] + ut[c.w]);
    dU1 += dv.w * (ur[d.y] + us[d.z] + ut[d.w]);
    float dU2 = dv.x * (ur[a.x] + us[a.x] + ut[a.x]);
    dU2 += dv.y * (ur[b.x] + us[b.x] + ut[b.x]);
    dU2 += dv.z * (ur[c.x] + us[c.x] + ut[c.x]);
    dU2 += dv.w * (ur[d.x] + us[d.x] + ut[d.x]);
    const float dpdr = .5f * (p2 - p1), dpds = .5f * (p3 - p1), dpdt = .5f * (p4 - p1);
    const float divU = .5f * (dU1 - dU2);
    const float *G = sG[e];
    const size_t id = n + (size_t)k * 4 * Np;
    rhsQ[id] = -divU;
    rhsQ[id + Np] = -(G[0] * dpdr + G[3] * dpds + G[6] * dpdt);
    rhsQ[id + 2 * Np] = -(G[1] * dpdr + G[4] * dpds + G[7] * dpdt);
    rhsQ[id + 3 * Np] = -(G[2] * dpdr + G[5] * dpds + G[8] * dpdt);
  }
}

// ---------------------------------------------------------- rk_surface_bern
// cpp/okl/WaveKernels.okl:479-647
template <int N>
__global__ void __launch_bounds__(256) k_rk_surface_bern(
    int K, int bc, const float *__restrict__ fgeo, const int *__restrict__ Fmask,
    const int *__restrict__ vmapP, int EEL_nnz, const int *__restrict__ EEL_ids,
    const float *__restrict__ EEL_vals, int L0_nnz, const int *__restrict__ L0_ids,
    const float *__restrict__ L0_vals, const float *__restrict__ Q, float *__restrict__ rhsQ) {
  constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N), EB = SURF_EB(N);
  __shared__ float s_pflux[EB][NF], s_Uflux[EB][NF], s_ptmp[EB][NF], s_Utmp[EB][NF];
  __shared__ float s_nxyz[EB][16];
  const int k0 = blockIdx.x * EB;
  for (int i = threadIdx.x; i < EB * 16; i += blockDim.x) {
    const int e = i / 16, j = i % 16, k = k0 + e;
    if (k >= K) continue;
    const int f = j / 4, c = j % 4;
    // s_nxyz[4f + {0,1,2,3}] = {nx, ny, nz, Fscale}
    s_nxyz[e][4 * f + (c == 0 ? 3 : c - 1)] = fgeo[(size_t)k * 16 + j];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * NF; i += blockDim.x) {
    const int e = i / NF, n = i % NF, k = k0 + e;
    if (k >= K) continue;
    const int f = n / Nfp;
    upwind_flux(Q, Fmask[n] + k * Np * 4, vmapP[n + (size_t)k * NF], Np, s_nxyz[e][4 * f + 3],
                s_nxyz[e][4 * f], s_nxyz[e][4 * f + 1], s_nxyz[e][4 * f + 2], bc, s_pflux[e][n],
                s_Uflux[e][n]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * NF; i += blockDim.x) {
    const int e = i / NF, n = i % NF, k = k0 + e;
    if (k >= K) continue;
    const int f = n / Nfp, nt = n % Nfp;
    float v1 = 0, v2 = 0;
    for (int j = 0; j < L0_nnz; ++j) {
      const float L = __ldg(L0_vals + nt + j * Nfp);
      const int id = __ldg(L0_ids + nt + j * Nfp) + f * Nfp;
      v1 += L * s_pflux[e][id];
      v2 += L * s_Uflux[e][id];
    }
    s_ptmp[e][n] = v1;
    s_Utmp[e][n] = v2;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < EB * Np; i += blockDim.x) {
    const int e = i / Np, n = i % Np, k = k0 + e;
    if (k >= K) continue;
    const size_t id = n + (size_t)k * 4 * Np;
    float v1 = rhsQ[id], v2 = rhsQ[id + Np], v3 = rhsQ[id + 2 * Np], v4 = rhsQ[id + 3 * Np];
    for (int j = 0; j < EEL_nnz; ++j) {
      const int col = __ldg(EEL_ids + n + j * Np);
      const float E = __ldg(EEL_vals + n + j * Np);
      const int fc = col / Nfp;
      const float Uf = s_Utmp[e][col];
      v1 += E * s_ptmp[e][col];
      v2 += E * Uf * s_nxyz[e][4 * fc];
      v3 += E * Uf * s_nxyz[e][4 * fc + 1];
      v4 += E * Uf * s_nxyz[e][4 * fc + 2];
    }
    rhsQ[id] = v1;
    rhsQ[id + Np] = v2;
    rhsQ[id + 2 * Np] = v3;
    rhsQ[id + 3 * Np] = v4;
  }
}

// ------------------------------------------------------------ host launchers

// --------------------------------------------------- rk_surface_bern_slice
// cpp/okl/WaveKernels.okl:652-939: the BB lift applied slice by slice.  After
// L0, slice 0 adds the face polynomial itself to the volume rows of its
// slice (slice_ids), each later slice reduces the previous slice's face
// polynomial by one degree with three nonzeros per node (EEL_ids / EEL_vals
// packed per slice, the reference's EEL_id_vec / EEL_val_vec) and adds it
// scaled by cEL[slice].  One CTA per element; the faces of one slice are
// applied in turn, so every accumulation into a volume row has a fixed order.
template <int N>
__global__ void __launch_bounds__(64) k_rk_surface_bern_slice(
    int K, int bc, const float *__restrict__ fgeo, const int *__restrict__ Fmask,
    const int *__restrict__ vmapP, const int4 *__restrict__ slice_ids,
    const int *__restrict__ EEL_ids, const float *__restrict__ EEL_vals, int L0_nnz,
    const int *__restrict__ L0_ids, const float *__restrict__ L0_vals,
    const float *__restrict__ cEL, const float *__restrict__ Q, float *__restrict__ rhsQ) {
  constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N);
  __shared__ float sp[2][NF], sU[2][NF], st[4][Np], sg[16], sc[N + 1];
  const int k = blockIdx.x, tid = threadIdx.x, T = blockDim.x;
  const size_t base = (size_t)k * 4 * Np;
  for (int i = tid; i < 4 * Np; i += T) st[i / Np][i % Np] = rhsQ[base + i];
  if (tid < 16) sg[tid] = fgeo[(size_t)k * 16 + tid];
  if (tid <= N) sc[tid] = cEL[tid];
  __syncthreads();
  for (int m = tid; m < NF; m += T) {
    const int f = m / Nfp;
    upwind_flux(Q, Fmask[m] + k * Np * 4, vmapP[m + (size_t)k * NF], Np, sg[4 * f],
                sg[4 * f + 1], sg[4 * f + 2], sg[4 * f + 3], bc, sp[0][m], sU[0][m]);
  }
  __syncthreads();
  for (int n = tid; n < Nfp; n += T) {  // L0 on every face
    float v1[4] = {0.f, 0.f, 0.f, 0.f}, v2[4] = {0.f, 0.f, 0.f, 0.f};
    for (int j = 0; j < L0_nnz; ++j) {
      const float L = L0_vals[n + j * Nfp];
      const int id = L0_ids[n + j * Nfp];
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        v1[f] += L * sp[0][id + f * Nfp];
        v2[f] += L * sU[0][id + f * Nfp];
      }
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) sp[1][n + f * Nfp] = v1[f], sU[1][n + f * Nfp] = v2[f];
  }
  __syncthreads();
  int off1 = 0, off2 = 0;
  for (int slice = 0; slice <= N; ++slice) {
    const int Ns = N - slice, Nps = (Ns + 1) * (Ns + 2) / 2;
    const int w = slice & 1, r = w ^ 1;
    const float cs = sc[slice];
    for (int f = 0; f < 4; ++f) {
      for (int n = tid; n < Nps; n += T) {
        const int4 v4 = slice_ids[n + off1];
        const int vol = f == 0 ? v4.x : f == 1 ? v4.y : f == 2 ? v4.z : v4.w;
        float rp, rU;
        if (slice == 0) {
          rp = sp[1][n + f * Nfp];
          rU = sU[1][n + f * Nfp];
        } else {
          const int i0 = n + off2;
          const float a = EEL_vals[i0], b = EEL_vals[i0 + Nps], c = EEL_vals[i0 + 2 * Nps];
          const int j1 = EEL_ids[i0] + f * Nfp, j2 = EEL_ids[i0 + Nps] + f * Nfp,
                    j3 = EEL_ids[i0 + 2 * Nps] + f * Nfp;
          rp = a * sp[r][j1] + b * sp[r][j2] + c * sp[r][j3];
          rU = a * sU[r][j1] + b * sU[r][j2] + c * sU[r][j3];
        }
        sp[w][n + f * Nfp] = rp;
        sU[w][n + f * Nfp] = rU;
        rp *= cs;
        rU *= cs;
        st[0][vol] += rp;
        st[1][vol] += rU * sg[4 * f + 1];
        st[2][vol] += rU * sg[4 * f + 2];
        st[3][vol] += rU * sg[4 * f + 3];
      }
      __syncthreads();
    }
    off1 += Nps;
    if (slice > 0) off2 += 3 * Nps;
  }
  for (int i = tid; i < 4 * Np; i += T) rhsQ[base + i] = st[i / Np][i % Np];
}

template <int N>
static bbw_status launch_volume(int K, int Kg, const float *vgeo, const float *Dr,
                                const float *Ds, const float *Dt, const float *Q, float *rhsQ,
                                cudaStream_t st) {
  constexpr int EB = VOL_EB(N);
  k_rk_volume<N><<<(K + EB - 1) / EB, 256, 0, st>>>(K, Kg, vgeo, Dr, Ds, Dt, Q, rhsQ);
  return check_launch("rk_volume");
}

template <int N>
static bbw_status launch_surface(int K, int Kg, int bc, const float *fgeo, const int *Fmask,
                                 const int *vmapP, const float *LIFT, const float *Q, float *rhsQ,
                                 cudaStream_t st) {
  constexpr int EB = SURF_EB(N);
  k_rk_surface<N><<<(K + EB - 1) / EB, 256, 0, st>>>(K, Kg, bc, fgeo, Fmask, vmapP, LIFT, Q,
                                                      rhsQ);
  return check_launch("rk_surface");
}

template <int N>
static bbw_status launch_wadg(int K, int Nq, const float *Vq, const float *Pq, const float *Jq,
                              const float *c2q, float fa, float fb, float fdt, const float *rhsQ,
                              float *resQ, float *Q, cudaStream_t st) {
  constexpr int Np = NP(N), EB = UPD_EB(N);
  const size_t sm = sizeof(float) * EB * 4 * (Np + Nq);
  if (sm > 200 * 1024) return set_error(BBW_ERR_UNSUPPORTED, "rk_update_WADG: Nq too large");
  bbw_status s =
      ensure_smem_limit(k_rk_update_wadg<N>, 200 * 1024, "rk_update_WADG attribute");
  if (s != BBW_OK) return s;
  k_rk_update_wadg<N><<<(K + EB - 1) / EB, 256, sm, st>>>(K, Nq, Vq, Pq, Jq, c2q, fa, fb, fdt,
                                                          rhsQ, resQ, Q);
  return check_launch("rk_update_WADG");
}

template <int N>
static bbw_status launch_volume_bern(int K, const float *vgeo, const int *D1, const int *D2,
                                     const int *D3, const int *D4, const float *Dv,
                                     const float *Q, float *rhsQ, cudaStream_t st) {
  constexpr int EB = VOL_EB(N);
  k_rk_volume_bern<N><<<(K + EB - 1) / EB, 256, 0, st>>>(
      K, vgeo, (const int4 *)D1, (const int4 *)D2, (const int4 *)D3, (const int4 *)D4,
      (const float4 *)Dv, Q, rhsQ);
  return check_launch("rk_volume_bern");
}

template <int N>
static bbw_status launch_surface_bern(int K, int bc, const float *fgeo, const int *Fmask,
                                      const int *vmapP, int EEL_nnz, const int *EEL_ids,
                                      const float *EEL_vals, int L0_nnz, const int *L0_ids,
                                      const float *L0_vals, const float *Q, float *rhsQ,
                                      cudaStream_t st) {
  constexpr int EB = SURF_EB(N);
  k_rk_surface_bern<N><<<(K + EB - 1) / EB, 256, 0, st>>>(
      K, bc, fgeo, Fmask, vmapP, EEL_nnz, EEL_ids, EEL_vals, L0_nnz, L0_ids, L0_vals, Q, rhsQ);
  return check_launch("rk_surface_bern");
}


template <int N>
static bbw_status launch_surface_bern_slice(int K, int bc, const float *fgeo, const int *Fmask,
                                            const int *vmapP, const int *slice_ids,
                                            const int *EEL_ids, const float *EEL_vals,
                                            int L0_nnz, const int *L0_ids, const float *L0_vals,
                                            const float *cEL, const float *Q, float *rhsQ,
                                            cudaStream_t st) {
  k_rk_surface_bern_slice<N><<<K, 64, 0, st>>>(K, bc, fgeo, Fmask, vmapP,
                                                (const int4 *)slice_ids, EEL_ids, EEL_vals,
                                                L0_nnz, L0_ids, L0_vals, cEL, Q, rhsQ);
  return check_launch("rk_surface_bern_slice");
}

}  // namespace bbw

using namespace bbw;

// node indices are int32, as the reference's vmapP: K * 4 * Np < 2^31
static bool too_many_nodes(int N, int K) { return (long long)K * 4 * NP(N) >= (1LL << 31); }

extern "C" bbw_status bbw_rk_volume(int N, int K, const float *vgeo, const float *Dr,
                                    const float *Ds, const float *Dt, const float *Q, float *rhsQ,
                                    void *stream) {
  if (K < 0 || (K > 0 && (!vgeo || !Dr || !Ds || !Dt || !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_volume: bad argument");
  if (too_many_nodes(N, K))
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_volume: K * 4 * Np must be below 2^31");
  if (K == 0) return BBW_OK;
  cudaStream_t st = (cudaStream_t)stream;
#define CALL(n) launch_volume<n>(K, K, vgeo, Dr, Ds, Dt, Q, rhsQ, st)
  switch (N) {
    case 1: return CALL(1);
    case 2: return CALL(2);
    case 3: return CALL(3);
    case 4: return CALL(4);
    case 5: return CALL(5);
    case 6: return CALL(6);
    case 7: return CALL(7);
    case 8: return CALL(8);
  }
#undef CALL
  return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_volume: N out of range");
}

extern "C" bbw_status bbw_rk_surface(int N, int K, int bc, const float *fgeo, const int *Fmask,
                                     const int *vmapP, const float *LIFT, const float *Q,
                                     float *rhsQ, void *stream) {
  if (K < 0 || (bc != 0 && bc != 1) ||
      (K > 0 && (!fgeo || !Fmask || !vmapP || !LIFT || !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_surface: bad argument");
  if (too_many_nodes(N, K))
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_surface: K * 4 * Np must be below 2^31");
  if (K == 0) return BBW_OK;
  cudaStream_t st = (cudaStream_t)stream;
#define CALL(n) launch_surface<n>(K, K, bc, fgeo, Fmask, vmapP, LIFT, Q, rhsQ, st)
  switch (N) {
    case 1: return CALL(1);
    case 2: return CALL(2);
    case 3: return CALL(3);
    case 4: return CALL(4);
    case 5: return CALL(5);
    case 6: return CALL(6);
    case 7: return CALL(7);
    case 8: return CALL(8);
  }
#undef CALL
  return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_surface: N out of range");
}

extern "C" bbw_status bbw_rk_update(int N, int K, float fa, float fb, float fdt,
                                    const float *rhsQ, float *resQ, float *Q, void *stream) {
  if (N < 1 || N > BBW_MAX_N) return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_update: N");
  if (K < 0 || (K > 0 && (!rhsQ || !resQ || !Q)))
    return set_error(BBW_ERR_ARG, "bbw_rk_update: bad argument");
  if (too_many_nodes(N, K))
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_update: K * 4 * Np must be below 2^31");
  if (K == 0) return BBW_OK;
  const long long n4 = (long long)K * 4 * NP(N) / 4;  // 4*Np floats per element: multiple of 4
  const int blocks = (int)std::min<long long>((n4 + 255) / 256, 148LL * 16);
  k_rk_update<<<blocks, 256, 0, (cudaStream_t)stream>>>(n4, fa, fb, fdt, (const float4 *)rhsQ,
                                                         (float4 *)resQ, (float4 *)Q);
  return check_launch("rk_update");
}

extern "C" bbw_status bbw_rk_update_wadg(int N, int K, int Nq, const float *Vq, const float *Pq,
                                         const float *Jq, const float *c2q, float fa, float fb,
                                         float fdt, const float *rhsQ, float *resQ, float *Q,
                                         void *stream) {
  if (K < 0 || Nq <= 0 || (K > 0 && (!Vq || !Pq || !Jq || !c2q || !rhsQ || !resQ || !Q)))
    return set_error(BBW_ERR_ARG, "bbw_rk_update_wadg: bad argument");
  if (too_many_nodes(N, K))
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_update_wadg: K * 4 * Np must be below 2^31");
  if (K == 0) return BBW_OK;
  cudaStream_t st = (cudaStream_t)stream;
#define CALL(n) launch_wadg<n>(K, Nq, Vq, Pq, Jq, c2q, fa, fb, fdt, rhsQ, resQ, Q, st)
  switch (N) {
    case 1: return CALL(1);
    case 2: return CALL(2);
    case 3: return CALL(3);
    case 4: return CALL(4);
    case 5: return CALL(5);
    case 6: return CALL(6);
    case 7: return CALL(7);
    case 8: return CALL(8);
  }
#undef CALL
  return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_update_wadg: N out of range");
}

extern "C" bbw_status bbw_rk_volume_bern(int N, int K, const float *vgeo, const int *D_ids1,
                                         const int *D_ids2, const int *D_ids3, const int *D_ids4,
                                         const float *Dvals4, const float *Q, float *rhsQ,
                                         void *stream) {
  if (K < 0 ||
      (K > 0 && (!vgeo || !D_ids1 || !D_ids2 || !D_ids3 || !D_ids4 || !Dvals4 || !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_volume_bern: bad argument");
  if (too_many_nodes(N, K))
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_volume_bern: K * 4 * Np must be below 2^31");
  if (K == 0) return BBW_OK;
  cudaStream_t st = (cudaStream_t)stream;
#define CALL(n) launch_volume_bern<n>(K, vgeo, D_ids1, D_ids2, D_ids3, D_ids4, Dvals4, Q, rhsQ, st)
  switch (N) {
    case 1: return CALL(1);
    case 2: return CALL(2);
    case 3: return CALL(3);
    case 4: return CALL(4);
    case 5: return CALL(5);
    case 6: return CALL(6);
    case 7: return CALL(7);
    case 8: return CALL(8);
  }
#undef CALL
  return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_volume_bern: N out of range");
}

extern "C" bbw_status bbw_rk_surface_bern(int N, int K, int bc, const float *fgeo,
                                          const int *Fmask, const int *vmapP,
                                          const int * /*slice_ids*/, int EEL_nnz,
                                          const int *EEL_ids, const float *EEL_vals, int L0_nnz,
                                          const int *L0_ids, const float *L0_vals,
                                          const float * /*cEL*/, const float *Q, float *rhsQ,
                                          void *stream) {
  if (K < 0 || (bc != 0 && bc != 1) || EEL_nnz <= 0 || L0_nnz <= 0 ||
      (K > 0 && (!fgeo || !Fmask || !vmapP || !EEL_ids || !EEL_vals || !L0_ids || !L0_vals ||
                 !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_surface_bern: bad argument");
  if (too_many_nodes(N, K))
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_surface_bern: K * 4 * Np must be below 2^31");
  if (K == 0) return BBW_OK;
  cudaStream_t st = (cudaStream_t)stream;
#define CALL(n)                                                                                \
  launch_surface_bern<n>(K, bc, fgeo, Fmask, vmapP, EEL_nnz, EEL_ids, EEL_vals, L0_nnz, L0_ids, \
                         L0_vals, Q, rhsQ, st)
  switch (N) {
    case 1: return CALL(1);
    case 2: return CALL(2);
    case 3: return CALL(3);
    case 4: return CALL(4);
    case 5: return CALL(5);
    case 6: return CALL(6);
    case 7: return CALL(7);
    case 8: return CALL(8);
  }
#undef CALL
  return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_surface_bern: N out of range");
}

extern "C" bbw_status bbw_rk_surface_bern_slice(int N, int K, int bc, const float *fgeo,
                                                const int *Fmask, const int *vmapP,
                                                const int *slice_ids, const int *EEL_ids,
                                                const float *EEL_vals, int L0_nnz,
                                                const int *L0_ids, const float *L0_vals,
                                                const float *cEL, const float *Q, float *rhsQ,
                                                void *stream) {
  if (K < 0 || (bc != 0 && bc != 1) || L0_nnz < 1 ||
      (K > 0 && (!fgeo || !Fmask || !vmapP || !slice_ids || !EEL_ids || !EEL_vals || !L0_ids ||
                 !L0_vals || !cEL || !Q || !rhsQ)))
    return set_error(BBW_ERR_ARG, "bbw_rk_surface_bern_slice: bad argument");
  if (too_many_nodes(N, K))
    return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_surface_bern_slice: K * 4 * Np must be below 2^31");
  if (K == 0) return BBW_OK;
  cudaStream_t st = (cudaStream_t)stream;
#define CALL(n)                                                                             \
  launch_surface_bern_slice<n>(K, bc, fgeo, Fmask, vmapP, slice_ids, EEL_ids, EEL_vals, L0_nnz, \
                               L0_ids, L0_vals, cEL, Q, rhsQ, st)
  switch (N) {
    case 1: return CALL(1);
    case 2: return CALL(2);
    case 3: return CALL(3);
    case 4: return CALL(4);
    case 5: return CALL(5);
    case 6: return CALL(6);
    case 7: return CALL(7);
    case 8: return CALL(8);
  }
#undef CALL
  return set_error(BBW_ERR_UNSUPPORTED, "bbw_rk_surface_bern_slice: N out of range");
}
