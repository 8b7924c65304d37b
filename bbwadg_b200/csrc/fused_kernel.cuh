#pragma once
// Fused LSRK stage for the affine-tet acoustic WADG method (sm_100a):
// kernel template and its host-side launch helpers, instantiated per order N
// by kernels_fused_n<N>.cu.
//
// One kernel per stage replaces the reference's three launches
// (rk_volume + rk_surface + rk_update_WADG, cpp/src/WaveOKL3d.cpp:2084-2106,
// or their BB counterparts): per element it forms the volume term, the upwind
// surface flux and lift, projects c^2 * rhs_p with the WADG operators and
// applies the LSRK45 stage update, reading each element's state once from
// HBM and writing the new state and residual once.
//
// Work decomposition: a persistent CTA owns a tile of E consecutive elements
// at a time (E = 32, or 16 where a 32-element tile's arrays do not fit in
// shared memory); the CTA's threads form groups of E, thread l of a group
// works on element l of the tile and group g owns a block of R output rows
// (nodes) or RQ cubature points.  With E = 32 a group is a warp; with E = 16
// a warp holds two groups.  The reference-element operators are staged in
// shared memory once per CTA in a per-group packed layout, so every operator
// read is a (half-)warp-uniform broadcast (float4) while the element data is
// read conflict-free with thread = element.  State tiles are moved between
// HBM and shared memory with coalesced traffic and transposed to
// [row][element] (row stride E + 1) on the way.
//
// Double-buffered state: the stage reads Qin (this element and its
// neighbours' face traces) and writes Qout, so neighbour gathers never race
// with updates.  res is updated in place.
//
// Connectivity: vmapP is compressed at context creation into, per element
// face, the neighbour element and the index of its face-node permutation
// (at most 24 distinct permutations exist: 4 faces x 6 orientations), the
// permutations being kept in a small table; boundary faces are flagged.
//
// Simplifications that are exact in exact arithmetic and checked at
// creation: Uflux = -pflux (both are formed from the same jump with opposite
// sign, cpp/okl/WaveKernels.okl:215-216), so one lift of pflux per face
// serves p and, scaled by -n_f, u,v,w; with Jq = 1 (affine tets,
// cpp/src/WaveOKL3d.cpp:463) the velocity rows of the WADG update are
// Pq*Vq = I and are skipped.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bbwadg.h"
#include "device_common.cuh"
#include "fused.h"

namespace bbw {

__host__ __device__ constexpr int round4(int x) { return (x + 3) & ~3; }
__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// warps per CTA: 8 or 16 (run-time choice, see fused_prepare / bbw_autotune)
__host__ __device__ constexpr int fused_default_warps_c(int N) { return N <= 3 ? 8 : 16; }

template <int N, int W_, int E_ = 32>
struct FusedCfg {
  static_assert(E_ == 16 || E_ == 32, "element tile of 16 or 32");
  static constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N);
  static constexpr int W = W_;  // warps per CTA
  static constexpr int T = 32 * W;
  static constexpr int E = E_;        // elements per tile
  static constexpr int ES = E_ + 1;   // shared-memory row stride (floats)
  static constexpr int NG = T / E_;   // thread groups (one element each) per CTA
  static constexpr int R = cdiv(Np, NG);    // node rows per group
  static constexpr int R2 = cdiv(R, 2);     // row pairs (packed FP32 FMAs)
  static constexpr int PR = round4(R);
  static constexpr int P3R = round4(6 * R2);
};

// packed FP32 pair helpers (sm_100 FFMA2: two independent FMAs per
// instruction, each rounded as a scalar FMA)
__device__ __forceinline__ float2 pair(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 pair(float a) { return make_float2(a, a); }
__device__ __forceinline__ float pick(const float2 *v, int i) { return (i & 1) ? v[i >> 1].y : v[i >> 1].x; }

// ------------------------------------------------------------------ layouts
// Operators, packed per thread group so that group g reads one contiguous,
// 16-byte aligned block per reduction index (NG groups):
//   vol  [NG][Np(m)][P3R]  rows in pairs p = i/2: (Dr, Ds, Dt)[r0+i][m] at
//                          6p + (i%2) + {0, 2, 4}
//   lift [NG][NF(m)][PR]   LIFT[r0+i][m]
//   pq   [NG][Nq(q)][PR]   Pq[r0+i][q]
//   vq   [NG][Np(n)][PRQ]  Vq[q0+i][n]
// plus, for BB, the sparse tables.  Built on the host (fused_host.cu).
struct FusedParams {
  int K, Nq, RQ, PRQ, bc, npat;
  int Kc;  // elements [K0, Kc) are advanced; the others supply neighbour traces only
  int pat_off, bb_off;              // int offsets of the tables (multiples of 4)
  float fa, fb, fdt;
  const float *__restrict__ Qin;
  float *__restrict__ Qout;
  float *__restrict__ res;
  const float *__restrict__ vgeo;   // [K][9]
  const float *__restrict__ fgeo;   // [K][16]
  const int *__restrict__ nbr;      // [K][4]  (k2 << 8) | pattern, pattern 255 = boundary
  const float *__restrict__ c2q;    // [K][Nq] c2/J at the cubature points
  const float *__restrict__ ops;    // packed operators (global copy)
  int off_lift, off_pq, off_vq, off_end;  // operator offsets in ops (floats)
  const int *__restrict__ tables;   // Fmask [NF] | patterns [npat][Nfp] | BB tables
  int table_ints;
  // batched shots: state arrays hold S consecutive [K][4][Np] blocks
  int S;
  // sources: entries [src_off[s], src_off[s+1]) of shot s add
  // ricker(t) * src_vec[j][:] to the projected rhs_p of element src_elem[j],
  // t = *time + cstage * fdt
  const int *__restrict__ src_off;
  const int *__restrict__ src_elem;
  const float *__restrict__ src_vec;
  float f0, tR, samp, cstage;
  const double *__restrict__ time;  // simulation time at the start of the step
  // optional: Vq (raw rhs_p) at the cubature points, before c2/J, stored as
  // [shot][Nq][K] (the c^2 gradient of the discrete adjoint needs it)
  float *__restrict__ vq_out;
  int K0;  // first advanced element (read only by the WIN variants; kept last
           // so the other fields keep their offsets)
};

// Ricker wavelet amp (1 - 2 a^2) exp(-a^2), a = pi f0 (t - tR)
__device__ __forceinline__ float ricker(float t, float f0, float tR, float amp) {
  const float a = 3.14159265358979f * f0 * (t - tR);
  return amp * (1.f - 2.f * a * a) * expf(-a * a);
}

// Shared-memory map (floats, rows of stride ES).  Input tiles are double
// buffered when they fit (PIPE): the next tile's copies are in flight while
// the current one is computed.
template <int N, bool BB, int E_>
struct FusedSmem {
  using C = FusedCfg<N, 8, E_>;  // row counts only; independent of the warp count
  static constexpr int ES = C::ES;
  static constexpr int inQ = 0;                               // [4Np][ES] state tile
  static constexpr int inGeo = 4 * C::Np * ES;                // [E][25]  vgeo + fgeo
  static constexpr int inNbr = inGeo + E_ * 25;               // [E][4]   neighbour codes
  static constexpr int inC2 = inNbr + E_ * 4;                 // [Nq][ES] c2 (runtime Nq)
  __host__ __device__ static int in_size(int Nq) { return inC2 + round4(Nq * ES); }
  static constexpr int sR = 0;                                // [4Np][ES] rhs / U scratch
  static constexpr int sF = sR + 4 * C::Np * ES;              // [NF][ES]  pflux
  static constexpr int sF2 = sF + C::NF * ES;                 // [NF][ES]  BB: L0 * pflux
  static constexpr int sQuad = sF2 + (BB ? C::NF * ES : 0);   // [Nq][ES]  c2 * p at the cubature
  __host__ __device__ static int work_size(int Nq) { return sQuad + round4(Nq * ES); }
};

// -------------------------------------------------------------- device code
__device__ __forceinline__ void cp_async4(void *smem_dst, const void *gmem_src, bool valid) {
  // 4-byte asynchronous copy; zero-fills the destination when !valid
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(gmem_src),
               "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// OPS_SMEM: the packed operators are staged in shared memory (every
// operator read is a shared-memory broadcast); otherwise they are read
// through the read-only data path (large N or large cubature rules).
// PIPE: two input-tile buffers (software pipelining across tiles).
// WIN: the advanced elements start at P.K0 (a window of a split stage);
// without it they start at 0, a constant, which keeps the window arithmetic
// out of the whole-mesh stage.
template <int N, bool BB, bool OPS_SMEM, bool PIPE, int W_, int E_ = 32, bool WIN = false>
__global__ void __launch_bounds__(FusedCfg<N, W_, E_>::T, 1) k_fused_stage(FusedParams P) {
  using C = FusedCfg<N, W_, E_>;
  const int K0 = WIN ? P.K0 : 0;  // first element advanced
  using L = FusedSmem<N, BB, E_>;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NF, T = C::T, R = C::R;
  constexpr int E = C::E, ES = C::ES, NG = C::NG;
  constexpr int FIT = cdiv(E * NF, T);        // flux items per thread
  constexpr int QIT = cdiv(E * 4 * Np, T);    // state-tile floats per thread
  extern __shared__ __align__(16) float sm[];
  const int Nq = P.Nq, RQ = P.RQ, PRQ = P.PRQ;
  const int inSize = L::in_size(Nq);
  float *sIn = sm;                                   // [PIPE ? 2 : 1][inSize]
  float *sW = sm + (PIPE ? 2 : 1) * inSize;          // work arrays
  float *sR = sW + L::sR, *sF = sW + L::sF, *sF2 = sW + L::sF2, *sQuad = sW + L::sQuad;
  // tables staged in shared memory: all of them with the operators, else
  // Fmask and the face permutations only (the BB tables are then read
  // through the cache like the operators)
  const int tabSmem = OPS_SMEM ? P.table_ints : P.bb_off;
  int *sTab = (int *)(sW + L::work_size(Nq));
  float *sOps = (float *)(sTab + tabSmem);
  // el: element of the tile this thread works on; grp: its row block
  const int tid = threadIdx.x, el = tid & (E - 1), grp = tid / E;
  const int r0 = grp * R;

  // stage operators (when they fit) and tables once per CTA
  if (OPS_SMEM)
    for (int i = tid; i < P.off_end / 4; i += T)
      reinterpret_cast<float4 *>(sOps)[i] = __ldg(reinterpret_cast<const float4 *>(P.ops) + i);
  for (int i = tid; i < tabSmem; i += T) sTab[i] = __ldg(P.tables + i);
  const int *sFmask = sTab;
  const int *sPat = sTab + P.pat_off;

  const float *opBase = OPS_SMEM ? (const float *)sOps : P.ops;
  const float *wVol = opBase + grp * Np * C::P3R;              // [NG][Np][P3R]
  const float *wLift = opBase + P.off_lift + grp * NF * C::PR;  // [NG][NF][PR]
  const float *wPq = opBase + P.off_pq + grp * Nq * C::PR;      // [NG][Nq][PR]
  const float *wVq = opBase + P.off_vq + grp * Np * PRQ;        // [NG][Np][PRQ]
  // BB tables: D ids int4 [4][Np], Dvals float4 [Np], then the lift tables
  const int *bbTab = OPS_SMEM ? sTab + P.bb_off : P.tables + P.bb_off;

  // asynchronous copies of one tile's inputs into buffer `buf`
  const int ntiles = cdiv(P.Kc - K0, E);
  const size_t sstride = (size_t)P.K * 4 * Np;  // floats per shot
  // parts of a tile's inputs: geometry + neighbour codes, state, c2
  constexpr int IN_GEO = 1, IN_Q = 2, IN_C2 = 4, IN_ALL = 7;
  auto issue_tile = [&](int vt, float *buf, int parts) {
    const int shot = vt / ntiles, tile = vt - shot * ntiles;
    const int k0 = K0 + tile * E, ne = min(E, P.Kc - k0);
    float *bQ = buf + L::inQ, *bGeo = buf + L::inGeo, *bC2 = buf + L::inC2;
    int *bNbr = (int *)(buf + L::inNbr);
    if (parts & IN_GEO) {
    for (int i = tid; i < E * 9; i += T)
      cp_async4(&bGeo[(i / 9) * 25 + i % 9], P.vgeo + (size_t)k0 * 9 + (i < ne * 9 ? i : 0), i < ne * 9);
    for (int i = tid; i < E * 16; i += T)
      cp_async4(&bGeo[(i / 16) * 25 + 9 + i % 16], P.fgeo + (size_t)k0 * 16 + (i < ne * 16 ? i : 0),
                i < ne * 16);
    // zero codes of absent elements: element 0, permutation 0 (the host
    // always provides that table row); their fluxes are never used
    for (int i = tid; i < E * 4; i += T)
      cp_async4(&bNbr[i], P.nbr + (size_t)k0 * 4 + (i < ne * 4 ? i : 0), i < ne * 4);
    }
    if (parts & IN_Q) {
    const float *Qg = P.Qin + shot * sstride + (size_t)k0 * 4 * Np;
#pragma unroll 4
    for (int j = 0; j < QIT; ++j) {
      const int i = tid + j * T;
      if (i < E * 4 * Np) {
        const int e = i / (4 * Np), fn = i - e * (4 * Np);
        const bool ok = e < ne;
        cp_async4(&bQ[fn * ES + e], ok ? Qg + i : P.Qin, ok);
      }
    }
    }
    if (parts & IN_C2) {
    const float *cg = P.c2q + (size_t)k0 * Nq;
    for (int i = tid; i < E * Nq; i += T) {
      const int e = i / Nq, q = i - e * Nq;
      const bool ok = e < ne;
      cp_async4(&bC2[q * ES + e], ok ? cg + i : P.c2q, ok);
    }
    }
    cp_async_commit();
  };
  // neighbour face traces of the tile in `buf` into registers
  auto load_traces = [&](const float *buf, int vt, float (&nb)[FIT][4]) {
    const int shot = vt / ntiles, tile_of_buf = vt - shot * ntiles;
    const int kb = K0 + tile_of_buf * E;  // first element of the tile
    const int ne_b = min(E, P.Kc - kb);
    const int *bNbr = (const int *)(buf + L::inNbr);
#pragma unroll
    for (int j = 0; j < FIT; ++j) {
      const int i = tid + j * T;
      nb[j][0] = nb[j][1] = nb[j][2] = nb[j][3] = 0.f;
      if (i < E * NF && (i & (E - 1)) < ne_b) {  // absent elements have no codes
        const int e = i & (E - 1), m = i / E, f = m / Nfp;
        const int code = bNbr[e * 4 + f];
        const int pat = code & 255;
        const unsigned rel = (unsigned)((code >> 8) - kb);
        if (pat != 255 && rel >= (unsigned)ne_b) {  // neighbours inside the tile: from smem
          const float *q2 = P.Qin + shot * sstride + (size_t)(code >> 8) * 4 * Np +
                            sPat[pat * Nfp + (m - f * Nfp)];
          nb[j][0] = __ldg(q2);
          nb[j][1] = __ldg(q2 + Np);
          nb[j][2] = __ldg(q2 + 2 * Np);
          nb[j][3] = __ldg(q2 + 3 * Np);
        }
      }
    }
  };

  const int nvt = P.S * ntiles;  // (shot, tile) work items
  int vt = blockIdx.x, b = 0;
  float nb[FIT][4];
  __syncthreads();  // tables staged
  if (vt < nvt) {
    issue_tile(vt, sIn, IN_ALL);
    cp_async_wait_all();
    __syncthreads();
    load_traces(sIn, vt, nb);
  }
  for (; vt < nvt; vt += gridDim.x) {
    const int shot = vt / ntiles, tile = vt - shot * ntiles;
    const int k0 = K0 + tile * E;
    const int ne = min(E, P.Kc - k0);
    const int next = vt + gridDim.x;
    const size_t sbase = shot * sstride;
    float *cur = sIn + b * inSize;
    const float *sQ = cur + L::inQ, *sGeo = cur + L::inGeo, *sC2 = cur + L::inC2;
    const int *sNbr = (const int *)(cur + L::inNbr);
    // inputs of the next tile: with two buffers all at once; with one
    // buffer each part as soon as this tile is done with it (geometry and
    // state after the lift, c2 after the cubature step), the update then
    // reading the old state from global memory
    if (PIPE && next < nvt) issue_tile(next, sIn + (b ^ 1) * inSize, IN_ALL);

    // ---- 1. upwind flux at the 4Nfp face nodes (Uflux = -pflux); traces of
    //         neighbours inside the tile come from the state tile itself
#pragma unroll
    for (int j = 0; j < FIT; ++j) {
      const int i = tid + j * T;
      if (i >= E * NF) continue;
      const int e = i & (E - 1), m = i / E, f = m / Nfp;
      const int code = sNbr[e * 4 + f];
      const int pat = code & 255;
      const unsigned rel = (unsigned)((code >> 8) - k0);
      if (pat != 255 && rel < (unsigned)ne) {
        const int vP = sPat[pat * Nfp + (m - f * Nfp)];
        nb[j][0] = sQ[vP * ES + rel];
        nb[j][1] = sQ[(Np + vP) * ES + rel];
        nb[j][2] = sQ[(2 * Np + vP) * ES + rel];
        nb[j][3] = sQ[(3 * Np + vP) * ES + rel];
      }
      const int vM = sFmask[m];
      const float pM = sQ[vM * ES + e], uM = sQ[(Np + vM) * ES + e],
                  vvM = sQ[(2 * Np + vM) * ES + e], wM = sQ[(3 * Np + vM) * ES + e];
      const float *fg = sGeo + e * 25 + 9 + 4 * f;
      const float Fscale = fg[0], nx = fg[1], ny = fg[2], nz = fg[3];
      float pjump, Unjump;
      if (pat == 255) {
        if (P.bc == BBW_BC_PRESSURE_RELEASE) {
          pjump = -2.f * pM;
          Unjump = 0.f;
        } else {
          pjump = 0.f;
          Unjump = -2.f * (uM * nx + vvM * ny + wM * nz);
        }
      } else {
        pjump = nb[j][0] - pM;
        Unjump = (nb[j][1] - uM) * nx + (nb[j][2] - vvM) * ny + (nb[j][3] - wM) * nz;
      }
      sF[m * ES + e] = .5f * (pjump - Unjump) * Fscale;
    }

    // ---- 2. contravariant velocities Ur, Us, Ut into sR rows [Np, 4Np)
    for (int i = tid; i < E * Np; i += T) {
      const int e = i & (E - 1), n = i / E;
      const float *G = sGeo + e * 25;
      const float u = sQ[(Np + n) * ES + e], v = sQ[(2 * Np + n) * ES + e],
                  w = sQ[(3 * Np + n) * ES + e];
      sR[(Np + n) * ES + e] = u * G[0] + v * G[1] + w * G[2];
      sR[(2 * Np + n) * ES + e] = u * G[3] + v * G[4] + w * G[5];
      sR[(3 * Np + n) * ES + e] = u * G[6] + v * G[7] + w * G[8];
    }
    __syncthreads();

    // ---- 3. volume term (registers: rows r0..r0+R of this group, thread = element)
    float rp[R], ru[R], rv[R], rw[R];
    {
      const float *G = sGeo + el * 25;
      if constexpr (!BB) {
        // rows in pairs: per pair the operator block is
        // (Dr, Dr', Ds, Ds', Dt, Dt') of rows (i, i+1)
        constexpr int R2 = C::R2;
        float2 dr[R2], ds[R2], dt[R2], dv[R2];
#pragma unroll
        for (int i = 0; i < R2; ++i) dr[i] = ds[i] = dt[i] = dv[i] = pair(0.f);
#pragma unroll 2
        for (int m = 0; m < Np; ++m) {
          const float2 pm = pair(sQ[m * ES + el]);
          const float2 ur = pair(sR[(Np + m) * ES + el]), us = pair(sR[(2 * Np + m) * ES + el]),
                       ut = pair(sR[(3 * Np + m) * ES + el]);
          const float4 *op = reinterpret_cast<const float4 *>(wVol + m * C::P3R);
          float o[C::P3R];
#pragma unroll
          for (int j = 0; j < C::P3R / 4; ++j) {
            const float4 t4 = op[j];
            o[4 * j] = t4.x, o[4 * j + 1] = t4.y, o[4 * j + 2] = t4.z, o[4 * j + 3] = t4.w;
          }
#pragma unroll
          for (int i = 0; i < R2; ++i) {
            const float2 Dr = pair(o[6 * i], o[6 * i + 1]), Ds = pair(o[6 * i + 2], o[6 * i + 3]),
                         Dt = pair(o[6 * i + 4], o[6 * i + 5]);
            dr[i] = __ffma2_rn(Dr, pm, dr[i]);
            ds[i] = __ffma2_rn(Ds, pm, ds[i]);
            dt[i] = __ffma2_rn(Dt, pm, dt[i]);
            dv[i] = __ffma2_rn(Dr, ur, dv[i]);
            dv[i] = __ffma2_rn(Ds, us, dv[i]);
            dv[i] = __ffma2_rn(Dt, ut, dv[i]);
          }
        }
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const float a = pick(dr, i), bs = pick(ds, i), c = pick(dt, i);
          rp[i] = -pick(dv, i);
          ru[i] = -(G[0] * a + G[3] * bs + G[6] * c);
          rv[i] = -(G[1] * a + G[4] * bs + G[7] * c);
          rw[i] = -(G[2] * a + G[5] * bs + G[8] * c);
        }
      } else {
        // sparse Bernstein derivative, cpp/okl/WaveKernels.okl:428-467
        const int4 *Dids = reinterpret_cast<const int4 *>(bbTab);          // [4][Np]
        const float4 *Dv = reinterpret_cast<const float4 *>(bbTab + 16 * Np);  // [Np]
        const float *p = sQ + el, *ur = sR + Np * ES + el, *us = sR + 2 * Np * ES + el,
                    *ut = sR + 3 * Np * ES + el;
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const int n = r0 + i;
          rp[i] = ru[i] = rv[i] = rw[i] = 0.f;
          if (n >= Np) continue;
          const float4 dv = Dv[n];
          const int4 a = Dids[n], bq = Dids[Np + n], c = Dids[2 * Np + n], d = Dids[3 * Np + n];
          const float p1 = dv.x * p[a.x * ES] + dv.y * p[bq.x * ES] + dv.z * p[c.x * ES] +
                           dv.w * p[d.x * ES];
          const float p2 = dv.x * p[a.y * ES] + dv.y * p[bq.y * ES] + dv.z * p[c.y * ES] +
                           dv.w * p[d.y * ES];
          const float p3 = dv.x * p[a.z * ES] + dv.y * p[bq.z * ES] + dv.z * p[c.z * ES] +
                           dv.w * p[d.z * ES];
          const float p4 = dv.x * p[a.w * ES] + dv.y * p[bq.w * ES] + dv.z * p[c.w * ES] +
                           dv.w * p[d.w * ES];
          float dU1 = dv.x * (ur[a.y * ES] + us[a.z * ES] + ut[a.w * ES]);
          dU1 += dv.y * (ur[bq.y * ES] + us[bq.z * ES] + ut[bq.w * ES]);
          dU1 += dv.z * (ur[c.y * ES] + us[c.z * ES] + ut[c.w * ES]);
          dU1 += dv.w * (ur[d.y * ES] + us[d.z * ES] + ut[d.w * ES]);
          float dU2 = dv.x * (ur[a.x * ES] + us[a.x * ES] + ut[a.x * ES]);
          dU2 += dv.y * (ur[bq.x * ES] + us[bq.x * ES] + ut[bq.x * ES]);
          dU2 += dv.z * (ur[c.x * ES] + us[c.x * ES] + ut[c.x * ES]);
          dU2 += dv.w * (ur[d.x * ES] + us[d.x * ES] + ut[d.x * ES]);
          const float dpdr = .5f * (p2 - p1), dpds = .5f * (p3 - p1), dpdt = .5f * (p4 - p1);
          rp[i] = -.5f * (dU1 - dU2);
          ru[i] = -(G[0] * dpdr + G[3] * dpds + G[6] * dpdt);
          rv[i] = -(G[1] * dpdr + G[4] * dpds + G[7] * dpdt);
          rw[i] = -(G[2] * dpdr + G[5] * dpds + G[8] * dpdt);
        }
      }
    }

    // ---- 4. lift of the face fluxes
    {
      const float *fgl = sGeo + el * 25 + 9;
      if constexpr (!BB) {
#pragma unroll 1
        for (int f = 0; f < 4; ++f) {
          float2 acc[C::PR / 2];
#pragma unroll
          for (int i = 0; i < C::PR / 2; ++i) acc[i] = pair(0.f);
#pragma unroll 3
          for (int j = 0; j < Nfp; ++j) {
            const int m = f * Nfp + j;
            const float2 pf = pair(sF[m * ES + el]);
            const float4 *op = reinterpret_cast<const float4 *>(wLift + m * C::PR);
#pragma unroll
            for (int q = 0; q < C::PR / 4; ++q) {
              const float4 t4 = op[q];
              acc[2 * q] = __ffma2_rn(pair(t4.x, t4.y), pf, acc[2 * q]);
              acc[2 * q + 1] = __ffma2_rn(pair(t4.z, t4.w), pf, acc[2 * q + 1]);
            }
          }
          const float nx = fgl[4 * f + 1], ny = fgl[4 * f + 2], nz = fgl[4 * f + 3];
#pragma unroll
          for (int i = 0; i < R; ++i) {
            const float a = pick(acc, i);
            rp[i] += a;
            ru[i] -= nx * a;
            rv[i] -= ny * a;
            rw[i] -= nz * a;
          }
        }
      } else {
        // BB lift: per face L0 (Nfp x Nfp sparse), then the degree elevation
        // EEL face by face (cpp/okl/WaveKernels.okl:576-644).  Tables: header
        // {L0nnz, EEL nnz}, L0 (offset, value) pairs [Nfp][L0nnz], EEL row
        // pointers [Np][5], EEL (offset, value) pairs; offsets are
        // pre-multiplied by the row stride.
        __syncthreads();  // pflux complete (written in step 1 by other warps)
        const int L0nnz = bbTab[20 * Np];
        const int2 *L0p = reinterpret_cast<const int2 *>(bbTab + 20 * Np + 4);
        const int *eelPtr = bbTab + 20 * Np + 4 + 2 * Nfp * L0nnz;
        const int2 *eelP = reinterpret_cast<const int2 *>(eelPtr + ((5 * Np + 1) & ~1));
        for (int m = grp; m < NF; m += NG) {
          const int f = m / Nfp, nt = m - f * Nfp;
          const float *src = sF + f * Nfp * ES + el;
          const int2 *row = L0p + nt * L0nnz;
          float v0 = 0.f, v1 = 0.f;
          int j = 0;
          for (; j + 1 < L0nnz; j += 2) {
            const int2 t0 = row[j], t1 = row[j + 1];
            v0 += __int_as_float(t0.y) * src[t0.x * ES];
            v1 += __int_as_float(t1.y) * src[t1.x * ES];
          }
          if (j < L0nnz) v0 += __int_as_float(row[j].y) * src[row[j].x * ES];
          sF2[m * ES + el] = v0 + v1;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const int n = r0 + i;
          if (n >= Np) continue;
          const int *ptr = eelPtr + 5 * n;
#pragma unroll 1
          for (int f = 0; f < 4; ++f) {
            float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
            int j = ptr[f];
            const int end = ptr[f + 1];
            for (; j + 3 < end; j += 4) {
              const int2 t0 = eelP[j], t1 = eelP[j + 1], t2 = eelP[j + 2], t3 = eelP[j + 3];
              a0 += __int_as_float(t0.y) * sF2[t0.x * ES + el];
              a1 += __int_as_float(t1.y) * sF2[t1.x * ES + el];
              a2 += __int_as_float(t2.y) * sF2[t2.x * ES + el];
              a3 += __int_as_float(t3.y) * sF2[t3.x * ES + el];
            }
            for (; j < end; ++j) a0 += __int_as_float(eelP[j].y) * sF2[eelP[j].x * ES + el];
            const float acc = (a0 + a1) + (a2 + a3);
            rp[i] += acc;
            ru[i] -= fgl[4 * f + 1] * acc;
            rv[i] -= fgl[4 * f + 2] * acc;
            rw[i] -= fgl[4 * f + 3] * acc;
          }
        }
      }
    }
    __syncthreads();  // all warps done reading Ur/Us/Ut from sR
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int n = r0 + i;
      if (n < Np) {
        sR[n * ES + el] = rp[i];
        sR[(Np + n) * ES + el] = ru[i];
        sR[(2 * Np + n) * ES + el] = rv[i];
        sR[(3 * Np + n) * ES + el] = rw[i];
      }
    }
    if (!PIPE && next < nvt) issue_tile(next, sIn, IN_GEO | IN_Q);  // sQ, sGeo, sNbr are dead
    if (PIPE) cp_async_wait_all();  // the next tile's inputs have landed
    __syncthreads();
    if (PIPE && next < nvt) load_traces(sIn + (b ^ 1) * inSize, next, nb);  // in flight from here

    // ---- 5. WADG: p at the cubature points, times c2/J
    {
      // blocks of QB cubature rows: QB independent accumulators per thread,
      // one state value and QB/4 operator broadcasts per node
      constexpr int QB = fused_vq_block(NG);
      const int q0 = grp * RQ;
      for (int qb = 0; qb < RQ; qb += QB) {
        float2 acc[QB / 2];
#pragma unroll
        for (int j = 0; j < QB / 2; ++j) acc[j] = pair(0.f);
#pragma unroll 2
        for (int n = 0; n < Np; ++n) {
          const float2 x = pair(sR[n * ES + el]);
          const float4 *v = reinterpret_cast<const float4 *>(wVq + n * PRQ + qb);
#pragma unroll
          for (int j = 0; j < QB / 4; ++j) {
            const float4 t4 = v[j];
            acc[2 * j] = __ffma2_rn(pair(t4.x, t4.y), x, acc[2 * j]);
            acc[2 * j + 1] = __ffma2_rn(pair(t4.z, t4.w), x, acc[2 * j + 1]);
          }
        }
#pragma unroll
        for (int j = 0; j < QB; ++j) {
          const int q = q0 + qb + j;
          if (qb + j < RQ && q < Nq) {
            sQuad[q * ES + el] = pick(acc, j) * sC2[q * ES + el];
            if (P.vq_out && el < ne)
              P.vq_out[((size_t)shot * Nq + q) * P.K + k0 + el] = pick(acc, j);
          }
        }
      }
    }
    __syncthreads();
    if (!PIPE && next < nvt) issue_tile(next, sIn, IN_C2);  // sC2 is dead

    // ---- 6. project back: rhs_p = Pq * (c2 p_q); the residual tile is
    //         fetched meanwhile for the stage update (scalar, coalesced)
    constexpr int UIT = cdiv(E * 4 * Np, T);
    const float *resg = P.res + sbase + (size_t)k0 * 4 * Np;
    float rpre[UIT];
#pragma unroll
    for (int j = 0; j < UIT; ++j) {
      const int i = tid + j * T;
      rpre[j] = i < ne * 4 * Np ? resg[i] : 0.f;
    }
    {
      float2 acc2[C::PR / 2];
#pragma unroll
      for (int i = 0; i < C::PR / 2; ++i) acc2[i] = pair(0.f);
#pragma unroll 2
      for (int q = 0; q < Nq; ++q) {
        const float2 x = pair(sQuad[q * ES + el]);
        const float4 *op = reinterpret_cast<const float4 *>(wPq + q * C::PR);
#pragma unroll
        for (int j = 0; j < C::PR / 4; ++j) {
          const float4 t4 = op[j];
          acc2[2 * j] = __ffma2_rn(pair(t4.x, t4.y), x, acc2[2 * j]);
          acc2[2 * j + 1] = __ffma2_rn(pair(t4.z, t4.w), x, acc2[2 * j + 1]);
        }
      }
      float acc[R];
#pragma unroll
      for (int i = 0; i < R; ++i) acc[i] = pick(acc2, i);
      // source term of this shot, added to the projected rhs_p as
      // rk_update_elas does (acous_elas_cpp/okl/ElasKernelsWADG.okl:400-403)
      if (P.src_off) {
        // entries of a shot are sorted by element: find the first one of
        // this tile by bisection, then walk the tile's entries
        int j0 = __ldg(P.src_off + shot), j1 = __ldg(P.src_off + shot + 1);
        if (j1 > j0) {
          int lo = j0, hi = j1;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(P.src_elem + mid) < k0) lo = mid + 1;
            else hi = mid;
          }
          if (lo < j1 && __ldg(P.src_elem + lo) < k0 + ne) {
            const float amp = ricker((float)(*P.time) + P.cstage * P.fdt, P.f0, P.tR, P.samp);
            for (int j = lo; j < j1; ++j) {
              const int rel = __ldg(P.src_elem + j) - k0;
              if (rel >= ne) break;
              if (el == rel) {
#pragma unroll
                for (int i = 0; i < R; ++i)
                  if (r0 + i < Np) acc[i] += amp * __ldg(P.src_vec + (size_t)j * Np + r0 + i);
              }
            }
          }
        }
      }
      __syncthreads();  // everyone has read sR rows [0, Np) in step 5
#pragma unroll
      for (int i = 0; i < R; ++i)
        if (r0 + i < Np) sR[(r0 + i) * ES + el] = acc[i];
    }
    __syncthreads();

    // ---- 7. LSRK stage update, coalesced and conflict-free:
    //         res = fa res + fdt rhs; Q += fb res
    {
      float *resw = P.res + sbase + (size_t)k0 * 4 * Np;
      float *qg = P.Qout + sbase + (size_t)k0 * 4 * Np;
      const float *qin = P.Qin + sbase + (size_t)k0 * 4 * Np;
      float qold[PIPE ? 1 : UIT];  // one buffer: the state tile is being refilled
      if (!PIPE) {
#pragma unroll
        for (int j = 0; j < UIT; ++j) {
          const int i = tid + j * T;
          qold[PIPE ? 0 : j] = i < ne * 4 * Np ? __ldg(qin + i) : 0.f;
        }
      }
#pragma unroll
      for (int j = 0; j < UIT; ++j) {
        const int i = tid + j * T;
        if (i >= ne * 4 * Np) continue;
        const int e = i / (4 * Np), fn = i - e * (4 * Np);
        const float r = P.fa * rpre[j] + P.fdt * sR[fn * ES + e];
        resw[i] = r;
        qg[i] = (PIPE ? sQ[fn * ES + e] : qold[PIPE ? 0 : j]) + P.fb * r;
      }
    }
    __syncthreads();  // tile buffers and work arrays free for reuse
    if (!PIPE && next < nvt) {
      cp_async_wait_all();
      __syncthreads();
      load_traces(sIn, next, nb);
    }
    b ^= PIPE ? 1 : 0;
  }
}

// --------------------------------------------------------------- host side
template <int N, bool BB, int E>
static size_t smem_bytes(int Nq, bool pipe, bool ops_smem, int ops_floats, int table_ints,
                         int bb_off) {
  if (!ops_smem) table_ints = bb_off;
  using L = FusedSmem<N, BB, E>;
  return sizeof(float) * ((size_t)(pipe ? 2 : 1) * L::in_size(Nq) + L::work_size(Nq) +
                          (ops_smem ? ops_floats : 0)) +
         sizeof(int) * (size_t)table_ints;
}

template <int N, bool BB, int E>
static bbw_status launch_fused(const FusedPlan &pl, const float *Qin, float *Qout, float *res,
                               float fa, float fb, float fdt, float cstage, cudaStream_t st) {
  FusedParams P;
  P.K = pl.K, P.Nq = pl.Nq, P.RQ = pl.RQ, P.PRQ = pl.PRQ, P.bc = pl.bc, P.npat = pl.npat;
  P.Kc = pl.Kc > 0 ? pl.Kc : pl.K;
  P.K0 = pl.K0;
  P.pat_off = pl.pat_off, P.bb_off = pl.bb_off;
  P.fa = fa, P.fb = fb, P.fdt = fdt;
  P.Qin = Qin, P.Qout = Qout, P.res = res;
  P.vgeo = pl.vgeo, P.fgeo = pl.fgeo, P.nbr = pl.nbr, P.c2q = pl.c2q;
  P.ops = pl.ops;
  P.off_lift = pl.off_lift, P.off_pq = pl.off_pq, P.off_vq = pl.off_vq, P.off_end = pl.ops_floats;
  P.tables = pl.tables, P.table_ints = pl.table_ints;
  P.S = pl.S;
  P.src_off = pl.src_off, P.src_elem = pl.src_elem, P.src_vec = pl.src_vec;
  P.f0 = pl.f0, P.tR = pl.tR, P.samp = pl.samp, P.cstage = cstage;
  P.time = pl.time;
  P.vq_out = pl.vq_out;
  const bool os = pl.ops_smem > 0;
  size_t sm = pl.smem;
  const int ctas = pl.max_ctas > 0 ? std::min(pl.max_ctas, pl.nsm) : pl.nsm;
  const int grid =
      std::min(cdiv((pl.Kc > 0 ? pl.Kc : pl.K) - pl.K0, E) * std::max(pl.S, 1), ctas);
  if (pl.K0 > 0) {  // a window of a split stage: the single-buffered WIN variants
    sm = smem_bytes<N, BB, E>(pl.Nq, false, os, pl.ops_floats, pl.table_ints, pl.bb_off);
    if (pl.W == 8) {
      if (os) k_fused_stage<N, BB, true, false, 8, E, true><<<grid, 256, sm, st>>>(P);
      else k_fused_stage<N, BB, false, false, 8, E, true><<<grid, 256, sm, st>>>(P);
    } else {
      if (os) k_fused_stage<N, BB, true, false, 16, E, true><<<grid, 512, sm, st>>>(P);
      else k_fused_stage<N, BB, false, false, 16, E, true><<<grid, 512, sm, st>>>(P);
    }
    return check_launch("fused stage (window)");
  }
  if (pl.W == 8) {
    constexpr int T = 256;
    if (os && pl.pipe) k_fused_stage<N, BB, true, true, 8, E><<<grid, T, sm, st>>>(P);
    else if (os) k_fused_stage<N, BB, true, false, 8, E><<<grid, T, sm, st>>>(P);
    else if (pl.pipe) k_fused_stage<N, BB, false, true, 8, E><<<grid, T, sm, st>>>(P);
    else k_fused_stage<N, BB, false, false, 8, E><<<grid, T, sm, st>>>(P);
  } else {
    constexpr int T = 512;
    if (os && pl.pipe) k_fused_stage<N, BB, true, true, 16, E><<<grid, T, sm, st>>>(P);
    else if (os) k_fused_stage<N, BB, true, false, 16, E><<<grid, T, sm, st>>>(P);
    else if (pl.pipe) k_fused_stage<N, BB, false, true, 16, E><<<grid, T, sm, st>>>(P);
    else k_fused_stage<N, BB, false, false, 16, E><<<grid, T, sm, st>>>(P);
  }
  return check_launch("fused stage");
}

// The dynamic shared-memory limit is a per-kernel, per-device attribute
// while a plan's size depends on its mesh (the face-permutation table), so
// every variant's limit is raised to the device maximum once: contexts on
// different meshes then never undercut each other's launches.
template <int N, bool BB, int E, int W>
static bbw_status set_smem_attr(int bytes) {
  const void *fn[6] = {(const void *)k_fused_stage<N, BB, true, true, W, E>,
                       (const void *)k_fused_stage<N, BB, true, false, W, E>,
                       (const void *)k_fused_stage<N, BB, false, true, W, E>,
                       (const void *)k_fused_stage<N, BB, false, false, W, E>,
                       (const void *)k_fused_stage<N, BB, true, false, W, E, true>,
                       (const void *)k_fused_stage<N, BB, false, false, W, E, true>};
  for (const void *f : fn) {
    const bbw_status s = ensure_smem_limit(f, bytes, "fused stage attribute");
    if (s != BBW_OK) return s;
  }
  return BBW_OK;
}

template <int N, bool BB, int E>
static bbw_status prepare(FusedPlan &pl) {
  int dev = 0, maxsm = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (pl.W != 8 && pl.W != 16) return set_error(BBW_ERR_ARG, "fused stage: warps must be 8 or 16");
  // requested placement (want_ops / want_pipe >= 0) or the first that fits of:
  // operators in shared memory, then double-buffered input tiles
  const bool cand[4][2] = {{true, true}, {true, false}, {false, true}, {false, false}};
  int pick = -1;
  for (int c = 0; c < 4 && pick < 0; ++c) {
    if (pl.want_ops >= 0 && cand[c][0] != (pl.want_ops > 0)) continue;
    if (pl.want_pipe >= 0 && cand[c][1] != (pl.want_pipe > 0)) continue;
    if (smem_bytes<N, BB, E>(pl.Nq, cand[c][1], cand[c][0], pl.ops_floats, pl.table_ints,
                             pl.bb_off) <= (size_t)maxsm)
      pick = c;
  }
  if (pick < 0)
    return set_error(BBW_ERR_UNSUPPORTED, "fused stage: element tile does not fit in shared memory");
  pl.ops_smem = cand[pick][0] ? pl.ops_floats : 0;
  pl.pipe = cand[pick][1];
  pl.smem = smem_bytes<N, BB, E>(pl.Nq, pl.pipe, pl.ops_smem > 0, pl.ops_floats, pl.table_ints,
                                 pl.bb_off);
  bbw_status st =
      pl.W == 8 ? set_smem_attr<N, BB, E, 8>(maxsm) : set_smem_attr<N, BB, E, 16>(maxsm);
  if (st != BBW_OK) return st;
  pl.nsm = nsm > 0 ? nsm : 148;
  pl.grid = std::min(cdiv(pl.Kc > 0 ? pl.Kc : pl.K, E) * std::max(pl.S, 1), pl.nsm);
  return BBW_OK;
}

}  // namespace bbw
