// Fused LSRK stage on the sm_100a tensor cores (tcgen05), nodal variant.
//
// Same stage as kernels_fused.cu (volume + surface + WADG projection + LSRK
// update per element, cpp/src/WaveOKL3d.cpp:2084-2106) with the dense
// reference-element contractions - Dr/Ds/Dt (gradient and divergence),
// LIFT, Vq and Pq - executed as tcgen05.mma (kind::f16, FP32 accumulation in
// tensor memory).
//
// Precision: every contraction A x is evaluated as
//     A_hi x_hi + A_hi x_lo + A_lo x_hi
// with A = A_hi + A_lo and s x = x_hi + x_lo split into FP16 pairs (22
// significant bits) and s a per-tile power of two that maps the operand into
// [-1, 1); the dropped A_lo x_lo term and the residual of the splits are
// O(2^-22) relative to the tile maximum, i.e. FP32-class.  State, fluxes,
// geometric factors and the LSRK update stay FP32.  The same kernel with
// BF16 pairs (BF = true; 16 significant bits, FP32's exponent range) gives
// the split-BF16 form of the precision study: O(2^-16) per contraction.
//
// Orientation: operator rows on the MMA M dimension (64 or 128), the 32
// elements of a tile on N, the reduction index on K.  Operators (A) are
// staged once per CTA; element operands (B) are written per tile by the
// CUDA-core producer phase.  Accumulators: TMEM columns [0,96) gradient
// (r,s,t), [96,128) divergence, [128,256) lift per face; then [0,32) Vq and
// [32,64) Pq.
//
// Inputs arrive by 1-D TMA bulk copies: each element's 4 Np state record
// into a row of stride RS (RS/4 odd, so lane-per-element float4 reads are
// conflict-free), the packed geometry record and the neighbour codes.  The
// state buffer is released as soon as the producers have consumed it, so
// the next tile's copies overlap the MMAs and epilogues.  The LSRK update
// reads the old state and residual from global memory in the epilogues
// (thread = node row, coalesced).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "bbwadg.h"
#include "device_common.cuh"
#include "fused.h"
#include "tc_sm100.cuh"

namespace bbw {

constexpr int TC_E = 32;   // elements per tile (MMA N)
constexpr int TC_T = 512;  // threads per CTA (16 warps)
constexpr uint32_t TC_WAIT = 1u << 22;  // bounded mbarrier polls

__host__ __device__ constexpr int r16(int x) { return (x + 15) & ~15; }
__host__ __device__ constexpr int cdv(int a, int b) { return (a + b - 1) / b; }

template <int N>
struct TcCfg {
  static constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N);
  static constexpr int KV = r16(Np), KF = r16(Nfp);
  // raw state row stride (floats): multiple of 4 with RS/4 odd
  static constexpr int RS = (Np % 2) ? 4 * Np : 4 * Np + 4;
  // flux items with lane = face node: (element, face) pairs per warp
  static constexpr int FPW = (4 * TC_E) / (TC_T / 32);
  static_assert((4 * TC_E) % (TC_T / 32) == 0, "face pairs per warp");
  static_assert(NFP(N) <= 32, "one face per warp pass");
  static_assert(Np <= 64 && Np % 4 == 0, "tensor-core stage: Np <= 64, Np % 4 == 0");
};

TcLayout tc_layout(int N, int Nq, int table_ints) {
  TcLayout L;
  const int Np = NP(N), Nfp = NFP(N);
  L.KV = r16(Np);
  L.KF = r16(Nfp);
  L.KQ = r16(Nq);
  L.MQ = Nq <= 64 ? 64 : 128;
  const int RS = (Np % 2) ? 4 * Np : 4 * Np + 4;
  // operator halves: D_d hi/lo [64][KV] x3, LIFT_f hi/lo [64][KF] x4,
  // Vq hi/lo [MQ][KV], Pq hi/lo [64][KQ]
  L.oD = 0;
  L.oL = L.oD + 6 * 64 * L.KV;
  L.oVq = L.oL + 8 * 64 * L.KF;
  L.oPq = L.oVq + 2 * L.MQ * L.KV;
  L.ops_halfs = L.oPq + 2 * 64 * L.KQ;
  auto al = [](int b) { return (b + 127) & ~127; };
  int o = 0;
  L.ops = o;
  o = al(o + 2 * L.ops_halfs);
  L.Bp = o;
  o = al(o + 2 * (2 * TC_E * L.KV));
  L.BU = o;
  o = al(o + 2 * std::max(6 * TC_E * L.KV, 2 * TC_E * L.KQ));
  L.BF = o;
  o = al(o + 2 * (8 * TC_E * L.KF));
  L.raw = o;
  o = al(o + 4 * TC_E * RS);
  L.geo = o;
  o = al(o + 4 * 2 * TC_E * TC_GEO);
  L.nbr = o;
  o = al(o + 4 * 4 * TC_E);
  L.tab = o;
  o = al(o + 4 * table_ints);
  L.misc = o;
  o = al(o + 64);
  L.total = o;
  return L;
}

struct TcParams {
  int K, Nq, bc;
  float fa, fb, fdt;
  const float *__restrict__ Qin;
  float *__restrict__ Qout;
  float *__restrict__ res;
  const float *__restrict__ geo;  // [K][TC_GEO]: vgeo 9 | fgeo 16 | pad
  const int *__restrict__ nbr;    // [K][4]
  const float *__restrict__ c2q;  // [K][Nq]
  const void *__restrict__ ops;  // split operators: __half, or __nv_bfloat16 (BF)
  const int *__restrict__ tables;
  int table_ints, pat_off;
  int *err;
  TcLayout L;
};

__device__ __forceinline__ float pow2_scale(int bits_of_max) {
  // s = 2^-E with max = m 2^E, m in [0.5, 1): max * s < 1.  E is clamped to
  // [-100, 100] so that s and 1/s stay finite normal numbers (a tile whose
  // values are all below 2^-100 keeps them below 1 after scaling; they are
  // far below the FP32 resolution of any tile that carries the solution)
  const float mx = __int_as_float(bits_of_max);
  if (!(mx > 0.f) || !isfinite(mx)) return 1.f;
  int E;
  frexpf(mx, &E);
  E = max(-100, min(100, E));
  return ldexpf(1.f, -E);
}

// float -> the operand type and back (round to nearest)
__device__ __forceinline__ void to_e(float x, __half &h) { h = __float2half_rn(x); }
__device__ __forceinline__ void to_e(float x, __nv_bfloat16 &h) { h = __float2bfloat16_rn(x); }
__device__ __forceinline__ float from_e(__half h) { return __half2float(h); }
__device__ __forceinline__ float from_e(__nv_bfloat16 h) { return __bfloat162float(h); }

template <class E>
__device__ __forceinline__ void split_store4(E *hi, E *lo, float4 v, float s) {
  const float x[4] = {v.x * s, v.y * s, v.z * s, v.w * s};
  E h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    to_e(x[i], h[i]);
    to_e(x[i] - from_e(h[i]), l[i]);
  }
  *reinterpret_cast<uint2 *>(hi) = *reinterpret_cast<uint2 *>(h);
  *reinterpret_cast<uint2 *>(lo) = *reinterpret_cast<uint2 *>(l);
}

template <class E>
__device__ __forceinline__ void split_store1(E *hi, E *lo, float x) {
  E h, l;
  to_e(x, h);
  to_e(x - from_e(h), l);
  *hi = h;
  *lo = l;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <int N, bool BF>
__global__ void __launch_bounds__(TC_T, 1) k_tc_stage(TcParams P) {
  // operand type; A and B of every MMA share it (the instruction descriptor
  // sets both formats from FMT)
  using E = typename std::conditional<BF, __nv_bfloat16, __half>::type;
  constexpr int FMT = BF ? 1 : 0;
  using C = TcCfg<N>;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NF, KV = C::KV, KF = C::KF, RS = C::RS;
  constexpr int FPW = C::FPW;
  extern __shared__ __align__(1024) unsigned char smem[];
  const TcLayout &L = P.L;
  const int KQ = L.KQ, MQ = L.MQ, Nq = P.Nq;
  E *sOps = reinterpret_cast<E *>(smem + L.ops);
  E *sBp = reinterpret_cast<E *>(smem + L.Bp);
  E *sBU = reinterpret_cast<E *>(smem + L.BU);
  E *sBF = reinterpret_cast<E *>(smem + L.BF);
  float *sRaw = reinterpret_cast<float *>(smem + L.raw);
  float *sGeoB = reinterpret_cast<float *>(smem + L.geo);
  int *sNbr = reinterpret_cast<int *>(smem + L.nbr);
  int *sTab = reinterpret_cast<int *>(smem + L.tab);
  uint64_t *mbarT = reinterpret_cast<uint64_t *>(smem + L.misc);
  uint64_t *mbarM = mbarT + 1;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbarT + 2);
  int *sRed = reinterpret_cast<int *>(tslot + 2);  // [8] maxima as float bits
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q4 = warp & 3, g8 = warp >> 2;  // TMEM sub-partition, element group

  // ---------------------------------------------------------------- setup
  if (tid == 0) {
    tc::mbar_init(mbarT, 1);
    tc::mbar_init(mbarM, 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, 256);
    tc::tmem_relinquish();
  }
  for (int i = tid; i < L.ops_halfs / 8; i += TC_T)
    reinterpret_cast<uint4 *>(sOps)[i] = __ldg(reinterpret_cast<const uint4 *>(P.ops) + i);
  for (int i = tid; i < P.table_ints; i += TC_T) sTab[i] = __ldg(P.tables + i);
  for (int i = tid; i < (L.raw - L.Bp) / 16; i += TC_T)  // B operands: zero padding
    reinterpret_cast<uint4 *>(smem + L.Bp)[i] = make_uint4(0, 0, 0, 0);
  for (int i = tid; i < TC_E * RS; i += TC_T) sRaw[i] = 0.f;  // absent elements stay finite
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  const int *sFmask = sTab;
  const int *sPat = sTab + P.pat_off;
  const int ntiles = cdv(P.K, TC_E);
  // Failure path: a bounded wait that gives up sets `fail` (made warp
  // uniform at once, so the warp-collective TMEM loads stay converged); the
  // thread then skips every shared-memory, TMEM and global access that
  // depends on the awaited data.  At the next CTA barrier the whole CTA
  // votes, stops issuing copies and MMAs, and leaves the tile loop; thread 0
  // then waits (bounded again) for the copies and MMAs it still has in
  // flight before the TMEM is freed, and the error flag is raised.
  bool fail = false;
  bool tma_pend = false, mma_pend = false;  // thread 0: issued, completion not yet seen
  uint32_t tma_par = 0, mma_par = 0;        // their mbarrier phases

  auto issue_tma = [&](int tile, int gb, uint32_t parity) {  // thread 0
    const int k0 = tile * TC_E, ne = min(TC_E, P.K - k0);
    tma_pend = true, tma_par = parity;
    const uint32_t bytes = (uint32_t)ne * (4 * Np * 4 + TC_GEO * 4 + 16);
    tc::mbar_expect_tx(mbarT, bytes);
    for (int e = 0; e < ne; ++e)
      tc::bulk_g2s(sRaw + e * RS, P.Qin + (size_t)(k0 + e) * 4 * Np, 4 * Np * 4, mbarT);
    tc::bulk_g2s(sGeoB + gb * TC_E * TC_GEO, P.geo + (size_t)k0 * TC_GEO, ne * TC_GEO * 4, mbarT);
    tc::bulk_g2s(sNbr, P.nbr + (size_t)k0 * 4, ne * 16, mbarT);
  };
  uint32_t tphase = 0, mphase = 0;
  auto mma_commit = [&]() {  // thread 0
    tc::mma_commit(mbarM);
    mma_pend = true, mma_par = mphase;
  };
  auto mma_wait = [&]() {
    const bool ok = tc::mbar_wait(mbarM, mphase, TC_WAIT);
    if (ok && tid == 0) mma_pend = false;
    fail = __any_sync(0xffffffffu, fail || !ok);
    mphase ^= 1u;
    tc::fence_after_sync();
  };
  auto sync_for_mma = [&]() {  // generic smem writes -> tensor core
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  };
  // one operator/operand product chain: D (+)= A B^T over ksteps, 3 products
  // descriptors of consecutive K steps differ only in the start-address field
  // (+256 bytes = +16 in 16-byte units)
  auto chain = [&](uint32_t d, const E *Ahi, const E *Alo, int asbo, const E *Bhi,
                   const E *Blo, int bsbo, int ksteps, uint32_t idesc, bool acc) {
    uint64_t ah = tc::smem_desc(tc::smem_u32(Ahi), 128, asbo);
    uint64_t al = tc::smem_desc(tc::smem_u32(Alo), 128, asbo);
    uint64_t bh = tc::smem_desc(tc::smem_u32(Bhi), 128, bsbo);
    uint64_t bl = tc::smem_desc(tc::smem_u32(Blo), 128, bsbo);
    for (int s = 0; s < ksteps; ++s) {
      tc::mma_f16(d, ah, bh, idesc, (acc || s > 0) ? 1u : 0u);
      tc::mma_f16(d, ah, bl, idesc, 1u);
      tc::mma_f16(d, al, bh, idesc, 1u);
      ah += 16, al += 16, bh += 16, bl += 16;
    }
  };

  // face traces of neighbours outside tile `tile` (whose inputs have landed)
  // into registers.  Lane = face node, warp = (element, face) pairs: one load
  // instruction reads the face of a single neighbour (a few sectors) instead
  // of one node of 32 neighbours.  Traces inside the tile are read from
  // shared memory in P1.
  float nbv[FPW][4];
  auto load_traces = [&](int tile) {
    const int k0 = tile * TC_E, ne = min(TC_E, P.K - k0);
#pragma unroll
    for (int j = 0; j < FPW; ++j) {
      nbv[j][0] = nbv[j][1] = nbv[j][2] = nbv[j][3] = 0.f;
      const int pp = warp * FPW + j, e = pp >> 2, f = pp & 3;
      if (lane >= Nfp || e >= ne) continue;
      const int code = sNbr[e * 4 + f];
      const int pat = code & 255;
      if (pat == 255) continue;
      const unsigned rel = (unsigned)((code >> 8) - k0);
      if (rel < (unsigned)ne) continue;
      const float *o = P.Qin + (size_t)(code >> 8) * 4 * Np + sPat[pat * Nfp + lane];
      nbv[j][0] = __ldg(o), nbv[j][1] = __ldg(o + Np), nbv[j][2] = __ldg(o + 2 * Np),
      nbv[j][3] = __ldg(o + 3 * Np);
    }
  };

  if (blockIdx.x < ntiles && tid == 0) issue_tma(blockIdx.x, 0, tphase);
  int it = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const int k0 = tile * TC_E, ne = min(TC_E, P.K - k0), gb = it & 1;
    const float *sGeo = sGeoB + gb * TC_E * TC_GEO;
    const int next = tile + gridDim.x;

    // ---- P0: tile inputs (issued during the previous tile's epilogues);
    //          outside neighbour traces in flight through the first half of P1
    {
      const bool ok = tc::mbar_wait(mbarT, tphase, TC_WAIT);
      if (ok && tid == 0) tma_pend = false;
      fail = __any_sync(0xffffffffu, fail || !ok);
    }
    tphase ^= 1u;
    if (!fail) load_traces(tile);
    if (tid < 8) sRed[tid] = 0;
    if (__syncthreads_or(fail)) {
      fail = true;
      break;
    }

    // ---- P1: p and contravariant velocities (4 nodes x 1 element per item),
    //          then the upwind flux; maxima
    constexpr int NC = KV / 4;  // node chunks incl. padding
    const int ce = tid & 31, cc = tid >> 5;  // item (chunk cc, element ce); TC_T = 16 * 32
    float G[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) G[i] = sGeo[ce * TC_GEO + i];
    float4 p4 = make_float4(0.f, 0.f, 0.f, 0.f), U4[3];
    U4[0] = U4[1] = U4[2] = p4;
    float mp = 0.f, mU = 0.f;
    if (cc < NC && 4 * cc < Np && ce < ne) {
      const float *rr = sRaw + ce * RS + 4 * cc;
      p4 = *reinterpret_cast<const float4 *>(rr);
      const float4 u4 = *reinterpret_cast<const float4 *>(rr + Np);
      const float4 v4 = *reinterpret_cast<const float4 *>(rr + 2 * Np);
      const float4 w4 = *reinterpret_cast<const float4 *>(rr + 3 * Np);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        U4[d].x = u4.x * G[3 * d] + v4.x * G[3 * d + 1] + w4.x * G[3 * d + 2];
        U4[d].y = u4.y * G[3 * d] + v4.y * G[3 * d + 1] + w4.y * G[3 * d + 2];
        U4[d].z = u4.z * G[3 * d] + v4.z * G[3 * d + 1] + w4.z * G[3 * d + 2];
        U4[d].w = u4.w * G[3 * d] + v4.w * G[3 * d + 1] + w4.w * G[3 * d + 2];
        mU = fmaxf(mU, fmaxf(fmaxf(fabsf(U4[d].x), fabsf(U4[d].y)),
                             fmaxf(fabsf(U4[d].z), fabsf(U4[d].w))));
      }
      mp = fmaxf(fmaxf(fabsf(p4.x), fabsf(p4.y)), fmaxf(fabsf(p4.z), fabsf(p4.w)));
    }
    // upwind flux (Uflux = -pflux), lane = face node: last, its outside
    // traces have had longest
    float pf[FPW];
    float mF = 0.f;
#pragma unroll
    for (int j = 0; j < FPW; ++j) {
      pf[j] = 0.f;
      const int pp = warp * FPW + j, e = pp >> 2, f = pp & 3;
      if (lane >= Nfp || e >= ne) continue;
      const int m = f * Nfp + lane;
      const int code = sNbr[e * 4 + f];
      const int pat = code & 255;
      const int vM = sFmask[m];
      const float *own = sRaw + e * RS + vM;
      const float pM = own[0], uM = own[Np], vvM = own[2 * Np], wM = own[3 * Np];
      const float *fg = sGeo + e * TC_GEO + 9 + 4 * f;
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
        const unsigned rel = (unsigned)((code >> 8) - k0);
        float pP = nbv[j][0], uP = nbv[j][1], vP_ = nbv[j][2], wP = nbv[j][3];
        if (rel < (unsigned)ne) {  // neighbour inside the tile
          const float *o = sRaw + rel * RS + sPat[pat * Nfp + lane];
          pP = o[0], uP = o[Np], vP_ = o[2 * Np], wP = o[3 * Np];
        }
        pjump = pP - pM;
        Unjump = (uP - uM) * nx + (vP_ - vvM) * ny + (wP - wM) * nz;
      }
      pf[j] = .5f * (pjump - Unjump) * Fscale;
      mF = fmaxf(mF, fabsf(pf[j]));
    }
    mp = warp_max(mp);
    mU = warp_max(mU);
    mF = warp_max(mF);
    if (lane == 0) {
      atomicMax(&sRed[0], __float_as_int(mp));
      atomicMax(&sRed[1], __float_as_int(mU));
      atomicMax(&sRed[2], __float_as_int(mF));
    }
    __syncthreads();
    const float sp = pow2_scale(sRed[0]), sU = pow2_scale(sRed[1]), sF = pow2_scale(sRed[2]);
    // B operands (element rows, K-major): p, U_d, per-face pflux
    if (cc < NC) {
      const int o = tc::kmajor_offset_f16(ce, 4 * cc, KV);
      split_store4(sBp + o, sBp + TC_E * KV + o, p4, sp);
#pragma unroll
      for (int d = 0; d < 3; ++d)
        split_store4(sBU + 2 * d * TC_E * KV + o, sBU + (2 * d + 1) * TC_E * KV + o, U4[d], sU);
    }
#pragma unroll
    for (int j = 0; j < FPW; ++j) {
      const int pp = warp * FPW + j, e = pp >> 2, f = pp & 3;
      if (lane >= Nfp) continue;  // absent elements store zeros (pf = 0)
      const int o = tc::kmajor_offset_f16(e, lane, KF);
      split_store1(sBF + 2 * f * TC_E * KF + o, sBF + (2 * f + 1) * TC_E * KF + o, pf[j] * sF);
    }
    sync_for_mma();

    // ---- P2: gradient, divergence, lift MMAs; meanwhile every thread fetches
    //          the old residual of u, v, w for its rows of epilogue 1
    const int n = 16 * q4 + lane;  // M = 64 layout: lanes 0..15 of each sub-partition
    const bool rowok = lane < 16 && n < Np;
    if (tid == 0) {
      const uint32_t id64 = tc::idesc_f16(64, TC_E, FMT);
      const int sboV = (KV / 8) * 128, sboF = (KF / 8) * 128;
      for (int d = 0; d < 3; ++d)
        chain(tbase + 32 * d, sOps + L.oD + 2 * d * 64 * KV, sOps + L.oD + (2 * d + 1) * 64 * KV,
              sboV, sBp, sBp + TC_E * KV, sboV, KV / 16, id64, false);
      for (int d = 0; d < 3; ++d)
        chain(tbase + 96, sOps + L.oD + 2 * d * 64 * KV, sOps + L.oD + (2 * d + 1) * 64 * KV, sboV,
              sBU + 2 * d * TC_E * KV, sBU + (2 * d + 1) * TC_E * KV, sboV, KV / 16, id64, d > 0);
      for (int f = 0; f < 4; ++f)
        chain(tbase + 128 + 32 * f, sOps + L.oL + 2 * f * 64 * KF,
              sOps + L.oL + (2 * f + 1) * 64 * KF, sboF, sBF + 2 * f * TC_E * KF,
              sBF + (2 * f + 1) * TC_E * KF, sboF, KF / 16, id64, false);
      mma_commit();
    }
    float ro[8][3];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = 8 * g8 + j;
      const size_t id = (size_t)(k0 + e) * 4 * Np + n;
#pragma unroll
      for (int fl = 1; fl < 4; ++fl) ro[j][fl - 1] = rowok && e < ne ? P.res[id + fl * Np] : 0.f;
    }
    mma_wait();

    // ---- P3: epilogue 1 (thread = node row n, 8 elements): rhs of p, u, v, w;
    //          LSRK update of u, v, w (old state from the tile in shared
    //          memory); rhs_p -> B operand of the Vq product
    const uint32_t trow = tbase + ((uint32_t)(32 * q4) << 16) + 8 * g8;
    float rp[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (!fail) {
      float gr[8], gs[8], gt[8], dv[8], lf[4][8];
      tc::tmem_ld8x4(trow + 0, trow + 32, trow + 64, trow + 96, gr, gs, gt, dv);
      tc::tmem_ld8x4(trow + 128, trow + 160, trow + 192, trow + 224, lf[0], lf[1], lf[2], lf[3]);
      const float isp = 1.f / sp, isU = 1.f / sU, isF = 1.f / sF;
      float mr = 0.f;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int e = 8 * g8 + j;
        const float *Ge = sGeo + e * TC_GEO;
        const float dr = gr[j] * isp, ds = gs[j] * isp, dt = gt[j] * isp;
        float vp = -dv[j] * isU;
        float vu = -(Ge[0] * dr + Ge[3] * ds + Ge[6] * dt);
        float vv = -(Ge[1] * dr + Ge[4] * ds + Ge[7] * dt);
        float vw = -(Ge[2] * dr + Ge[5] * ds + Ge[8] * dt);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const float a = lf[f][j] * isF;
          vp += a;
          vu -= Ge[9 + 4 * f + 1] * a;
          vv -= Ge[9 + 4 * f + 2] * a;
          vw -= Ge[9 + 4 * f + 3] * a;
        }
        const bool ok = rowok && e < ne;
        rp[j] = ok ? vp : 0.f;
        mr = fmaxf(mr, fabsf(rp[j]));
        if (ok) {
          const size_t id = (size_t)(k0 + e) * 4 * Np + n;
          const float rv3[3] = {vu, vv, vw};
#pragma unroll
          for (int fl = 1; fl < 4; ++fl) {
            const float r = P.fa * ro[j][fl - 1] + P.fdt * rv3[fl - 1];
            P.res[id + fl * Np] = r;
            P.Qout[id + fl * Np] = sRaw[e * RS + fl * Np + n] + P.fb * r;
          }
        }
      }
      mr = warp_max(mr);
      if (lane == 0) atomicMax(&sRed[3], __float_as_int(mr));
    }
    if (__syncthreads_or(fail)) {
      fail = true;
      break;
    }
    // the state tile is dead: the next tile's copies overlap the rest
    if (tid == 0 && next < ntiles) issue_tma(next, gb ^ 1, tphase);
    const float srp = pow2_scale(sRed[3]);
    if (lane < 16) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int e = 8 * g8 + j;
        const int o = tc::kmajor_offset_f16(e, n, KV);
        if (n < KV) split_store1(sBp + o, sBp + TC_E * KV + o, rp[j] * srp);
      }
    }
    sync_for_mma();

    // ---- P4: Vq product; meanwhile c2/J of this thread's cubature row
    if (tid == 0) {
      chain(tbase + 0, sOps + L.oVq, sOps + L.oVq + MQ * KV, (KV / 8) * 128, sBp, sBp + TC_E * KV,
            (KV / 8) * 128, KV / 16, tc::idesc_f16(MQ, TC_E, FMT), false);
      mma_commit();
    }
    const int q = MQ == 128 ? 32 * q4 + lane : (lane < 16 ? 16 * q4 + lane : MQ);
    float c2v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = 8 * g8 + j;
      c2v[j] = q < Nq && e < ne ? __ldg(P.c2q + (size_t)(k0 + e) * Nq + q) : 0.f;
    }
    mma_wait();

    // ---- P5: epilogue 2 (thread = cubature row q): c2/J * p_q -> B operand
    {
      float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (!fail) tc::tmem_ld8(tbase + ((uint32_t)(32 * q4) << 16) + 8 * g8, v);
      const float isr = 1.f / srp;
      float mc = 0.f;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        v[j] = v[j] * isr * c2v[j];
        mc = fmaxf(mc, fabsf(v[j]));
      }
      mc = warp_max(mc);
      if (lane == 0) atomicMax(&sRed[4], __float_as_int(mc));
      if (__syncthreads_or(fail)) {
        fail = true;
        break;
      }
      const float sc = pow2_scale(sRed[4]);
      if (q < KQ) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int e = 8 * g8 + j;
          const int o = tc::kmajor_offset_f16(e, q, KQ);
          split_store1(sBU + o, sBU + TC_E * KQ + o, v[j] * sc);
        }
      }
      sync_for_mma();

      // ---- P6: Pq product
      if (tid == 0) {
        chain(tbase + 32, sOps + L.oPq, sOps + L.oPq + 64 * KQ, (KQ / 8) * 128, sBU,
              sBU + TC_E * KQ, (KQ / 8) * 128, KQ / 16, tc::idesc_f16(64, TC_E, FMT), false);
        mma_commit();
      }
      float r7[8], q7[8];  // old residual and state of p, fetched during the MMAs
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int e = 8 * g8 + j;
        const size_t id = (size_t)(k0 + e) * 4 * Np + n;
        r7[j] = rowok && e < ne ? P.res[id] : 0.f;
        q7[j] = rowok && e < ne ? __ldg(P.Qin + id) : 0.f;
      }
      mma_wait();

      // ---- P7: epilogue 3: rhs_p = Pq (c2 p_q); LSRK update of p
      float w[8];
      if (!fail) tc::tmem_ld8(tbase + ((uint32_t)(32 * q4) << 16) + 32 + 8 * g8, w);
      const float isc = 1.f / sc;
      if (rowok && !fail) {
        const float *ro = r7, *qo = q7;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int e = 8 * g8 + j;
          if (e >= ne) continue;
          const size_t id = (size_t)(k0 + e) * 4 * Np + n;
          const float r = P.fa * ro[j] + P.fdt * (w[j] * isc);
          P.res[id] = r;
          P.Qout[id] = qo[j] + P.fb * r;
        }
      }
    }
    tc::fence_before_sync();
    // TMEM, B operands and reduction slots free for the next tile
    if (__syncthreads_or(fail)) {
      fail = true;
      break;
    }
    tc::fence_after_sync();
  }
  if (fail && tid == 0) {
    // drain this CTA's own copies and MMAs still in flight (bounded), so
    // nothing lands in shared memory or TMEM after they are released
    if (tma_pend) tc::mbar_wait(mbarT, tma_par, TC_WAIT);
    if (mma_pend) tc::mbar_wait(mbarM, mma_par, TC_WAIT);
    atomicAdd(P.err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 256);
}

// --------------------------------------------------------------- host side
template <int N, bool BF>
static bbw_status tc_prepare_n(TcPlan &pl) {
  int dev = 0, maxsm = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (pl.L.total > maxsm)
    return set_error(BBW_ERR_UNSUPPORTED, "tensor-core stage: shared-memory footprint too large");
  // the limit is per kernel and device while the footprint depends on the
  // mesh (face-permutation table): raise it to the device maximum once
  const bbw_status s = ensure_smem_limit(k_tc_stage<N, BF>, maxsm, "tensor-core stage attribute");
  if (s != BBW_OK) return s;
  pl.nsm = nsm > 0 ? nsm : 148;
  pl.grid = std::min(cdv(pl.K, TC_E), pl.nsm);
  return BBW_OK;
}

template <int N, bool BF>
static bbw_status tc_launch_n(const TcPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                              float fb, float fdt, cudaStream_t st) {
  TcParams P;
  P.K = pl.K, P.Nq = pl.Nq, P.bc = pl.bc;
  P.fa = fa, P.fb = fb, P.fdt = fdt;
  P.Qin = Qin, P.Qout = Qout, P.res = res;
  P.geo = pl.geo, P.nbr = pl.nbr, P.c2q = pl.c2q;
  P.ops = pl.ops;
  P.tables = pl.tables, P.table_ints = pl.table_ints, P.pat_off = pl.pat_off;
  P.err = pl.err;
  P.L = pl.L;
  const int grid = pl.max_ctas > 0 ? std::min(pl.grid, pl.max_ctas) : pl.grid;
  k_tc_stage<N, BF><<<grid, TC_T, pl.L.total, st>>>(P);
  return check_launch("tensor-core stage");
}

bool tc_supported(int N, int Nq) {
  return (N == 3 || N == 5) && Nq >= 1 && Nq <= 128;
}

bbw_status tc_prepare(TcPlan &pl) {
  switch (pl.N * 2 + (pl.bf ? 1 : 0)) {
    case 6: return tc_prepare_n<3, false>(pl);
    case 7: return tc_prepare_n<3, true>(pl);
    case 10: return tc_prepare_n<5, false>(pl);
    case 11: return tc_prepare_n<5, true>(pl);
  }
  return set_error(BBW_ERR_UNSUPPORTED, "tensor-core stage: N must be 3 or 5");
}

bbw_status tc_launch(const TcPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                     float fb, float fdt, cudaStream_t st) {
  switch (pl.N * 2 + (pl.bf ? 1 : 0)) {
    case 6: return tc_launch_n<3, false>(pl, Qin, Qout, res, fa, fb, fdt, st);
    case 7: return tc_launch_n<3, true>(pl, Qin, Qout, res, fa, fb, fdt, st);
    case 10: return tc_launch_n<5, false>(pl, Qin, Qout, res, fa, fb, fdt, st);
    case 11: return tc_launch_n<5, true>(pl, Qin, Qout, res, fa, fb, fdt, st);
  }
  return set_error(BBW_ERR_UNSUPPORTED, "tensor-core stage: N must be 3 or 5");
}

// FP16 (or BF16, bf) hi/lo split of an FP32 operator into the canonical
// K-major layout (rows padded to `rows`, K padded to kp), as raw 16-bit
// words; host side
void tc_pack_operator(const float *A, int nrows, int ncols, int ld_row, int ld_col, int rows,
                      int kp, uint16_t *hi, uint16_t *lo, bool bf) {
  for (int r = 0; r < rows; ++r)
    for (int k = 0; k < kp; ++k) {
      const float a = (r < nrows && k < ncols) ? A[(size_t)r * ld_row + (size_t)k * ld_col] : 0.f;
      const int o = tc::kmajor_offset_f16(r, k, kp);
      if (bf) {
        const __nv_bfloat16 h = __float2bfloat16_rn(a);
        const __nv_bfloat16 l = __float2bfloat16_rn(a - __bfloat162float(h));
        std::memcpy(&hi[o], &h, 2), std::memcpy(&lo[o], &l, 2);
      } else {
        const __half h = __float2half_rn(a);
        const __half l = __float2half_rn(a - __half2float(h));
        std::memcpy(&hi[o], &h, 2), std::memcpy(&lo[o], &l, 2);
      }
    }
}

}  // namespace bbw
