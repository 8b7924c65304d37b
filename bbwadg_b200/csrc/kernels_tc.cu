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
// staged once per CTA with only round8(Np) rows (round16(Nq) for Vq) stored:
// an M = 64 (128) MMA reads its remaining rows from whatever follows in
// shared memory, and those rows only feed accumulator rows that are never
// read.  The operators' K padding is stored as zeros, so it meets the zero K
// padding of the element operands (B) in exact zero products.
//
// Work items are (shot, tile of 32 elements); a persistent CTA walks them
// with a grid stride and keeps two in flight in one instruction stream:
//
//   a. epilogue 1 of tile T: rhs of u, v, w and the LSRK update of u, v, w
//      from the gradient / divergence / lift accumulators; rhs_p split into
//      the B operand of Vq; issue the Vq MMAs
//   b. while they run: tile T+1 (its bulk copies were issued one tile
//      earlier) - neighbour traces, upwind flux, B operands of its first
//      MMA group
//   c. epilogue 2 of T: c^2 / J at the cubature points -> B operand of Pq;
//      issue the Pq MMAs of T, the first MMA group of T+1, the bulk copies
//      of T+2
//   d. epilogue 3 of T: rhs_p, sources, LSRK update of p, while T+1's MMAs
//      run.
//
// TMEM (512 columns): [0,96) gradient r,s,t, [96,128) divergence,
// [128,256) lift per face, [256,288) Vq, [288,320) Pq.  For M = 64 an
// accumulator row m lives in lane (m % 16) + 32 (m / 16); the epilogues read
// those with the 16x64b shape, so all 32 threads of a warp hold a (row,
// element) pair.  The LSRK update reads the old state and residual from
// global memory (L2), so the state tile in shared memory is free for the
// next copies as soon as the tile's B operands are built.
//
// Every mbarrier wait is bounded.  A wait that gives up sets a warp-uniform
// failure flag; the thread then skips every access that depends on the
// awaited data, the CTA votes at its next barrier, issues no further copy or
// MMA and leaves the loop; thread 0 waits (bounded) for what it still has
// in flight before the TMEM is freed and the error flag is raised.
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
constexpr uint32_t TC_COLS = 512;       // TMEM columns allocated
constexpr uint32_t cGrad = 0, cDiv = 96, cLift = 128, cVq = 256, cPq = 288;

__host__ __device__ constexpr int r16(int x) { return (x + 15) & ~15; }
__host__ __device__ constexpr int r8(int x) { return (x + 7) & ~7; }
__host__ __device__ constexpr int cdv(int a, int b) { return (a + b - 1) / b; }

template <int N>
struct TcCfg {
  static constexpr int Np = NP(N), Nfp = NFP(N), NF = 4 * NFP(N);
  static constexpr int KV = r16(Np), KF = r16(Nfp);
  // raw state row stride (floats): multiple of 4 with RS/4 odd, so the
  // lane-per-element reads of one node hit distinct bank groups
  static constexpr int RS = (Np % 2) ? 4 * Np : 4 * Np + 4;
  static constexpr bool V4 = Np % 4 == 0;  // field rows 16-byte aligned in the raw tile
  // flux items with lane = face node: (element, face) pairs per warp
  static constexpr int FPW = (4 * TC_E) / (TC_T / 32);
  static_assert((4 * TC_E) % (TC_T / 32) == 0, "face pairs per warp");
  static_assert(NFP(N) <= 32, "one face per warp pass");
  static_assert(Np <= 64, "tensor-core stage: Np <= 64 (operator rows of one M = 64 MMA)");
};

TcLayout tc_layout(int N, int Nq, int table_ints) {
  TcLayout L;
  const int Np = NP(N), Nfp = NFP(N);
  L.KV = r16(Np);
  L.KF = r16(Nfp);
  L.KQ = r16(Nq);
  L.MQ = Nq <= 64 ? 64 : 128;
  L.MR = r8(Np);
  L.MRQ = L.KQ;  // Vq rows [Nq, KQ) are stored zeros: they reach Pq's K padding
  const int RS = (Np % 2) ? 4 * Np : 4 * Np + 4;
  // operator planes (hi, lo): D_d [MR][KV] x3, LIFT_f [MR][KF] x4, Pq [MR][KQ],
  // Vq [MRQ][KV]; each MMA reads 64 - MR (MQ - MRQ) rows past its plane
  L.oD = 0;
  L.oL = L.oD + 6 * L.MR * L.KV;
  L.oPq = L.oL + 8 * L.MR * L.KF;
  L.oVq = L.oPq + 2 * L.MR * L.KQ;
  L.ops_halfs = L.oVq + 2 * L.MRQ * L.KV;
  auto al = [](int b) { return (b + 127) & ~127; };
  int o = 0;
  L.ops = o;
  o = al(o + 2 * L.ops_halfs);
  L.Bp = o;
  o = al(o + 2 * (2 * TC_E * L.KV));
  L.BU = o;
  o = al(o + 2 * (6 * TC_E * L.KV));
  L.BF = o;
  o = al(o + 2 * (8 * TC_E * L.KF));
  L.BW = o;
  o = al(o + 2 * std::max(2 * TC_E * L.KV, 2 * TC_E * L.KQ));
  L.raw = o;
  o = al(o + 4 * TC_E * RS);
  L.geo = o;
  o = al(o + 4 * 2 * TC_E * TC_GEO);
  L.nbr = o;
  o = al(o + 4 * 4 * TC_E);
  L.tab = o;
  o = al(o + 4 * table_ints);
  L.misc = o;
  o = al(o + 128);
  L.total = o;
  return L;
}

struct TcParams {
  int K, Nq, bc, S;
  float fa, fb, fdt, cstage;
  const float *__restrict__ Qin;
  float *__restrict__ Qout;
  float *__restrict__ res;
  const float *__restrict__ geo;  // [K][TC_GEO]: fgeo 16 | vgeo 9 | pad 3 (16-byte groups)
  const int *__restrict__ nbr;    // [K][4]
  const float *__restrict__ c2q;  // [K][Nq]
  const void *__restrict__ ops;   // split operators: __half, or __nv_bfloat16 (BF)
  const int *__restrict__ tables;
  int table_ints, pat_off;
  int *err;
  // sources: entries [src_off[s], src_off[s+1]) of shot s, sorted by element,
  // add ricker(t) * src_vec[j][:] to the projected rhs_p of element
  // src_elem[j], t = *time + cstage * fdt (as the FP32 fused stage)
  const int *__restrict__ src_off;
  const int *__restrict__ src_elem;
  const float *__restrict__ src_vec;
  float f0, tR, samp;
  const double *__restrict__ time;
  // optional: Vq (raw rhs_p) at the cubature points, before c2/J, stored as
  // [shot][Nq][K] (what the adjoint's gradient needs, as the FP32 stage)
  float *__restrict__ vq_out;
  TcLayout L;
};

__device__ __forceinline__ float pow2_scale(int bits_of_max) {
  // s = 2^-E with max = m 2^E, m in [0.5, 1): max * s < 1.  E is clamped to
  // [-100, 100] so that s and 1/s stay finite normal numbers (a tile whose
  // values are all below 2^-100 keeps them below 1 after scaling; they are
  // far below the FP32 resolution of any tile that carries the solution).
  // From the exponent field: E = field - 126 for a normal max; a subnormal
  // max has E <= -126, clamped to -100.
  const float mx = __int_as_float(bits_of_max);
  const int field = (bits_of_max >> 23) & 255;
  if (!(mx > 0.f) || field == 255) return 1.f;
  const int E = max(-100, min(100, field - 126));
  return __int_as_float((127 - E) << 23);
}

// float -> the operand type and back (round to nearest)
__device__ __forceinline__ void to_e(float x, __half &h) { h = __float2half_rn(x); }
__device__ __forceinline__ void to_e(float x, __nv_bfloat16 &h) { h = __float2bfloat16_rn(x); }
__device__ __forceinline__ float from_e(__half h) { return __half2float(h); }
__device__ __forceinline__ float from_e(__nv_bfloat16 h) { return __bfloat162float(h); }

// pairs: float -> two packed values of the operand type and back
__device__ __forceinline__ uint32_t to_e2(float a, float b, __half) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ uint32_t to_e2(float a, float b, __nv_bfloat16) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ float2 from_e2(uint32_t v, __half) {
  return __half22float2(*reinterpret_cast<const __half2 *>(&v));
}
__device__ __forceinline__ float2 from_e2(uint32_t v, __nv_bfloat16) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&v));
}

template <class E>
__device__ __forceinline__ void split_store4(E *hi, E *lo, float4 v, float s) {
  const float x0 = v.x * s, x1 = v.y * s, x2 = v.z * s, x3 = v.w * s;
  const uint32_t h01 = to_e2(x0, x1, E()), h23 = to_e2(x2, x3, E());
  const float2 f01 = from_e2(h01, E()), f23 = from_e2(h23, E());
  const uint32_t l01 = to_e2(x0 - f01.x, x1 - f01.y, E()), l23 = to_e2(x2 - f23.x, x3 - f23.y, E());
  *reinterpret_cast<uint2 *>(hi) = make_uint2(h01, h23);
  *reinterpret_cast<uint2 *>(lo) = make_uint2(l01, l23);
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

// Ricker wavelet amp (1 - 2 a^2) exp(-a^2), a = pi f0 (t - tR)
__device__ __forceinline__ float tc_ricker(float t, float f0, float tR, float amp) {
  const float a = 3.14159265358979f * f0 * (t - tR);
  return amp * (1.f - 2.f * a * a) * expf(-a * a);
}

// An M = 64 accumulator block read with tcgen05.ld.16x64b.x4: the warp
// reads the 16 lanes of its sub-partition (rows 16 q .. 16 q + 15) and 8
// element columns; register j of thread t holds TMEM lane (t / 4) + 8 (t % 2)
// of the sub-partition and column 2 j + (t / 2) % 2 (measured on the B200
// with a store / load round trip of known values).
__device__ __forceinline__ int ep_row(int lane) { return (lane >> 2) + 8 * (lane & 1); }
__device__ __forceinline__ int ep_col(int lane, int j) { return 2 * j + ((lane >> 1) & 1); }

template <int N, bool BF>
__global__ void __launch_bounds__(TC_T, 1) k_tc_stage(TcParams P) {
  // operand type; A and B of every MMA share it (the instruction descriptor
  // sets both formats from FMT)
  using E = typename std::conditional<BF, __nv_bfloat16, __half>::type;
  constexpr int FMT = BF ? 1 : 0;
  using C = TcCfg<N>;
  constexpr int Np = C::Np, Nfp = C::Nfp, KV = C::KV, KF = C::KF, RS = C::RS;
  constexpr int FPW = C::FPW;
  extern __shared__ __align__(1024) unsigned char smem[];
  const TcLayout &L = P.L;
  const int KQ = L.KQ, MQ = L.MQ, MR = L.MR, MRQ = L.MRQ, Nq = P.Nq;
  E *sOps = reinterpret_cast<E *>(smem + L.ops);
  E *sBp = reinterpret_cast<E *>(smem + L.Bp);
  E *sBU = reinterpret_cast<E *>(smem + L.BU);
  E *sBF = reinterpret_cast<E *>(smem + L.BF);
  E *sBW = reinterpret_cast<E *>(smem + L.BW);
  float *sRaw = reinterpret_cast<float *>(smem + L.raw);
  float *sGeoB = reinterpret_cast<float *>(smem + L.geo);
  int *sNbr = reinterpret_cast<int *>(smem + L.nbr);
  int *sTab = reinterpret_cast<int *>(smem + L.tab);
  uint64_t *mbT = reinterpret_cast<uint64_t *>(smem + L.misc);  // tile copies
  uint64_t *mbM = mbT + 1;                                      // gradient/divergence/lift MMAs
  uint64_t *mbW = mbT + 2;                                      // Vq, Pq MMAs
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbT + 3);
  int *sRed = reinterpret_cast<int *>(tslot + 1);  // [5] maxima as float bits
  int *sPend = sRed + 5;  // [6] thread 0's copies / MMAs in flight and their phases
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q4 = warp & 3, g8 = warp >> 2;  // TMEM sub-partition, element group of 8
  // single-thread issue work is spread over lane 0 of five warps, so that no
  // warp carries all of it between two barriers: gradient / divergence /
  // lift MMAs (each chain in issue order from one thread), Vq and Pq MMAs,
  // bulk copies and L2 prefetches
  constexpr int I_GRAD = 0, I_DIV = 32, I_LIFT = 64, I_WADG = 96, I_COPY = 128;

  // ---------------------------------------------------------------- setup
  if (tid == 0) {
    tc::mbar_init(mbT, 1);
    tc::mbar_init(mbM, 3);  // one commit from each of the three issuing threads
    tc::mbar_init(mbW, 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, TC_COLS);
    tc::tmem_relinquish();
  }
  for (int i = tid; i < L.ops_halfs / 8; i += TC_T)
    reinterpret_cast<uint4 *>(sOps)[i] = __ldg(reinterpret_cast<const uint4 *>(P.ops) + i);
  for (int i = tid; i < P.table_ints; i += TC_T) sTab[i] = __ldg(P.tables + i);
  for (int i = tid; i < (L.raw - L.Bp) / 16; i += TC_T)  // B operands: zero padding
    reinterpret_cast<uint4 *>(smem + L.Bp)[i] = make_uint4(0, 0, 0, 0);
  for (int i = tid; i < TC_E * RS; i += TC_T) sRaw[i] = 0.f;  // absent elements stay finite
  if (tid < 11) sRed[tid] = 0;
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  const int *sFmask = sTab;
  const int *sPat = sTab + P.pat_off;
  const int ntiles = cdv(P.K, TC_E);
  const int nvt = P.S * ntiles;
  const size_t sstride = (size_t)P.K * 4 * Np;  // floats per shot
  // TMEM address of this warp's M = 64 rows (sub-partition q4) and elements
  const uint32_t tsub = tbase + ((uint32_t)(32 * q4) << 16) + 8 * g8;
  const int rowM = 16 * q4 + ep_row(lane);  // M = 64 accumulator row of this thread
  const bool rowok = rowM < Np;

  bool fail = false;
  uint32_t tphase = 0, mphase = 0, wphase = 0;

  // I_COPY: bulk copies of a work item's inputs (state rows of its shot,
  // geometry, neighbour codes) into the raw tile and geometry buffer gb
  auto issue_tma = [&](int vt, int gb) {
    const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
    const uint32_t bytes = (uint32_t)ne * (4 * Np * 4 + TC_GEO * 4 + 16);
    tc::mbar_expect_tx(mbT, bytes);
    const float *q = P.Qin + shot * sstride + (size_t)k0 * 4 * Np;
    for (int e = 0; e < ne; ++e)
      tc::bulk_g2s(sRaw + e * RS, q + (size_t)e * 4 * Np, 4 * Np * 4, mbT);
    tc::bulk_g2s(sGeoB + gb * TC_E * TC_GEO, P.geo + (size_t)k0 * TC_GEO, ne * TC_GEO * 4, mbT);
    tc::bulk_g2s(sNbr, P.nbr + (size_t)k0 * 4, ne * 16, mbT);
    sPend[0] = 1, sPend[1] = (int)tphase;  // in flight, awaited with this parity
  };
  // I_COPY: L2 prefetch of the blocks the epilogues of a work item read
  // from global memory (old residual and state, c^2 at the cubature points)
  auto prefetch_item = [&](int vt) {
    const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
    const size_t off = shot * sstride + (size_t)k0 * 4 * Np;
    tc::prefetch_l2(P.res + off, ne * 4 * Np * 4);
    tc::prefetch_l2(P.Qin + off, ne * 4 * Np * 4);
    const uint32_t cb = (uint32_t)(ne * Nq * 4) & ~15u;
    if (cb) tc::prefetch_l2(P.c2q + (size_t)k0 * Nq, cb);
  };
  // bounded wait; the thread `owner` clears sPend[pend] on success
  auto wait_bar = [&](uint64_t *bar, uint32_t &ph, int pend, int owner) {
    const bool ok = tc::mbar_wait(bar, ph, TC_WAIT);
    if (ok && tid == owner) sPend[pend] = 0;
    fail = __any_sync(0xffffffffu, fail || !ok);
    ph ^= 1u;
    tc::fence_after_sync();
  };
  // generic smem writes -> tensor core, with the CTA-wide failure vote
  auto sync_for_mma = [&]() -> bool {
    tc::fence_proxy_async();
    tc::fence_before_sync();
    const bool any = __syncthreads_or(fail);
    tc::fence_after_sync();
    return any;
  };
  // one operator/operand product chain: D (+)= A B^T over ksteps, 3 products;
  // descriptors of consecutive K steps differ only in the start-address
  // field (+256 bytes = +16 in 16-byte units)
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
  // I_GRAD / I_DIV / I_LIFT: their part of the gradient, divergence and
  // lift products of the B1 operands, each committed to mbM
  auto issue_mma1 = [&]() {
    const uint32_t id64 = tc::idesc_f16(64, TC_E, FMT);
    const int sboV = (KV / 8) * 128, sboF = (KF / 8) * 128;
    const int pD = MR * KV, pL = MR * KF;  // plane sizes (halves)
    if (tid == I_GRAD) {
      for (int d = 0; d < 3; ++d)
        chain(tbase + cGrad + 32 * d, sOps + L.oD + 2 * d * pD, sOps + L.oD + (2 * d + 1) * pD,
              sboV, sBp, sBp + TC_E * KV, sboV, KV / 16, id64, false);
      sPend[2] = 1, sPend[3] = (int)mphase;
    } else if (tid == I_DIV) {
      for (int d = 0; d < 3; ++d)
        chain(tbase + cDiv, sOps + L.oD + 2 * d * pD, sOps + L.oD + (2 * d + 1) * pD, sboV,
              sBU + 2 * d * TC_E * KV, sBU + (2 * d + 1) * TC_E * KV, sboV, KV / 16, id64, d > 0);
    } else {
      for (int f = 0; f < 4; ++f)
        chain(tbase + cLift + 32 * f, sOps + L.oL + 2 * f * pL, sOps + L.oL + (2 * f + 1) * pL,
              sboF, sBF + 2 * f * TC_E * KF, sBF + (2 * f + 1) * TC_E * KF, sboF, KF / 16, id64,
              false);
    }
    tc::mma_commit(mbM);
  };
  auto mma1_issuer = [&]() { return tid == I_GRAD || tid == I_DIV || tid == I_LIFT; };

  // neighbour face traces of the work item in the raw tile, outside the
  // tile, into registers.  Lane = face node, warp = (element, face) pairs:
  // one load instruction reads the face of a single neighbour.
  float nbv[FPW][4];
  auto load_traces = [&](int vt) {
    const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
    const float *q = P.Qin + shot * sstride;
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
      const float *o = q + (size_t)(code >> 8) * 4 * Np + sPat[pat * Nfp + lane];
      nbv[j][0] = __ldg(o), nbv[j][1] = __ldg(o + Np), nbv[j][2] = __ldg(o + 2 * Np),
      nbv[j][3] = __ldg(o + 3 * Np);
    }
  };

  // producer: p, contravariant velocities and upwind flux of the work item
  // in the raw tile -> B operands of the first MMA group; sets the scales;
  // returns the CTA-wide failure vote
  float sp = 1.f, sU = 1.f, sF = 1.f;
  auto produce = [&](int vt, int gb) -> bool {
    const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
    (void)shot;
    const float *sGeo = sGeoB + gb * TC_E * TC_GEO;
    constexpr int NC = KV / 4;               // node chunks incl. padding
    const int ce = tid & 31, cc = tid >> 5;  // item (chunk cc, element ce); TC_T = 16 * 32
    float4 p4 = make_float4(0.f, 0.f, 0.f, 0.f), U4[3];
    U4[0] = U4[1] = U4[2] = p4;
    float mp = 0.f, mU = 0.f, mF = 0.f;
    float pf[FPW];
#pragma unroll
    for (int j = 0; j < FPW; ++j) pf[j] = 0.f;
    if (!fail) {
      if (cc < NC && 4 * cc < Np && ce < ne) {
        const float4 g0 = *reinterpret_cast<const float4 *>(sGeo + ce * TC_GEO + 16);
        const float4 g1 = *reinterpret_cast<const float4 *>(sGeo + ce * TC_GEO + 20);
        const float G[9] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w,
                            sGeo[ce * TC_GEO + 24]};
        const float *rr = sRaw + ce * RS + 4 * cc;
        float4 u4, v4, w4;
        if constexpr (C::V4) {
          p4 = *reinterpret_cast<const float4 *>(rr);
          u4 = *reinterpret_cast<const float4 *>(rr + Np);
          v4 = *reinterpret_cast<const float4 *>(rr + 2 * Np);
          w4 = *reinterpret_cast<const float4 *>(rr + 3 * Np);
        } else {  // field rows not 16-byte aligned; nodes past Np read as zero
          float a[4][4];
#pragma unroll
          for (int fl = 0; fl < 4; ++fl)
#pragma unroll
            for (int i = 0; i < 4; ++i) a[fl][i] = (4 * cc + i < Np) ? rr[fl * Np + i] : 0.f;
          p4 = make_float4(a[0][0], a[0][1], a[0][2], a[0][3]);
          u4 = make_float4(a[1][0], a[1][1], a[1][2], a[1][3]);
          v4 = make_float4(a[2][0], a[2][1], a[2][2], a[2][3]);
          w4 = make_float4(a[3][0], a[3][1], a[3][2], a[3][3]);
        }
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
      // upwind flux (Uflux = -pflux), lane = face node
#pragma unroll
      for (int j = 0; j < FPW; ++j) {
        const int pp = warp * FPW + j, e = pp >> 2, f = pp & 3;
        if (lane >= Nfp || e >= ne) continue;
        const int m = f * Nfp + lane;
        const int code = sNbr[e * 4 + f];
        const int pat = code & 255;
        const int vM = sFmask[m];
        const float *own = sRaw + e * RS + vM;
        const float pM = own[0], uM = own[Np], vvM = own[2 * Np], wM = own[3 * Np];
        const float4 fg = *reinterpret_cast<const float4 *>(sGeo + e * TC_GEO + 4 * f);
        const float Fscale = fg.x, nx = fg.y, ny = fg.z, nz = fg.w;
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
    }
    mp = warp_max(mp);
    mU = warp_max(mU);
    mF = warp_max(mF);
    if (lane == 0) {
      atomicMax(&sRed[0], __float_as_int(mp));
      atomicMax(&sRed[1], __float_as_int(mU));
      atomicMax(&sRed[2], __float_as_int(mF));
    }
    __syncthreads();  // maxima complete
    sp = pow2_scale(sRed[0]), sU = pow2_scale(sRed[1]), sF = pow2_scale(sRed[2]);
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
    return sync_for_mma();  // B1 written; the raw tile and codes no longer read
  };

  // ---------------------------------------------------------------- prologue
  int vt = blockIdx.x, it = 0;
  if (vt < nvt) {
    if (tid == I_COPY) issue_tma(vt, 0);
    wait_bar(mbT, tphase, 0, I_COPY);
    if (!fail) load_traces(vt);
    fail = produce(vt, 0) || fail;
    if (!fail) {
      if (mma1_issuer()) issue_mma1();
      if (tid == I_COPY) {
        prefetch_item(vt);
        if (vt + (int)gridDim.x < nvt) issue_tma(vt + gridDim.x, 1);
      }
    }
    if (tid < 3) sRed[tid] = 0;
  }
  float sp_cur = sp, sU_cur = sU, sF_cur = sF;  // scales of the item in acc1

  // ------------------------------------------------------------- item loop
  // (fail is CTA-uniform here; inside the loop a missed wait is acted on at
  // the next CTA-wide vote, so every thread leaves at the same point)
  if (!fail)
  for (; vt < nvt; vt += gridDim.x, ++it) {
    const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
    const int gb = it & 1;
    const int next = vt + gridDim.x, next2 = next + gridDim.x;
    const size_t sbase = shot * sstride;
    const float *sGeo = sGeoB + gb * TC_E * TC_GEO;

    // ---- a. epilogue 1 (thread = node row, four elements): rhs of u, v, w;
    //         LSRK update of u, v, w (old values from global memory, fetched
    //         before the wait); rhs_p -> B operand of the Vq product
    float ro[4][3], qo[4][3];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = 8 * g8 + ep_col(lane, j);
      const bool ok = rowok && e < ne;
      const size_t id = sbase + (size_t)(k0 + e) * 4 * Np + rowM;
#pragma unroll
      for (int fl = 1; fl < 4; ++fl) {
        ro[j][fl - 1] = ok ? P.res[id + fl * Np] : 0.f;
        qo[j][fl - 1] = ok ? __ldg(P.Qin + id + fl * Np) : 0.f;
      }
    }
    wait_bar(mbM, mphase, 2, I_GRAD);
    float rp[4] = {0.f, 0.f, 0.f, 0.f};
    if (!fail) {
      float gr[4], gs[4], gt[4], dv[4], lf[4][4];
      tc::tmem_ld16x64b_x4x4(tsub + cGrad, tsub + cGrad + 32, tsub + cGrad + 64, tsub + cDiv, gr,
                             gs, gt, dv);
      tc::tmem_ld16x64b_x4x4(tsub + cLift, tsub + cLift + 32, tsub + cLift + 64,
                             tsub + cLift + 96, lf[0], lf[1], lf[2], lf[3]);
      const float isp = 1.f / sp_cur, isU = 1.f / sU_cur, isF = 1.f / sF_cur;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int e = 8 * g8 + ep_col(lane, j);
        const float *Ge = sGeo + e * TC_GEO;
        const float4 g0 = *reinterpret_cast<const float4 *>(Ge + 16);
        const float4 g1 = *reinterpret_cast<const float4 *>(Ge + 20);
        const float g8v = Ge[24];
        const float dr = gr[j] * isp, ds = gs[j] * isp, dt = gt[j] * isp;
        float vp = -dv[j] * isU;
        float vu = -(g0.x * dr + g0.w * ds + g1.z * dt);
        float vv = -(g0.y * dr + g1.x * ds + g1.w * dt);
        float vw = -(g0.z * dr + g1.y * ds + g8v * dt);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const float a = lf[f][j] * isF;
          const float4 fn = *reinterpret_cast<const float4 *>(Ge + 4 * f);  // Fscale nx ny nz
          vp += a;
          vu -= fn.y * a;
          vv -= fn.z * a;
          vw -= fn.w * a;
        }
        const bool ok = rowok && e < ne;
        rp[j] = ok ? vp : 0.f;
        if (ok) {
          const size_t id = sbase + (size_t)(k0 + e) * 4 * Np + rowM;
          const float rv3[3] = {vu, vv, vw};
#pragma unroll
          for (int fl = 1; fl < 4; ++fl) {
            const float r = P.fa * ro[j][fl - 1] + P.fdt * rv3[fl - 1];
            P.res[id + fl * Np] = r;
            P.Qout[id + fl * Np] = qo[j][fl - 1] + P.fb * r;
          }
        }
      }
    }
    {
      float mr = fmaxf(fmaxf(fabsf(rp[0]), fabsf(rp[1])), fmaxf(fabsf(rp[2]), fabsf(rp[3])));
      mr = warp_max(mr);
      if (lane == 0) atomicMax(&sRed[3], __float_as_int(mr));
    }
    tc::fence_before_sync();
    __syncthreads();  // maxima of rhs_p; acc1 and this item's geometry no longer read
    tc::fence_after_sync();
    const float srp = pow2_scale(sRed[3]);
    if (rowM < KV) {  // rows [Np, KV) store the zero K padding
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int o = tc::kmajor_offset_f16(8 * g8 + ep_col(lane, j), rowM, KV);
        split_store1(sBW + o, sBW + TC_E * KV + o, rp[j] * srp);
      }
    }
    if (tid == 0) sRed[4] = 0;
    if (sync_for_mma()) {
      fail = true;
      break;
    }
    if (tid == I_WADG) {
      chain(tbase + cVq, sOps + L.oVq, sOps + L.oVq + MRQ * KV, (KV / 8) * 128, sBW,
            sBW + TC_E * KV, (KV / 8) * 128, KV / 16, tc::idesc_f16(MQ, TC_E, FMT), false);
      tc::mma_commit(mbW);
      sPend[4] = 1, sPend[5] = (int)wphase;
    }

    // c^2 of epilogue 2, fetched here so that its latency hides under b
    const bool q128 = MQ == 128;
    const int qrow = q128 ? 32 * q4 + lane : rowM;
    const int nq = q128 ? 8 : 4;  // elements per thread in epilogue 2
    float c2v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = 8 * g8 + (q128 ? j : ep_col(lane, j & 3));
      c2v[j] = j < nq && qrow < Nq && e < ne ? __ldg(P.c2q + (size_t)(k0 + e) * Nq + qrow) : 0.f;
    }
    // ---- b. next item: its inputs landed during this item's first MMAs;
    //         traces, flux and B operands of its first product group
    if (next < nvt) {
      wait_bar(mbT, tphase, 0, I_COPY);
      if (!fail) load_traces(next);
      if (produce(next, gb ^ 1)) {
        fail = true;
        break;
      }
    }

    // ---- c. epilogue 2 (thread = cubature row q): c2/J * p_q -> B operand of Pq
    wait_bar(mbW, wphase, 4, I_WADG);
    float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (!fail) {
      if (q128) {
        tc::tmem_ld8(tbase + ((uint32_t)(32 * q4) << 16) + cVq + 8 * g8, v);
      } else {
        float v4[4];
        tc::tmem_ld16x64b_x4(tsub + cVq, v4);
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = v4[j];
      }
    }
    const float isr = 1.f / srp;
    float mc = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float raw = v[j] * isr;
      if (P.vq_out && j < nq && qrow < Nq) {
        const int e = 8 * g8 + (q128 ? j : ep_col(lane, j));
        if (e < ne) P.vq_out[((size_t)shot * Nq + qrow) * P.K + k0 + e] = raw;
      }
      v[j] = qrow < Nq ? raw * c2v[j] : 0.f;  // rows past Nq: exact zeros
      mc = fmaxf(mc, fabsf(v[j]));
    }
    mc = warp_max(mc);
    if (lane == 0) atomicMax(&sRed[4], __float_as_int(mc));
    tc::fence_before_sync();
    __syncthreads();  // maxima; the Vq product has read its B operand in BW
    tc::fence_after_sync();
    const float sc = pow2_scale(sRed[4]);
    if (qrow < KQ) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (j >= nq) break;
        const int o = tc::kmajor_offset_f16(8 * g8 + (q128 ? j : ep_col(lane, j)), qrow, KQ);
        split_store1(sBW + o, sBW + TC_E * KQ + o, v[j] * sc);
      }
    }
    if (tid == 0) sRed[3] = 0;
    if (sync_for_mma()) {
      fail = true;
      break;
    }
    sp_cur = sp, sU_cur = sU, sF_cur = sF;  // scales of the next item's B1 operands
    if (tid < 3) sRed[tid] = 0;
    if (tid == I_WADG) {
      chain(tbase + cPq, sOps + L.oPq, sOps + L.oPq + MR * KQ, (KQ / 8) * 128, sBW,
            sBW + TC_E * KQ, (KQ / 8) * 128, KQ / 16, tc::idesc_f16(64, TC_E, FMT), false);
      tc::mma_commit(mbW);
      sPend[4] = 1, sPend[5] = (int)wphase;
    }
    if (next < nvt) {
      if (mma1_issuer()) issue_mma1();  // acc1 drained in a, B1 written in b
      if (tid == I_COPY) {
        prefetch_item(next);
        if (next2 < nvt) issue_tma(next2, gb);  // raw tile free after b, geometry gb after a
      }
    }

    // ---- d. epilogue 3: rhs_p = Pq (c2 p_q) + sources; LSRK update of p
    float r7[4], q7[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = 8 * g8 + ep_col(lane, j);
      const bool ok = rowok && e < ne;
      const size_t id = sbase + (size_t)(k0 + e) * 4 * Np + rowM;
      r7[j] = ok ? P.res[id] : 0.f;
      q7[j] = ok ? __ldg(P.Qin + id) : 0.f;
    }
    wait_bar(mbW, wphase, 4, I_WADG);
    if (!fail) {
      float w[4];
      tc::tmem_ld16x64b_x4(tsub + cPq, w);
      const float isc = 1.f / sc;
#pragma unroll
      for (int j = 0; j < 4; ++j) w[j] *= isc;
      if (P.src_off) {
        // the entries of a shot are sorted by element: find the first one of
        // this tile by bisection, then walk the tile's entries
        const int j0 = __ldg(P.src_off + shot), j1 = __ldg(P.src_off + shot + 1);
        int lo = j0, hi = j1;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (__ldg(P.src_elem + mid) < k0) lo = mid + 1;
          else hi = mid;
        }
        if (lo < j1 && __ldg(P.src_elem + lo) < k0 + ne) {
          const float amp = tc_ricker((float)(*P.time) + P.cstage * P.fdt, P.f0, P.tR, P.samp);
          for (int s = lo; s < j1; ++s) {
            const int rel = __ldg(P.src_elem + s) - k0;
            if (rel >= ne) break;
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (rowok && rel == 8 * g8 + ep_col(lane, j))
                w[j] += amp * __ldg(P.src_vec + (size_t)s * Np + rowM);
          }
        }
      }
      if (rowok) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int e = 8 * g8 + ep_col(lane, j);
          if (e >= ne) continue;
          const size_t id = sbase + (size_t)(k0 + e) * 4 * Np + rowM;
          const float r = P.fa * r7[j] + P.fdt * w[j];
          P.res[id] = r;
          P.Qout[id] = q7[j] + P.fb * r;
        }
      }
    }
  }
  // (sPend is written by the issuing threads and read after this barrier)
  if (__syncthreads_or(fail) && tid == 0) {
    // drain this CTA's own copies and MMAs still in flight (bounded), so
    // nothing lands in shared memory or TMEM after they are released; a Vq
    // or Pq product is awaited before the next one is issued, so at most
    // the last of them can still be in flight
    if (sPend[0]) tc::mbar_wait(mbT, (uint32_t)sPend[1], TC_WAIT);
    if (sPend[2]) tc::mbar_wait(mbM, (uint32_t)sPend[3], TC_WAIT);
    if (sPend[4]) tc::mbar_wait(mbW, (uint32_t)sPend[5], TC_WAIT);
    atomicAdd(P.err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, TC_COLS);
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
  // the MMAs read up to 64 - MR (MQ - MRQ) rows past an operator plane: the
  // buffers after the operators must cover the last plane's over-read
  const TcLayout &L = pl.L;
  const int over = std::max((64 - L.MR) * std::max(L.KV, std::max(L.KF, L.KQ)),
                            (L.MQ - L.MRQ) * L.KV) * 2;
  if (L.total - L.Bp < over)
    return set_error(BBW_ERR_UNSUPPORTED, "tensor-core stage: operator layout");
  // the limit is per kernel and device while the footprint depends on the
  // mesh (face-permutation table): raise it to the device maximum once
  const bbw_status s = ensure_smem_limit(k_tc_stage<N, BF>, maxsm, "tensor-core stage attribute");
  if (s != BBW_OK) return s;
  pl.nsm = nsm > 0 ? nsm : 148;
  return BBW_OK;
}

template <int N, bool BF>
static bbw_status tc_launch_n(const TcPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                              float fb, float fdt, float cstage, cudaStream_t st) {
  TcParams P;
  P.K = pl.K, P.Nq = pl.Nq, P.bc = pl.bc, P.S = std::max(pl.S, 1);
  P.fa = fa, P.fb = fb, P.fdt = fdt, P.cstage = cstage;
  P.Qin = Qin, P.Qout = Qout, P.res = res;
  P.geo = pl.geo, P.nbr = pl.nbr, P.c2q = pl.c2q;
  P.ops = pl.ops;
  P.tables = pl.tables, P.table_ints = pl.table_ints, P.pat_off = pl.pat_off;
  P.err = pl.err;
  P.src_off = pl.src_off, P.src_elem = pl.src_elem, P.src_vec = pl.src_vec;
  P.f0 = pl.f0, P.tR = pl.tR, P.samp = pl.samp, P.time = pl.time;
  P.vq_out = pl.vq_out;
  P.L = pl.L;
  const int items = cdv(pl.K, TC_E) * P.S;
  int grid = std::min(items, pl.nsm);
  if (pl.max_ctas > 0) grid = std::min(grid, pl.max_ctas);
  k_tc_stage<N, BF><<<grid, TC_T, pl.L.total, st>>>(P);
  return check_launch("tensor-core stage");
}

bool tc_supported(int N, int Nq) { return N >= 2 && N <= 5 && Nq >= 1 && Nq <= 128; }

bbw_status tc_prepare(TcPlan &pl) {
  switch (pl.N * 2 + (pl.bf ? 1 : 0)) {
    case 4: return tc_prepare_n<2, false>(pl);
    case 5: return tc_prepare_n<2, true>(pl);
    case 6: return tc_prepare_n<3, false>(pl);
    case 7: return tc_prepare_n<3, true>(pl);
    case 8: return tc_prepare_n<4, false>(pl);
    case 9: return tc_prepare_n<4, true>(pl);
    case 10: return tc_prepare_n<5, false>(pl);
    case 11: return tc_prepare_n<5, true>(pl);
  }
  return set_error(BBW_ERR_UNSUPPORTED, "tensor-core stage: N must be in [2, 5]");
}

bbw_status tc_launch(const TcPlan &pl, const float *Qin, float *Qout, float *res, float fa,
                     float fb, float fdt, float cstage, cudaStream_t st) {
  switch (pl.N * 2 + (pl.bf ? 1 : 0)) {
    case 4: return tc_launch_n<2, false>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
    case 5: return tc_launch_n<2, true>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
    case 6: return tc_launch_n<3, false>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
    case 7: return tc_launch_n<3, true>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
    case 8: return tc_launch_n<4, false>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
    case 9: return tc_launch_n<4, true>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
    case 10: return tc_launch_n<5, false>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
    case 11: return tc_launch_n<5, true>(pl, Qin, Qout, res, fa, fb, fdt, cstage, st);
  }
  return set_error(BBW_ERR_UNSUPPORTED, "tensor-core stage: N must be in [2, 5]");
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
