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
// with a grid stride.  Its 16 warps form two groups that work on different
// items at the same time and meet only through mbarriers:
//
//   producer (warps 8-15), item T+1: neighbour traces, upwind flux, p and
//     the contravariant velocities -> split B operands of the first MMA
//     group (gradient, divergence, lift); then the bulk copies of item T+2
//     and the first MMA group of T+1, issued from lane 0 of four warps
//   epilogue (warps 0-7), item T: first-group accumulators -> rhs and LSRK
//     update of u, v, w; rhs_p split -> Vq MMAs; c^2 / J at the cubature
//     points split -> Pq MMAs; rhs_p, sources, LSRK update of p
//
// Handshakes: copies landed (mbT), first group done (mbM), Vq / Pq done
// (mbW), first-group accumulators read out (mbF) and geometry buffer read
// out (mbG); the producer passes each item's B1 scales through a tagged
// shared-memory slot.  Within a group, named barriers (1: epilogue, 2:
// producer) carry the per-tile maxima of the power-of-two scaling.
//
// TMEM (512 columns): [0,96) gradient r,s,t, [96,128) divergence,
// [128,256) lift per face, [256,288) Vq, [288,320) Pq.  For M = 64 an
// accumulator row m lives in lane (m % 16) + 32 (m / 16); the epilogue reads
// those with the 16x64b shape, so all 32 threads of a warp hold a (row,
// element) pair; epilogue warp w reads sub-partition w % 4 and elements
// 16 (w / 4) .. 16 (w / 4) + 15.  The LSRK update reads the old state and
// residual from global memory (L2, prefetched one item ahead), so the state
// tile in shared memory is free for the next copies as soon as the
// producer has built its B operands.
//
// Every mbarrier wait is bounded.  A wait that gives up records the failure
// (per thread, warp-uniform where warp-collective TMEM loads follow, and in
// a shared flag); the thread skips every access that depends on the awaited
// data, its group leaves the loop at its next named-barrier vote, a waiting
// partner group runs out of its own bounded waits, and thread 0 waits
// (bounded) for the copies and MMAs still in flight before the TMEM is
// freed and the error flag is raised.
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
  // flux items with lane = face node: the 4 TC_E (element, face) pairs of
  // a tile over the 8 producer warps, in two halves of FPW pairs each
  static constexpr int FPW = (4 * TC_E) / 16;
  static_assert((4 * TC_E) % 16 == 0, "face pairs per producer warp and half");
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
  o = al(o + 256);
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
  // sources: entries j in [src_tile[vt], src_tile[vt+1]) of work item vt
  // (entries sorted by shot and element) add ricker(t) * src_vec[j][:] to
  // the projected rhs_p of element src_elem[j], t = *time + cstage * fdt (as
  // the FP32 fused stage)
  const int *__restrict__ src_tile;
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

__device__ __forceinline__ void mbar_arrive1(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(tc::smem_u32(mbar)) : "memory");
}
// group barriers: the epilogue warps (0-7) use named barrier 1, the
// producer warps (8-15) barrier 2 (__syncthreads keeps barrier 0); each
// is a barrier with an OR vote over the group's 256 threads
__device__ __forceinline__ bool group_sync_or(int id, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, %2, 256, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id)
      : "memory");
  return r != 0;
}

template <int N, bool BF>
__global__ void __launch_bounds__(TC_T, 1) k_tc_stage(TcParams P) {
  // operand type; A and B of every MMA share it (the instruction descriptor
  // sets both formats from FMT)
  using E = typename std::conditional<BF, __nv_bfloat16, __half>::type;
  constexpr int FMT = BF ? 1 : 0;
  using C = TcCfg<N>;
  constexpr int Np = C::Np, Nfp = C::Nfp, KV = C::KV, KF = C::KF, RS = C::RS;
  constexpr int FPW = C::FPW;  // flux items per producer warp and half
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
  uint64_t *mbT = reinterpret_cast<uint64_t *>(smem + L.misc);  // tile copies landed
  uint64_t *mbM = mbT + 1;  // gradient/divergence/lift MMAs done (3 commits)
  uint64_t *mbW = mbT + 2;  // Vq / Pq MMAs done
  uint64_t *mbF = mbT + 3;  // first-group accumulators read out (8 epilogue warps)
  uint64_t *mbG = mbT + 4;  // geometry buffer read out (8 epilogue warps)
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbT + 5);
  int *sRed = reinterpret_cast<int *>(tslot + 1);  // [10] maxima as float bits
  int *sPend = sRed + 10;                          // [6] copies / MMAs in flight, phases
  volatile int *sFail = sPend + 6;                 // any wait gave up
  volatile int *sTag = sFail + 1;                  // [2] tile of the scales in slot
  float *sScale = reinterpret_cast<float *>(sPend + 9);  // [2][3] B1 scales per slot
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool isEpi = warp < 8;
  // epilogue warps: TMEM sub-partition q4, element half eh (columns 16 eh ..)
  const int q4 = warp & 3, eh = (warp >> 2) & 1;
  const int ptid = tid - 256;  // producer thread index (0..255)
  // single-thread issuers: first-group MMA chains on lane 0 of producer
  // warps 8, 9, 10, bulk copies on warp 11; Vq / Pq on epilogue warp 0
  constexpr int I_GRAD = 256, I_DIV = 288, I_LIFT = 320, I_COPY = 352, I_WADG = 0;

  // ---------------------------------------------------------------- setup
  if (tid == 0) {
    tc::mbar_init(mbT, 1);
    tc::mbar_init(mbM, 3);
    tc::mbar_init(mbW, 1);
    tc::mbar_init(mbF, 8);
    tc::mbar_init(mbG, 8);
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
  if (tid < 10) sRed[tid] = 0;
  if (tid < 6) sPend[tid] = 0;
  if (tid == 0) *sFail = 0, sTag[0] = sTag[1] = -1;
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
  bool fail = false;

  // bounded wait of one thread; a miss is recorded for the group votes
  auto wait1 = [&](uint64_t *bar, uint32_t parity) -> bool {
    const bool ok = tc::mbar_wait(bar, parity, TC_WAIT);
    if (!ok) fail = true, *sFail = 1;
    tc::fence_after_sync();
    return ok;
  };
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

  if (!isEpi) {
    // ============================================================ producer
    // per work item: neighbour traces, upwind flux, p and contravariant
    // velocities -> split B operands of the first MMA group; then the bulk
    // copies of the next item and the first MMA group of this one
    const int pw = warp - 8;
    auto issue_tma = [&](int vt, int gb, uint32_t ph) {
      const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
      const uint32_t bytes = (uint32_t)ne * (4 * Np * 4 + TC_GEO * 4 + 16);
      tc::mbar_expect_tx(mbT, bytes);
      const float *q = P.Qin + shot * sstride + (size_t)k0 * 4 * Np;
      for (int e = 0; e < ne; ++e)
        tc::bulk_g2s(sRaw + e * RS, q + (size_t)e * 4 * Np, 4 * Np * 4, mbT);
      tc::bulk_g2s(sGeoB + gb * TC_E * TC_GEO, P.geo + (size_t)k0 * TC_GEO, ne * TC_GEO * 4, mbT);
      tc::bulk_g2s(sNbr, P.nbr + (size_t)k0 * 4, ne * 16, mbT);
      sPend[0] = 1, sPend[1] = (int)ph;
    };
    auto prefetch_item = [&](int vt) {
      const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
      const size_t off = shot * sstride + (size_t)k0 * 4 * Np;
      tc::prefetch_l2(P.res + off, ne * 4 * Np * 4);
      tc::prefetch_l2(P.Qin + off, ne * 4 * Np * 4);
      const uint32_t cb = (uint32_t)(ne * Nq * 4) & ~15u;
      if (cb) tc::prefetch_l2(P.c2q + (size_t)k0 * Nq, cb);
    };
    // L2 prefetch of the blocks a later item's bulk copies read, one item
    // ahead of them (the copies of an item are issued only once the raw
    // tile is free, just before the item is needed)
    auto prefetch_copies = [&](int vt) {
      const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
      tc::prefetch_l2(P.Qin + shot * sstride + (size_t)k0 * 4 * Np, ne * 4 * Np * 4);
      tc::prefetch_l2(P.geo + (size_t)k0 * TC_GEO, ne * TC_GEO * 4);
      tc::prefetch_l2(P.nbr + (size_t)k0 * 4, ne * 16);
    };
    if (ptid == I_COPY - 256 && (int)blockIdx.x < nvt) {
      issue_tma(blockIdx.x, 0, 0);
      prefetch_item(blockIdx.x);
      if ((int)(blockIdx.x + gridDim.x) < nvt) prefetch_copies(blockIdx.x + gridDim.x);
    }
    int it = 0;
    for (int vt = blockIdx.x; vt < nvt; vt += gridDim.x, ++it) {
      const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
      const int gb = it & 1, next = vt + gridDim.x;
      const float *sGeo = sGeoB + gb * TC_E * TC_GEO;
      const float *qs = P.Qin + shot * sstride;
      // the item's copies
      {
        const bool ok = tc::mbar_wait(mbT, (uint32_t)(it & 1), TC_WAIT);
        if (!ok) fail = true, *sFail = 1;
        else if (ptid == I_COPY - 256) sPend[0] = 0;
        tc::fence_after_sync();
      }
      // state part: item (chunk cc, element ce), two per thread
      constexpr int NC = KV / 4;
      float4 p4[2], U4[2][3];
      float mp = 0.f, mU = 0.f, mF = 0.f;
      float pf[2 * FPW];
#pragma unroll
      for (int j = 0; j < 2 * FPW; ++j) pf[j] = 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        p4[h] = make_float4(0.f, 0.f, 0.f, 0.f);
        U4[h][0] = U4[h][1] = U4[h][2] = p4[h];
      }
      if (!fail) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int item = ptid + 256 * h, ce = item & 31, cc = item >> 5;
          if (cc < NC && 4 * cc < Np && ce < ne) {
            const float4 g0 = *reinterpret_cast<const float4 *>(sGeo + ce * TC_GEO + 16);
            const float4 g1 = *reinterpret_cast<const float4 *>(sGeo + ce * TC_GEO + 20);
            const float G[9] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w,
                                sGeo[ce * TC_GEO + 24]};
            const float *rr = sRaw + ce * RS + 4 * cc;
            float4 u4, v4, w4;
            if constexpr (C::V4) {
              p4[h] = *reinterpret_cast<const float4 *>(rr);
              u4 = *reinterpret_cast<const float4 *>(rr + Np);
              v4 = *reinterpret_cast<const float4 *>(rr + 2 * Np);
              w4 = *reinterpret_cast<const float4 *>(rr + 3 * Np);
            } else {
              float a[4][4];
#pragma unroll
              for (int fl = 0; fl < 4; ++fl)
#pragma unroll
                for (int i = 0; i < 4; ++i) a[fl][i] = (4 * cc + i < Np) ? rr[fl * Np + i] : 0.f;
              p4[h] = make_float4(a[0][0], a[0][1], a[0][2], a[0][3]);
              u4 = make_float4(a[1][0], a[1][1], a[1][2], a[1][3]);
              v4 = make_float4(a[2][0], a[2][1], a[2][2], a[2][3]);
              w4 = make_float4(a[3][0], a[3][1], a[3][2], a[3][3]);
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              float4 &U = U4[h][d];
              U.x = u4.x * G[3 * d] + v4.x * G[3 * d + 1] + w4.x * G[3 * d + 2];
              U.y = u4.y * G[3 * d] + v4.y * G[3 * d + 1] + w4.y * G[3 * d + 2];
              U.z = u4.z * G[3 * d] + v4.z * G[3 * d + 1] + w4.z * G[3 * d + 2];
              U.w = u4.w * G[3 * d] + v4.w * G[3 * d + 1] + w4.w * G[3 * d + 2];
              mU = fmaxf(mU, fmaxf(fmaxf(fabsf(U.x), fabsf(U.y)), fmaxf(fabsf(U.z), fabsf(U.w))));
            }
            mp = fmaxf(mp, fmaxf(fmaxf(fabsf(p4[h].x), fabsf(p4[h].y)),
                                 fmaxf(fabsf(p4[h].z), fabsf(p4[h].w))));
          }
        }
        // upwind flux (Uflux = -pflux), lane = face node; warp pw owns the
        // (element, face) pairs 16 pw .. 16 pw + 15, in two halves whose
        // outside-tile neighbour traces are fetched together
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float nbv[FPW][4];
#pragma unroll
          for (int j = 0; j < FPW; ++j) {
            nbv[j][0] = nbv[j][1] = nbv[j][2] = nbv[j][3] = 0.f;
            const int pp = pw * 2 * FPW + h * FPW + j, e = pp >> 2, f = pp & 3;
            if (lane >= Nfp || e >= ne) continue;
            const int code = sNbr[e * 4 + f];
            const int pat = code & 255;
            if (pat == 255) continue;
            const unsigned rel = (unsigned)((code >> 8) - k0);
            if (rel < (unsigned)ne) continue;
            const float *o = qs + (size_t)(code >> 8) * 4 * Np + sPat[pat * Nfp + lane];
            nbv[j][0] = __ldg(o), nbv[j][1] = __ldg(o + Np), nbv[j][2] = __ldg(o + 2 * Np),
            nbv[j][3] = __ldg(o + 3 * Np);
          }
#pragma unroll
          for (int j = 0; j < FPW; ++j) {
            const int pp = pw * 2 * FPW + h * FPW + j, e = pp >> 2, f = pp & 3;
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
              if (rel < (unsigned)ne) {
                const float *o = sRaw + rel * RS + sPat[pat * Nfp + lane];
                pP = o[0], uP = o[Np], vP_ = o[2 * Np], wP = o[3 * Np];
              }
              pjump = pP - pM;
              Unjump = (uP - uM) * nx + (vP_ - vvM) * ny + (wP - wM) * nz;
            }
            pf[h * FPW + j] = .5f * (pjump - Unjump) * Fscale;
            mF = fmaxf(mF, fabsf(pf[h * FPW + j]));
          }
        }
      }
      const int rs = 3 * (it & 1);  // maxima slot set of this item
      mp = warp_max(mp);
      mU = warp_max(mU);
      mF = warp_max(mF);
      if (lane == 0) {
        atomicMax(&sRed[rs], __float_as_int(mp));
        atomicMax(&sRed[rs + 1], __float_as_int(mU));
        atomicMax(&sRed[rs + 2], __float_as_int(mF));
      }
      if (group_sync_or(2, fail || *sFail)) break;  // maxima complete
      const float sp = pow2_scale(sRed[rs]), sU = pow2_scale(sRed[rs + 1]),
                  sF = pow2_scale(sRed[rs + 2]);
      if (ptid < 3) sRed[3 - rs + ptid] = 0;  // the other set: read one item ago
      if (ptid == 0) {  // scales of this item's B1 for the epilogue warps
        float *sc = sScale + 3 * (it & 1);
        sc[0] = sp, sc[1] = sU, sc[2] = sF;
        __threadfence_block();
        sTag[it & 1] = it;
      }
      // B1 is free once the previous item's first MMA group has read it
      if (it > 0) {
        const bool ok = tc::mbar_wait(mbM, (uint32_t)((it - 1) & 1), TC_WAIT);
        if (!ok) fail = true, *sFail = 1;
      }
      if (!fail) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int item = ptid + 256 * h, ce = item & 31, cc = item >> 5;
          if (cc < NC) {
            const int o = tc::kmajor_offset_f16(ce, 4 * cc, KV);
            split_store4(sBp + o, sBp + TC_E * KV + o, p4[h], sp);
#pragma unroll
            for (int d = 0; d < 3; ++d)
              split_store4(sBU + 2 * d * TC_E * KV + o, sBU + (2 * d + 1) * TC_E * KV + o,
                           U4[h][d], sU);
          }
        }
#pragma unroll
        for (int j = 0; j < 2 * FPW; ++j) {
          const int pp = pw * 2 * FPW + j, e = pp >> 2, f = pp & 3;
          if (lane >= Nfp) continue;  // absent elements store zeros (pf = 0)
          const int o = tc::kmajor_offset_f16(e, lane, KF);
          split_store1(sBF + 2 * f * TC_E * KF + o, sBF + (2 * f + 1) * TC_E * KF + o,
                       pf[j] * sF);
        }
      }
      tc::fence_proxy_async();
      tc::fence_before_sync();
      if (group_sync_or(2, fail || *sFail)) break;  // B1 written; raw tile and codes free
      tc::fence_after_sync();
      if (ptid == I_COPY - 256) {
        if (next < nvt) {
          // the geometry buffer of the next item was read by the epilogue
          // of the item before this one
          const bool ok = it == 0 || wait1(mbG, (uint32_t)((it - 1) & 1));
          if (ok) {
            issue_tma(next, gb ^ 1, (uint32_t)((it + 1) & 1));
            prefetch_item(next);
            if (next + (int)gridDim.x < nvt) prefetch_copies(next + gridDim.x);
          }
        }
      } else if (ptid == I_GRAD - 256 || ptid == I_DIV - 256 || ptid == I_LIFT - 256) {
        // the accumulators of the previous item have been read out
        const bool ok = it == 0 || wait1(mbF, (uint32_t)((it - 1) & 1));
        if (ok) {
          const uint32_t id64 = tc::idesc_f16(64, TC_E, FMT);
          const int sboV = (KV / 8) * 128, sboF = (KF / 8) * 128;
          const int pD = MR * KV, pL = MR * KF;
          if (ptid == I_GRAD - 256) {
            for (int d = 0; d < 3; ++d)
              chain(tbase + cGrad + 32 * d, sOps + L.oD + 2 * d * pD,
                    sOps + L.oD + (2 * d + 1) * pD, sboV, sBp, sBp + TC_E * KV, sboV, KV / 16,
                    id64, false);
            sPend[2] = 1, sPend[3] = it & 1;
          } else if (ptid == I_DIV - 256) {
            for (int d = 0; d < 3; ++d)
              chain(tbase + cDiv, sOps + L.oD + 2 * d * pD, sOps + L.oD + (2 * d + 1) * pD, sboV,
                    sBU + 2 * d * TC_E * KV, sBU + (2 * d + 1) * TC_E * KV, sboV, KV / 16, id64,
                    d > 0);
          } else {
            for (int f = 0; f < 4; ++f)
              chain(tbase + cLift + 32 * f, sOps + L.oL + 2 * f * pL,
                    sOps + L.oL + (2 * f + 1) * pL, sboF, sBF + 2 * f * TC_E * KF,
                    sBF + (2 * f + 1) * TC_E * KF, sboF, KF / 16, id64, false);
          }
          tc::mma_commit(mbM);
        }
      }
    }
  } else {
    // ============================================================ epilogue
    // per work item, thread = node row x 8 elements (two groups of four):
    //   1. first-group accumulators -> rhs of u, v, w, their LSRK update;
    //      rhs_p split -> Vq MMAs
    //   2. c^2 / J * (Vq rhs_p) split -> Pq MMAs
    //   3. rhs_p = Pq (...) + sources, LSRK update of p
    const uint32_t tq = tbase + ((uint32_t)(32 * q4) << 16);
    const int rowM = 16 * q4 + ep_row(lane);
    const bool rowok = rowM < Np;
    const bool q128 = MQ == 128;
    const int qrow = q128 ? 32 * q4 + lane : rowM;
    float *sVo = reinterpret_cast<float *>(sBW);  // vq_out staging, [Nq][TC_E]
    uint32_t wphase = 0;
    int it = 0;
    for (int vt = blockIdx.x; vt < nvt; vt += gridDim.x, ++it) {
      const int shot = vt / ntiles, k0 = (vt - shot * ntiles) * TC_E, ne = min(TC_E, P.K - k0);
      const int gb = it & 1;
      const size_t sbase = shot * sstride;
      const float *sGeo = sGeoB + gb * TC_E * TC_GEO;
      const int rs = 6 + 2 * (it & 1);  // maxima slot set of this item
      // the item's source entries [src_lo, src_hi), fetched here and used
      // in epilogue 3
      int src_lo = 0, src_hi = 0;
      if (P.src_tile) src_lo = __ldg(P.src_tile + vt), src_hi = __ldg(P.src_tile + vt + 1);
      // ---- 1. first group
      float rp[2][4];
      // old u, v, w and their residual, fetched before the wait
      float ro[2][4][3], qo[2][4][3];
#pragma unroll
      for (int hh = 0; hh < 2; ++hh)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int e = 8 * (2 * eh + hh) + ep_col(lane, j);
          const bool ok = rowok && e < ne && !fail;
          const size_t id = sbase + (size_t)(k0 + e) * 4 * Np + rowM;
#pragma unroll
          for (int fl = 1; fl < 4; ++fl) {
            ro[hh][j][fl - 1] = ok ? P.res[id + fl * Np] : 0.f;
            qo[hh][j][fl - 1] = ok ? __ldg(P.Qin + id + fl * Np) : 0.f;
          }
        }
      {
        const bool ok = tc::mbar_wait(mbM, (uint32_t)(it & 1), TC_WAIT);
        if (!ok) fail = true, *sFail = 1;
        else if (tid == 0) sPend[2] = 0;
        fail = __any_sync(0xffffffffu, fail);  // the TMEM loads are warp-collective
        tc::fence_after_sync();
      }
      float isp = 1.f, isU = 1.f, isF = 1.f;
      if (!fail) {
        // the producer wrote this item's scales before its MMAs were issued
        uint32_t n = 0;
        while (sTag[it & 1] != it && ++n < TC_WAIT) {
        }
        if (sTag[it & 1] != it) fail = true, *sFail = 1;
        __threadfence_block();
      }
      fail = __any_sync(0xffffffffu, fail);
      if (!fail) {
        const float *sc = sScale + 3 * (it & 1);
        isp = 1.f / sc[0], isU = 1.f / sc[1], isF = 1.f / sc[2];
      }
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int g8 = 2 * eh + hh;
        const uint32_t tsub = tq + 8 * g8;
        float gr[4], gs[4], gt[4], dv[4], lf[4][4];
        if (!fail) {
          tc::tmem_ld16x64b_x4x4(tsub + cGrad, tsub + cGrad + 32, tsub + cGrad + 64, tsub + cDiv,
                                 gr, gs, gt, dv);
          tc::tmem_ld16x64b_x4x4(tsub + cLift, tsub + cLift + 32, tsub + cLift + 64,
                                 tsub + cLift + 96, lf[0], lf[1], lf[2], lf[3]);
        }
        if (hh == 1) {  // both halves read: the first group's accumulators are free
          tc::fence_before_sync();
          __syncwarp();
          if (lane == 0) mbar_arrive1(mbF);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          rp[hh][j] = 0.f;
          if (fail) continue;
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
            const float4 fn = *reinterpret_cast<const float4 *>(Ge + 4 * f);
            vp += a;
            vu -= fn.y * a;
            vv -= fn.z * a;
            vw -= fn.w * a;
          }
          const bool ok = rowok && e < ne;
          rp[hh][j] = ok ? vp : 0.f;
          if (ok) {
            const size_t id = sbase + (size_t)(k0 + e) * 4 * Np + rowM;
            const float rv3[3] = {vu, vv, vw};
#pragma unroll
            for (int fl = 1; fl < 4; ++fl) {
              const float r = P.fa * ro[hh][j][fl - 1] + P.fdt * rv3[fl - 1];
              P.res[id + fl * Np] = r;
              P.Qout[id + fl * Np] = qo[hh][j][fl - 1] + P.fb * r;
            }
          }
        }
      }
      // this item's geometry has been read
      __syncwarp();
      if (lane == 0) mbar_arrive1(mbG);
      {
        float mr = 0.f;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh)
          mr = fmaxf(mr, fmaxf(fmaxf(fabsf(rp[hh][0]), fabsf(rp[hh][1])),
                               fmaxf(fabsf(rp[hh][2]), fabsf(rp[hh][3]))));
        mr = warp_max(mr);
        if (lane == 0) atomicMax(&sRed[rs], __float_as_int(mr));
      }
      if (group_sync_or(1, fail || *sFail)) break;  // maxima of rhs_p
      const float srp = pow2_scale(sRed[rs]);
      if (tid < 2) sRed[14 - rs + tid] = 0;  // the other set: read one item ago
      if (rowM < KV) {  // rows [Np, KV) store the zero K padding
#pragma unroll
        for (int hh = 0; hh < 2; ++hh)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int o = tc::kmajor_offset_f16(8 * (2 * eh + hh) + ep_col(lane, j), rowM, KV);
            split_store1(sBW + o, sBW + TC_E * KV + o, rp[hh][j] * srp);
          }
      }
      tc::fence_proxy_async();
      tc::fence_before_sync();
      if (group_sync_or(1, fail || *sFail)) break;
      tc::fence_after_sync();
      if (tid == I_WADG) {
        chain(tbase + cVq, sOps + L.oVq, sOps + L.oVq + MRQ * KV, (KV / 8) * 128, sBW,
              sBW + TC_E * KV, (KV / 8) * 128, KV / 16, tc::idesc_f16(MQ, TC_E, FMT), false);
        tc::mma_commit(mbW);
        sPend[4] = 1, sPend[5] = (int)wphase;
      }
      // ---- 2. c^2 / J at the cubature points; c2 fetched under the Vq MMAs
      const int nq = q128 ? 8 : 4;  // elements per thread and group of eight
      float v[2][8];
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int g8 = 2 * eh + hh;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int e = 8 * g8 + (q128 ? j : ep_col(lane, j & 3));
          v[hh][j] = j < nq && qrow < Nq && e < ne ? __ldg(P.c2q + (size_t)(k0 + e) * Nq + qrow)
                                                   : 0.f;
        }
      }
      {
        const bool ok = tc::mbar_wait(mbW, wphase, TC_WAIT);
        if (!ok) fail = true, *sFail = 1;
        else if (tid == I_WADG) sPend[4] = 0;
        wphase ^= 1u;
        fail = __any_sync(0xffffffffu, fail);
        tc::fence_after_sync();
      }
      const float isr = 1.f / srp;
      float mc = 0.f;
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int g8 = 2 * eh + hh;
        float a[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (!fail) {
          if (q128) {
            tc::tmem_ld8(tq + cVq + 8 * g8, a);
          } else {
            float a4[4];
            tc::tmem_ld16x64b_x4(tq + 8 * g8 + cVq, a4);
#pragma unroll
            for (int j = 0; j < 4; ++j) a[j] = a4[j];
          }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float raw = a[j] * isr;
          if (P.vq_out && j < nq && qrow < Nq && !fail) {
            // staged in BW (the Vq product has read it) as [q][element],
            // elements XOR-swizzled by the row against bank conflicts
            const int e = 8 * g8 + (q128 ? j : ep_col(lane, j));
            sVo[qrow * TC_E + (e ^ (qrow & 31))] = raw;
          }
          v[hh][j] = qrow < Nq ? raw * v[hh][j] : 0.f;  // rows past Nq: exact zeros
          mc = fmaxf(mc, fabsf(v[hh][j]));
        }
      }
      mc = warp_max(mc);
      if (lane == 0) atomicMax(&sRed[rs + 1], __float_as_int(mc));
      // the residual and state of p, fetched under the Pq MMAs
      float r7[2][4], q7[2][4];
      tc::fence_before_sync();
      if (group_sync_or(1, fail || *sFail)) break;  // maxima; Vq has read BW
      tc::fence_after_sync();
      if (P.vq_out) {
        // the staged pre-c2 cubature values, one row of the tile's elements
        // per warp store
        if (!fail)
          for (int q = warp; q < Nq; q += 8)
            if (lane < ne) P.vq_out[((size_t)shot * Nq + q) * P.K + k0 + lane] =
                sVo[q * TC_E + (lane ^ (q & 31))];
        if (group_sync_or(1, fail || *sFail)) break;  // staging read before BW is rewritten
      }
      const float sc = pow2_scale(sRed[rs + 1]);
      if (qrow < KQ) {
#pragma unroll
        for (int hh = 0; hh < 2; ++hh)
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (j >= nq) break;
            const int o = tc::kmajor_offset_f16(8 * (2 * eh + hh) + (q128 ? j : ep_col(lane, j)),
                                                qrow, KQ);
            split_store1(sBW + o, sBW + TC_E * KQ + o, v[hh][j] * sc);
          }
      }
      tc::fence_proxy_async();
      tc::fence_before_sync();
      if (group_sync_or(1, fail || *sFail)) break;
      tc::fence_after_sync();
      if (tid == I_WADG) {
        chain(tbase + cPq, sOps + L.oPq, sOps + L.oPq + MR * KQ, (KQ / 8) * 128, sBW,
              sBW + TC_E * KQ, (KQ / 8) * 128, KQ / 16, tc::idesc_f16(64, TC_E, FMT), false);
        tc::mma_commit(mbW);
        sPend[4] = 1, sPend[5] = (int)wphase;
      }
      // ---- 3. rhs_p = Pq (c2 p_q) + sources; LSRK update of p
#pragma unroll
      for (int hh = 0; hh < 2; ++hh)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int e = 8 * (2 * eh + hh) + ep_col(lane, j);
          const bool ok = rowok && e < ne;
          const size_t id = sbase + (size_t)(k0 + e) * 4 * Np + rowM;
          r7[hh][j] = ok ? P.res[id] : 0.f;
          q7[hh][j] = ok ? __ldg(P.Qin + id) : 0.f;
        }
      {
        const bool ok = tc::mbar_wait(mbW, wphase, TC_WAIT);
        if (!ok) fail = true, *sFail = 1;
        else if (tid == I_WADG) sPend[4] = 0;
        wphase ^= 1u;
        fail = __any_sync(0xffffffffu, fail);
        tc::fence_after_sync();
      }
      if (!fail) {
        const float isc = 1.f / sc;
        const float amp = src_lo < src_hi
                              ? tc_ricker((float)(*P.time) + P.cstage * P.fdt, P.f0, P.tR, P.samp)
                              : 0.f;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const int g8 = 2 * eh + hh;
          float w[4];
          tc::tmem_ld16x64b_x4(tq + 8 * g8 + cPq, w);
#pragma unroll
          for (int j = 0; j < 4; ++j) w[j] *= isc;
          for (int s = src_lo; s < src_hi; ++s) {
            const int rel = __ldg(P.src_elem + s) - k0;
            if (rel >= ne) break;
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (rowok && rel == 8 * g8 + ep_col(lane, j))
                w[j] += amp * __ldg(P.src_vec + (size_t)s * Np + rowM);
          }
          if (rowok) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int e = 8 * g8 + ep_col(lane, j);
              if (e >= ne) continue;
              const size_t id = sbase + (size_t)(k0 + e) * 4 * Np + rowM;
              const float r = P.fa * r7[hh][j] + P.fdt * w[j];
              P.res[id] = r;
              P.Qout[id] = q7[hh][j] + P.fb * r;
            }
          }
        }
      }
    }
  }
  // (sPend is written by the issuing threads and read after this barrier)
  if (__syncthreads_or(fail || *sFail) && tid == 0) {
    // drain this CTA's own copies and MMAs still in flight (bounded), so
    // nothing lands in shared memory or TMEM after they are released
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
  P.src_tile = pl.src_tile, P.src_elem = pl.src_elem, P.src_vec = pl.src_vec;
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
