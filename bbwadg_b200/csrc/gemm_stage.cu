// Precision-study form of the LSRK stage: the dense contractions of the
// stage (Dr/Ds/Dt gradient and divergence, LIFT per face, Vq, Pq) over all
// elements as plain cuBLAS GEMMs, the rest in the kernels of this file.
//
// The contractions are those of the reference's rk_volume, rk_surface and
// rk_update_WADG (cpp/okl/WaveKernels.okl:122-135, 235-247,
// cpp/okl/WaveKernelsWADG.okl:1810-1817, 1847-1856); the element operands
// are [rows x K] column-major matrices (column = element), so each
// contraction is one GEMM of the operator with all elements at once.
// Arithmetic:
//   F16X3 / BF16X3: operator and operand split into hi + lo pairs of the
//     16-bit type, A x = A_hi x_hi + A_hi x_lo + A_lo x_hi as three GEMMs
//     accumulating in FP32, each element column scaled by its own power of
//     two before the split (the fused tensor-core stage scales per tile);
//   TF32: one GEMM per contraction on the FP32 operands with TF32 inputs and
//     FP32 accumulation.
// Fluxes, geometric factors, the c^2 / J multiply and the LSRK update stay
// FP32.  One CUDA block per element in the element kernels.  This form
// serves orders whose operators do not fit one SM's shared memory beside an
// element tile (N >= 6 for the fused tensor-core stage) and the TF32 rows
// of the precision study; its speed is that of separate launches over HBM
// intermediates.
#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "bbwadg.h"
#include "device_common.cuh"
#include "gemm_stage.h"
#include "internal.h"

namespace bbw {

namespace {

constexpr int GS_T = 128;  // threads per element block
constexpr int GS_MAXNP = 165, GS_MAXNF = 4 * 45, GS_MAXNQ = 1024;

// s = 2^-E with max = m 2^E, m in [0.5, 1): max * s < 1, E clamped to
// [-100, 100] (exponent-field arithmetic, as the fused tensor-core stage)
__device__ __forceinline__ float gs_pow2_scale(float mx) {
  const int bits = __float_as_int(mx);
  const int field = (bits >> 23) & 255;
  if (!(mx > 0.f) || field == 255) return 1.f;
  const int E = max(-100, min(100, field - 126));
  return __int_as_float((127 - E) << 23);
}

// operand type traits: split x into hi + lo of T (T = float: TF32 operands,
// x itself and no lo plane)
template <class T> struct Split;
template <> struct Split<__half> {
  static constexpr bool split = true;
  __device__ static void store(__half *hi, __half *lo, size_t i, float x) {
    const __half h = __float2half_rn(x);
    hi[i] = h;
    lo[i] = __float2half_rn(x - __half2float(h));
  }
};
template <> struct Split<__nv_bfloat16> {
  static constexpr bool split = true;
  __device__ static void store(__nv_bfloat16 *hi, __nv_bfloat16 *lo, size_t i, float x) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    hi[i] = h;
    lo[i] = __float2bfloat16_rn(x - __bfloat162float(h));
  }
};
template <> struct Split<float> {
  static constexpr bool split = false;
  __device__ static void store(float *hi, float *, size_t i, float x) { hi[i] = x; }
};

// block-wide maximum of three values (GS_T threads)
__device__ __forceinline__ void block_max3(float &a, float &b, float &c, float *red) {
  for (int o = 16; o > 0; o >>= 1) {
    a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
    b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o));
    c = fmaxf(c, __shfl_xor_sync(0xffffffffu, c, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) red[3 * w] = a, red[3 * w + 1] = b, red[3 * w + 2] = c;
  __syncthreads();
  a = b = c = 0.f;
  for (int i = 0; i < GS_T / 32; ++i)
    a = fmaxf(a, red[3 * i]), b = fmaxf(b, red[3 * i + 1]), c = fmaxf(c, red[3 * i + 2]);
  __syncthreads();
}

struct GsArgs {
  int K, Np, Nfp, Nq, bc, pat_off;
  float fa, fb, fdt;
  const float *Qin;
  float *Qout, *res;
  const float *vgeo, *fgeo, *c2q;
  const int *nbr, *tables;
  void *Bp[2], *BU[3][2], *BF[2], *BR[2], *BC[2];
  const float *G[3], *Div, *Lf[4], *W, *Z;
  float *scale;
};

// per element: p and the contravariant velocities U_d = G_d . (u, v, w),
// the upwind pressure flux at the 4 Nfp face nodes (Uflux = -pflux,
// cpp/okl/WaveKernels.okl:209-216), each scaled by the element's power of
// two and split into the B operands
template <class T>
__global__ void __launch_bounds__(GS_T) k_gs_prep(GsArgs a) {
  __shared__ float sq[4 * GS_MAXNP], su[3 * GS_MAXNP], sf[GS_MAXNF], red[3 * GS_T / 32];
  const int k = blockIdx.x, Np = a.Np, Nfp = a.Nfp, NF = 4 * Nfp;
  const float *q = a.Qin + (size_t)k * 4 * Np;
  for (int i = threadIdx.x; i < 4 * Np; i += GS_T) sq[i] = q[i];
  __syncthreads();
  const float *G = a.vgeo + (size_t)k * 9;  // rx ry rz sx sy sz tx ty tz
  float mp = 0.f, mU = 0.f, mF = 0.f;
  for (int n = threadIdx.x; n < Np; n += GS_T) {
    const float u = sq[Np + n], v = sq[2 * Np + n], w = sq[3 * Np + n];
    for (int d = 0; d < 3; ++d) {
      const float U = u * G[3 * d] + v * G[3 * d + 1] + w * G[3 * d + 2];
      su[d * Np + n] = U;
      mU = fmaxf(mU, fabsf(U));
    }
    mp = fmaxf(mp, fabsf(sq[n]));
  }
  const int *Fmask = a.tables, *pats = a.tables + a.pat_off;
  for (int m = threadIdx.x; m < NF; m += GS_T) {
    const int f = m / Nfp, i = m - f * Nfp;
    const int code = a.nbr[(size_t)k * 4 + f], pat = code & 255;
    const int vM = Fmask[m];
    const float pM = sq[vM], uM = sq[Np + vM], vvM = sq[2 * Np + vM], wM = sq[3 * Np + vM];
    const float *fg = a.fgeo + (size_t)k * 16 + 4 * f;  // Fscale nx ny nz
    const float nx = fg[1], ny = fg[2], nz = fg[3];
    float pjump, Unjump;
    if (pat == 255) {
      if (a.bc == BBW_BC_PRESSURE_RELEASE) {
        pjump = -2.f * pM;
        Unjump = 0.f;
      } else {
        pjump = 0.f;
        Unjump = -2.f * (uM * nx + vvM * ny + wM * nz);
      }
    } else {
      const float *o = a.Qin + (size_t)(code >> 8) * 4 * Np + pats[pat * Nfp + i];
      pjump = o[0] - pM;
      Unjump = (o[Np] - uM) * nx + (o[2 * Np] - vvM) * ny + (o[3 * Np] - wM) * nz;
    }
    const float pf = .5f * (pjump - Unjump) * fg[0];
    sf[m] = pf;
    mF = fmaxf(mF, fabsf(pf));
  }
  block_max3(mp, mU, mF, red);  // also orders the su / sf writes before the reads below
  const bool sp_ = Split<T>::split;
  const float sp = sp_ ? gs_pow2_scale(mp) : 1.f, sU = sp_ ? gs_pow2_scale(mU) : 1.f,
              sF = sp_ ? gs_pow2_scale(mF) : 1.f;
  T **Bp = reinterpret_cast<T **>(a.Bp);
  for (int n = threadIdx.x; n < Np; n += GS_T) {
    const size_t o = (size_t)k * Np + n;
    Split<T>::store(Bp[0], Bp[1], o, sq[n] * sp);
    for (int d = 0; d < 3; ++d) {
      T **B = reinterpret_cast<T **>(a.BU[d]);
      Split<T>::store(B[0], B[1], o, su[d * Np + n] * sU);
    }
  }
  T **BF = reinterpret_cast<T **>(a.BF);
  for (int m = threadIdx.x; m < NF; m += GS_T)
    Split<T>::store(BF[0], BF[1], (size_t)k * NF + m, sf[m] * sF);
  if (threadIdx.x == 0) {
    float *s = a.scale + (size_t)k * 5;
    s[0] = sp, s[1] = sU, s[2] = sF;
  }
}

// per element: rhs of u, v, w from the gradient, divergence and lift
// products, their LSRK update; rhs_p scaled and split into the Vq operand
template <class T>
__global__ void __launch_bounds__(GS_T) k_gs_epi1(GsArgs a) {
  __shared__ float srp[GS_MAXNP], red[3 * GS_T / 32];
  const int k = blockIdx.x, Np = a.Np;
  const float *s = a.scale + (size_t)k * 5;
  const float isp = 1.f / s[0], isU = 1.f / s[1], isF = 1.f / s[2];
  const float *G = a.vgeo + (size_t)k * 9;
  const float *fg = a.fgeo + (size_t)k * 16;
  const size_t base = (size_t)k * 4 * Np;
  float mr = 0.f, d1 = 0.f, d2 = 0.f;
  for (int n = threadIdx.x; n < Np; n += GS_T) {
    const size_t o = (size_t)k * Np + n;
    const float dr = a.G[0][o] * isp, ds = a.G[1][o] * isp, dt = a.G[2][o] * isp;
    float vp = -a.Div[o] * isU;
    float vu = -(G[0] * dr + G[3] * ds + G[6] * dt);
    float vv = -(G[1] * dr + G[4] * ds + G[7] * dt);
    float vw = -(G[2] * dr + G[5] * ds + G[8] * dt);
    for (int f = 0; f < 4; ++f) {
      const float l = a.Lf[f][o] * isF;
      vp += l;
      vu -= fg[4 * f + 1] * l;
      vv -= fg[4 * f + 2] * l;
      vw -= fg[4 * f + 3] * l;
    }
    const float rv[3] = {vu, vv, vw};
    for (int fl = 1; fl < 4; ++fl) {
      const size_t id = base + fl * Np + n;
      const float r = a.fa * a.res[id] + a.fdt * rv[fl - 1];
      a.res[id] = r;
      a.Qout[id] = a.Qin[id] + a.fb * r;
    }
    srp[n] = vp;
    mr = fmaxf(mr, fabsf(vp));
  }
  block_max3(mr, d1, d2, red);
  const float sr = Split<T>::split ? gs_pow2_scale(mr) : 1.f;
  T **BR = reinterpret_cast<T **>(a.BR);
  for (int n = threadIdx.x; n < Np; n += GS_T)
    Split<T>::store(BR[0], BR[1], (size_t)k * Np + n, srp[n] * sr);
  if (threadIdx.x == 0) a.scale[(size_t)k * 5 + 3] = sr;
}

// per element: c^2 / J times (Vq rhs_p) at the cubature points, scaled and
// split into the Pq operand
template <class T>
__global__ void __launch_bounds__(GS_T) k_gs_epi2(GsArgs a) {
  __shared__ float sv[GS_MAXNQ], red[3 * GS_T / 32];
  const int k = blockIdx.x, Nq = a.Nq;
  const float isr = 1.f / a.scale[(size_t)k * 5 + 3];
  float mc = 0.f, d1 = 0.f, d2 = 0.f;
  for (int q = threadIdx.x; q < Nq; q += GS_T) {
    const size_t o = (size_t)k * Nq + q;
    const float v = a.W[o] * isr * a.c2q[o];
    sv[q] = v;
    mc = fmaxf(mc, fabsf(v));
  }
  block_max3(mc, d1, d2, red);
  const float sc = Split<T>::split ? gs_pow2_scale(mc) : 1.f;
  T **BC = reinterpret_cast<T **>(a.BC);
  for (int q = threadIdx.x; q < Nq; q += GS_T)
    Split<T>::store(BC[0], BC[1], (size_t)k * Nq + q, sv[q] * sc);
  if (threadIdx.x == 0) a.scale[(size_t)k * 5 + 4] = sc;
}

// per element: rhs_p = Pq (c2 p_q), LSRK update of p
__global__ void __launch_bounds__(GS_T) k_gs_epi3(GsArgs a) {
  const int k = blockIdx.x, Np = a.Np;
  const float isc = 1.f / a.scale[(size_t)k * 5 + 4];
  const size_t base = (size_t)k * 4 * Np;
  for (int n = threadIdx.x; n < Np; n += GS_T) {
    const size_t id = base + n;
    const float r = a.fa * a.res[id] + a.fdt * (a.Z[(size_t)k * Np + n] * isc);
    a.res[id] = r;
    a.Qout[id] = a.Qin[id] + a.fb * r;
  }
}

}  // namespace

// ------------------------------------------------------------------ host
namespace {

bool is_split(int precision) {
  return precision == BBW_PREC_F16X3 || precision == BBW_PREC_BF16X3;
}

// operator planes of the operand type: hi / lo 16-bit pairs, or FP32
bbw_status upload_operator(const std::vector<float> &A, int precision, void *(&out)[2],
                           const char *what) {
  const size_t n = A.size();
  if (!is_split(precision)) {
    if (cudaMalloc(&out[0], n * 4) != cudaSuccess) return set_error(BBW_ERR_NOMEM, what);
    return set_cuda_error(cudaMemcpy(out[0], A.data(), n * 4, cudaMemcpyHostToDevice), what);
  }
  std::vector<uint16_t> hi(n), lo(n);
  for (size_t i = 0; i < n; ++i) {
    if (precision == BBW_PREC_F16X3) {
      const __half h = __float2half_rn(A[i]);
      const __half l = __float2half_rn(A[i] - __half2float(h));
      std::memcpy(&hi[i], &h, 2), std::memcpy(&lo[i], &l, 2);
    } else {
      const __nv_bfloat16 h = __float2bfloat16_rn(A[i]);
      const __nv_bfloat16 l = __float2bfloat16_rn(A[i] - __bfloat162float(h));
      std::memcpy(&hi[i], &h, 2), std::memcpy(&lo[i], &l, 2);
    }
  }
  for (int p = 0; p < 2; ++p) {
    if (cudaMalloc(&out[p], n * 2) != cudaSuccess) return set_error(BBW_ERR_NOMEM, what);
    const cudaError_t e =
        cudaMemcpy(out[p], (p ? lo : hi).data(), n * 2, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_cuda_error(e, what);
  }
  return BBW_OK;
}

bbw_status alloc_planes(void *(&out)[2], size_t n, int precision, const char *what) {
  const size_t bytes = is_split(precision) ? 2 : 4;
  for (int p = 0; p < (is_split(precision) ? 2 : 1); ++p)
    if (cudaMalloc(&out[p], n * bytes) != cudaSuccess) return set_error(BBW_ERR_NOMEM, what);
  return BBW_OK;
}

}  // namespace

bbw_status gemm_stage_create(GemmStage &g, int N, int K, int Nq, int bc, int precision,
                             const std::vector<float> (&D)[3], const std::vector<float> &LIFT,
                             const std::vector<float> &Vq, const std::vector<float> &Pq) {
  g = GemmStage();
  g.N = N, g.K = K, g.Nq = Nq, g.Np = np_of(N), g.Nfp = nfp_of(N), g.bc = bc;
  g.precision = precision;
  const int Np = g.Np, NF = 4 * g.Nfp;
  if (Np > GS_MAXNP || NF > GS_MAXNF || Nq > GS_MAXNQ)
    return set_error(BBW_ERR_UNSUPPORTED, "GEMM stage: order or cubature rule too large");
  cublasHandle_t h = nullptr;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS)
    return set_error(BBW_ERR_CUDA, "GEMM stage: cublasCreate");
  g.handle = h;
  // a caller-owned workspace keeps cuBLAS from allocating inside a captured step
  g.workspace_bytes = (size_t)32 << 20;
  if (cudaMalloc(&g.workspace, g.workspace_bytes) != cudaSuccess)
    return set_error(BBW_ERR_NOMEM, "GEMM stage: workspace");
  if (cublasSetWorkspace(h, g.workspace, g.workspace_bytes) != CUBLAS_STATUS_SUCCESS)
    return set_error(BBW_ERR_CUDA, "GEMM stage: cublasSetWorkspace");
  bbw_status s;
  for (int d = 0; d < 3; ++d)
    if ((s = upload_operator(D[d], precision, g.D[d], "GEMM stage: D")) != BBW_OK) return s;
  if ((s = upload_operator(LIFT, precision, g.LIFT, "GEMM stage: LIFT")) != BBW_OK ||
      (s = upload_operator(Vq, precision, g.Vq, "GEMM stage: Vq")) != BBW_OK ||
      (s = upload_operator(Pq, precision, g.Pq, "GEMM stage: Pq")) != BBW_OK)
    return s;
  const size_t kn = (size_t)K * Np, kf = (size_t)K * NF, kq = (size_t)K * Nq;
  if ((s = alloc_planes(g.Bp, kn, precision, "GEMM stage: operands")) != BBW_OK) return s;
  for (int d = 0; d < 3; ++d)
    if ((s = alloc_planes(g.BU[d], kn, precision, "GEMM stage: operands")) != BBW_OK) return s;
  if ((s = alloc_planes(g.BF, kf, precision, "GEMM stage: operands")) != BBW_OK ||
      (s = alloc_planes(g.BR, kn, precision, "GEMM stage: operands")) != BBW_OK ||
      (s = alloc_planes(g.BC, kq, precision, "GEMM stage: operands")) != BBW_OK)
    return s;
  float **res[] = {&g.G[0], &g.G[1], &g.G[2], &g.Div, &g.Lf[0], &g.Lf[1], &g.Lf[2], &g.Lf[3], &g.Z};
  for (float **r : res)
    if (cudaMalloc(r, kn * 4) != cudaSuccess) return set_error(BBW_ERR_NOMEM, "GEMM stage: results");
  if (cudaMalloc(&g.W, kq * 4) != cudaSuccess || cudaMalloc(&g.scale, (size_t)K * 5 * 4) != cudaSuccess)
    return set_error(BBW_ERR_NOMEM, "GEMM stage: results");
  return BBW_OK;
}

void gemm_stage_release(GemmStage &g) {
  if (g.handle) cublasDestroy(static_cast<cublasHandle_t>(g.handle));
  cudaFree(g.workspace);
  for (int p = 0; p < 2; ++p) {
    for (int d = 0; d < 3; ++d) cudaFree(g.D[d][p]), cudaFree(g.BU[d][p]);
    cudaFree(g.LIFT[p]), cudaFree(g.Vq[p]), cudaFree(g.Pq[p]);
    cudaFree(g.Bp[p]), cudaFree(g.BF[p]), cudaFree(g.BR[p]), cudaFree(g.BC[p]);
  }
  for (int d = 0; d < 3; ++d) cudaFree(g.G[d]);
  for (int f = 0; f < 4; ++f) cudaFree(g.Lf[f]);
  cudaFree(g.Div), cudaFree(g.W), cudaFree(g.Z), cudaFree(g.scale);
  g = GemmStage();
}

namespace {

// C (m x n, ldc) = A (m x k) B (k x n) + beta C, column-major; split
// operands: three GEMMs A_hi B_hi + A_hi B_lo + A_lo B_hi accumulating in
// FP32; TF32: one GEMM of the FP32 operands
cublasStatus_t gemm_op(const GemmStage &g, int m, int n, int k, void *const (&A)[2],
                       size_t aoff, int lda, void *const (&B)[2], size_t boff, int ldb, float *C,
                       int ldc, float beta) {
  cublasHandle_t h = static_cast<cublasHandle_t>(g.handle);
  const float one = 1.f;
  if (!is_split(g.precision)) {
    const float *a = static_cast<const float *>(A[0]) + aoff;
    const float *b = static_cast<const float *>(B[0]) + boff;
    return cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &one, a, CUDA_R_32F, lda, b,
                        CUDA_R_32F, ldb, &beta, C, CUDA_R_32F, ldc,
                        CUBLAS_COMPUTE_32F_FAST_TF32, CUBLAS_GEMM_DEFAULT);
  }
  const cudaDataType_t t = g.precision == BBW_PREC_F16X3 ? CUDA_R_16F : CUDA_R_16BF;
  const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};
  for (int i = 0; i < 3; ++i) {
    const float bt = i == 0 ? beta : 1.f;
    const uint16_t *a = static_cast<const uint16_t *>(A[pa[i]]) + aoff;
    const uint16_t *b = static_cast<const uint16_t *>(B[pb[i]]) + boff;
    const cublasStatus_t r = cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &one, a, t, lda,
                                          b, t, ldb, &bt, C, CUDA_R_32F, ldc, CUBLAS_COMPUTE_32F,
                                          CUBLAS_GEMM_DEFAULT);
    if (r != CUBLAS_STATUS_SUCCESS) return r;
  }
  return CUBLAS_STATUS_SUCCESS;
}

template <class T>
bbw_status launch_t(GemmStage &g, const GsArgs &a, cudaStream_t st) {
  const int K = g.K, Np = g.Np, Nfp = g.Nfp, NF = 4 * Nfp, Nq = g.Nq;
  cublasHandle_t h = static_cast<cublasHandle_t>(g.handle);
  if (cublasSetStream(h, st) != CUBLAS_STATUS_SUCCESS)
    return set_error(BBW_ERR_CUDA, "GEMM stage: cublasSetStream");
  bbw_status s;
  k_gs_prep<T><<<K, GS_T, 0, st>>>(a);
  if ((s = check_launch("GEMM stage: operands")) != BBW_OK) return s;
  cublasStatus_t r = CUBLAS_STATUS_SUCCESS;
  // gradient of p, divergence of U (rk_volume), lift per face (rk_surface)
  for (int d = 0; d < 3 && r == CUBLAS_STATUS_SUCCESS; ++d)
    r = gemm_op(g, Np, K, Np, g.D[d], 0, Np, g.Bp, 0, Np, g.G[d], Np, 0.f);
  for (int d = 0; d < 3 && r == CUBLAS_STATUS_SUCCESS; ++d)
    r = gemm_op(g, Np, K, Np, g.D[d], 0, Np, g.BU[d], 0, Np, g.Div, Np, d ? 1.f : 0.f);
  for (int f = 0; f < 4 && r == CUBLAS_STATUS_SUCCESS; ++f)
    r = gemm_op(g, Np, K, Nfp, g.LIFT, (size_t)f * Nfp * Np, Np, g.BF, (size_t)f * Nfp, NF,
                g.Lf[f], Np, 0.f);
  if (r != CUBLAS_STATUS_SUCCESS) return set_error(BBW_ERR_CUDA, "GEMM stage: volume / lift GEMM");
  k_gs_epi1<T><<<K, GS_T, 0, st>>>(a);
  if ((s = check_launch("GEMM stage: epilogue 1")) != BBW_OK) return s;
  // WADG (rk_update_WADG): Vq rhs_p, c^2 / J, Pq
  r = gemm_op(g, Nq, K, Np, g.Vq, 0, Nq, g.BR, 0, Np, g.W, Nq, 0.f);
  if (r != CUBLAS_STATUS_SUCCESS) return set_error(BBW_ERR_CUDA, "GEMM stage: Vq GEMM");
  k_gs_epi2<T><<<K, GS_T, 0, st>>>(a);
  if ((s = check_launch("GEMM stage: epilogue 2")) != BBW_OK) return s;
  r = gemm_op(g, Np, K, Nq, g.Pq, 0, Np, g.BC, 0, Nq, g.Z, Np, 0.f);
  if (r != CUBLAS_STATUS_SUCCESS) return set_error(BBW_ERR_CUDA, "GEMM stage: Pq GEMM");
  k_gs_epi3<<<K, GS_T, 0, st>>>(a);
  return check_launch("GEMM stage: update");
}

}  // namespace

bbw_status gemm_stage_launch(GemmStage &g, const GemmInputs &in, const float *Qin, float *Qout,
                             float *res, float fa, float fb, float fdt, cudaStream_t st) {
  GsArgs a;
  a.K = g.K, a.Np = g.Np, a.Nfp = g.Nfp, a.Nq = g.Nq, a.bc = g.bc, a.pat_off = in.pat_off;
  a.fa = fa, a.fb = fb, a.fdt = fdt;
  a.Qin = Qin, a.Qout = Qout, a.res = res;
  a.vgeo = in.vgeo, a.fgeo = in.fgeo, a.c2q = in.c2q, a.nbr = in.nbr, a.tables = in.tables;
  for (int p = 0; p < 2; ++p) {
    a.Bp[p] = g.Bp[p], a.BF[p] = g.BF[p], a.BR[p] = g.BR[p], a.BC[p] = g.BC[p];
    for (int d = 0; d < 3; ++d) a.BU[d][p] = g.BU[d][p];
  }
  for (int d = 0; d < 3; ++d) a.G[d] = g.G[d];
  for (int f = 0; f < 4; ++f) a.Lf[f] = g.Lf[f];
  a.Div = g.Div, a.W = g.W, a.Z = g.Z, a.scale = g.scale;
  switch (g.precision) {
    case BBW_PREC_F16X3: return launch_t<__half>(g, a, st);
    case BBW_PREC_BF16X3: return launch_t<__nv_bfloat16>(g, a, st);
    default: return launch_t<float>(g, a, st);
  }
}

}  // namespace bbw
