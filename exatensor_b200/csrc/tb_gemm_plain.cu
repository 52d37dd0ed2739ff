// tb_gemm_plain.cu -- GEMMs of the plain TTGT contraction, in the tensor's
// own data type: C[m + n*ldc] = alpha * sum_k A[k + m*lda] * B[k + n*ldb]
// (+ beta * C), both operands K-major (the matricized operands of TAL-SH's
// GEMM('T','N') call, TALSH/tensor_algebra_gpu_nvidia.cu:6899-7024).
//   R8: FP64 tensor-core MMA (mma.sync m8n8k4 f64; tcgen05 has no FP64 kind)
//   C8: the same MMA on real/imaginary fragments (4 real products)
//   R4, C4: FP32 FFMA on the CUDA cores
#include "tb_common.cuh"
#include "tb_gemm.h"

namespace tb {

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool pred) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(pred ? 16 : 0));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool pred) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(pred ? 8 : 0));
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src, bool pred) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(pred ? 4 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// ------------------------------------------------------------------ R8 -----
constexpr int D_BM = 128, D_BN = 128, D_BK = 16, D_LD = 20, D_ST = 3;

template <bool VEC16>
__global__ void __launch_bounds__(256) dgemm_tn_kernel(int M, int N, int K, const double* __restrict__ A,
                                                       int64_t lda, const double* __restrict__ B, int64_t ldb,
                                                       double* __restrict__ C, int64_t ldc, double alpha,
                                                       double beta) {
  extern __shared__ __align__(16) double sm[];
  double* As = sm;                              // [ST][BM][LD]
  double* Bs = sm + D_ST * D_BM * D_LD;         // [ST][BN][LD]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;      // 2 x 4 warps, warp tile 64 x 32
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.y * D_BM, n0 = blockIdx.x * D_BN;
  const int ktiles = (K + D_BK - 1) / D_BK;

  auto load_stage = [&](int st, int kt) {
    const int k0 = kt * D_BK;
    double* as = As + st * D_BM * D_LD;
    double* bs = Bs + st * D_BN * D_LD;
    if (VEC16) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int c = tid + i * 256, r = c >> 3, kc = (c & 7) * 2;
        const bool pa = (m0 + r < M) && (k0 + kc < K);
        const bool pb = (n0 + r < N) && (k0 + kc < K);
        cp_async16(as + r * D_LD + kc, pa ? A + (int64_t)(m0 + r) * lda + k0 + kc : A, pa);
        cp_async16(bs + r * D_LD + kc, pb ? B + (int64_t)(n0 + r) * ldb + k0 + kc : B, pb);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int c = tid + i * 256, r = c >> 4, kc = c & 15;
        const bool pa = (m0 + r < M) && (k0 + kc < K);
        const bool pb = (n0 + r < N) && (k0 + kc < K);
        cp_async8(as + r * D_LD + kc, pa ? A + (int64_t)(m0 + r) * lda + k0 + kc : A, pa);
        cp_async8(bs + r * D_LD + kc, pb ? B + (int64_t)(n0 + r) * ldb + k0 + kc : B, pb);
      }
    }
  };

  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int s = 0; s < D_ST - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<D_ST - 2>();
    __syncthreads();
    const int nk = kt + D_ST - 1;
    if (nk < ktiles) load_stage(nk % D_ST, nk);
    cp_async_commit();
    const double* as = As + (kt % D_ST) * D_BM * D_LD + (wm * 64 + g) * D_LD + t;
    const double* bs = Bs + (kt % D_ST) * D_BN * D_LD + (wn * 32 + g) * D_LD + t;
#pragma unroll
    for (int kk = 0; kk < D_BK; kk += 4) {
      double a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = as[i * 8 * D_LD + kk];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[j * 8 * D_LD + kk];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int m = m0 + wm * 64 + i * 8 + g;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = n0 + wn * 32 + j * 8 + 2 * t + h;
        if (n >= N) continue;
        double* c = C + m + (int64_t)n * ldc;
        const double v = alpha * acc[i][j][h];
        *c = (beta == 0.0) ? v : v + beta * *c;
      }
    }
  }
}

// ------------------------------------------------------------------ C8 -----
constexpr int Z_BM = 64, Z_BN = 64, Z_BK = 8, Z_LD = 12, Z_ST = 3;

__global__ void __launch_bounds__(256) zgemm_tn_kernel(int M, int N, int K, const double2* __restrict__ A,
                                                       int64_t lda, const double2* __restrict__ B, int64_t ldb,
                                                       double2* __restrict__ C, int64_t ldc, double ar,
                                                       double ai, double br, double bi, int lconj, int rconj) {
  extern __shared__ __align__(16) double2 smz[];
  double2* As = smz;                           // [ST][BM][LD]
  double2* Bs = smz + Z_ST * Z_BM * Z_LD;      // [ST][BN][LD]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;     // 2 x 4 warps, warp tile 32 x 16
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.y * Z_BM, n0 = blockIdx.x * Z_BN;
  const int ktiles = (K + Z_BK - 1) / Z_BK;
  auto load_stage = [&](int st, int kt) {
    const int k0 = kt * Z_BK;
    double2* as = As + st * Z_BM * Z_LD;
    double2* bs = Bs + st * Z_BN * Z_LD;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = tid + i * 256, r = c >> 3, kc = c & 7;
      const bool pa = (m0 + r < M) && (k0 + kc < K);
      const bool pb = (n0 + r < N) && (k0 + kc < K);
      cp_async16(as + r * Z_LD + kc, pa ? A + (int64_t)(m0 + r) * lda + k0 + kc : A, pa);
      cp_async16(bs + r * Z_LD + kc, pb ? B + (int64_t)(n0 + r) * ldb + k0 + kc : B, pb);
    }
  };
  double cr[4][2][2], ci[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;
  const double sa = lconj ? -1.0 : 1.0, sb = rconj ? -1.0 : 1.0;
#pragma unroll
  for (int s = 0; s < Z_ST - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<Z_ST - 2>();
    __syncthreads();
    const int nk = kt + Z_ST - 1;
    if (nk < ktiles) load_stage(nk % Z_ST, nk);
    cp_async_commit();
    const double2* as = As + (kt % Z_ST) * Z_BM * Z_LD + (wm * 32 + g) * Z_LD + t;
    const double2* bs = Bs + (kt % Z_ST) * Z_BN * Z_LD + (wn * 16 + g) * Z_LD + t;
#pragma unroll
    for (int kk = 0; kk < Z_BK; kk += 4) {
      double are[4], aim[4], anim[4], bre[2], bim[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 v = as[i * 8 * Z_LD + kk];
        are[i] = v.x; aim[i] = sa * v.y; anim[i] = -aim[i];
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const double2 v = bs[j * 8 * Z_LD + kk];
        bre[j] = v.x; bim[j] = sb * v.y;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          dmma(cr[i][j][0], cr[i][j][1], are[i], bre[j]);
          dmma(cr[i][j][0], cr[i][j][1], anim[i], bim[j]);
          dmma(ci[i][j][0], ci[i][j][1], are[i], bim[j]);
          dmma(ci[i][j][0], ci[i][j][1], aim[i], bre[j]);
        }
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + wm * 32 + i * 8 + g;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = n0 + wn * 16 + j * 8 + 2 * t + h;
        if (n >= N) continue;
        double2* c = C + m + (int64_t)n * ldc;
        const double xr = cr[i][j][h], xi = ci[i][j][h];
        double2 o = make_double2(ar * xr - ai * xi, ar * xi + ai * xr);
        if (br != 0.0 || bi != 0.0) {
          const double2 old = *c;
          o.x += br * old.x - bi * old.y;
          o.y += br * old.y + bi * old.x;
        }
        *c = o;
      }
  }
}

// ------------------------------------------------------------- R4 / C4 -----
// 128x128 tile, BK=8, 256 threads, 8x8 outputs per thread (two 4x4 quads
// per dimension so that shared-memory reads are float4 and conflict-free).
constexpr int S_BM = 128, S_BN = 128, S_BK = 8;

__global__ void __launch_bounds__(256) sgemm_tn_kernel(int M, int N, int K, const float* __restrict__ A,
                                                       int64_t lda, const float* __restrict__ B, int64_t ldb,
                                                       float* __restrict__ C, int64_t ldc, float alpha,
                                                       float beta) {
  __shared__ __align__(16) float As[2][S_BK][S_BM + 4];
  __shared__ __align__(16) float Bs[2][S_BK][S_BN + 4];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * S_BM, n0 = blockIdx.x * S_BN;
  // loader: each thread loads 4 elements of A and 4 of B per k-tile (rows r, k = kq..kq+3)
  const int lr = tid >> 1, lk = (tid & 1) * 4;
  float ra[4], rb[4];
  auto gload = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = k0 + lk + q;
      ra[q] = (m0 + lr < M && k < K) ? A[(int64_t)(m0 + lr) * lda + k] : 0.f;
      rb[q] = (n0 + lr < N && k < K) ? B[(int64_t)(n0 + lr) * ldb + k] : 0.f;
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) { As[buf][lk + q][lr] = ra[q]; Bs[buf][lk + q][lr] = rb[q]; }
  };
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
  const int ktiles = (K + S_BK - 1) / S_BK;
  gload(0);
  sstore(0);
  __syncthreads();
  for (int kt = 0; kt < ktiles; ++kt) {
    const int cur = kt & 1;
    if (kt + 1 < ktiles) gload((kt + 1) * S_BK);
#pragma unroll
    for (int kk = 0; kk < S_BK; ++kk) {
      float a[8], b[8];
      const float4 a0 = *reinterpret_cast<const float4*>(&As[cur][kk][ty * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[cur][kk][64 + ty * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[cur][kk][tx * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[cur][kk][64 + tx * 4]);
      a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w; a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
      b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w; b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if (kt + 1 < ktiles) sstore(cur ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int m = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int n = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
      if (n >= N) continue;
      float* c = C + m + (int64_t)n * ldc;
      const float v = alpha * acc[i][j];
      *c = (beta == 0.f) ? v : v + beta * *c;
    }
  }
}

// Complex FP32: 64x64 tile, BK=8, 256 threads, 4x4 complex outputs per thread.
__global__ void __launch_bounds__(256) cgemm_tn_kernel(int M, int N, int K, const float2* __restrict__ A,
                                                       int64_t lda, const float2* __restrict__ B, int64_t ldb,
                                                       float2* __restrict__ C, int64_t ldc, float ar, float ai,
                                                       float br, float bi, int lconj, int rconj) {
  __shared__ __align__(16) float2 As[8][64 + 2];
  __shared__ __align__(16) float2 Bs[8][64 + 2];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  const float sa = lconj ? -1.f : 1.f, sb = rconj ? -1.f : 1.f;
  float accr[4][4], acci[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) accr[i][j] = acci[i][j] = 0.f;
  for (int k0 = 0; k0 < K; k0 += 8) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = tid + q * 256, r = c >> 3, kk = c & 7;
      float2 va = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
      if (m0 + r < M && k0 + kk < K) va = A[(int64_t)(m0 + r) * lda + k0 + kk];
      if (n0 + r < N && k0 + kk < K) vb = B[(int64_t)(n0 + r) * ldb + k0 + kk];
      va.y *= sa; vb.y *= sb;
      As[kk][r] = va; Bs[kk][r] = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
      float2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          accr[i][j] = fmaf(a[i].x, b[j].x, accr[i][j]);
          accr[i][j] = fmaf(-a[i].y, b[j].y, accr[i][j]);
          acci[i][j] = fmaf(a[i].x, b[j].y, acci[i][j]);
          acci[i][j] = fmaf(a[i].y, b[j].x, acci[i][j]);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      float2* c = C + m + (int64_t)n * ldc;
      const float xr = accr[i][j], xi = acci[i][j];
      float2 o = make_float2(ar * xr - ai * xi, ar * xi + ai * xr);
      if (br != 0.f || bi != 0.f) {
        const float2 old = *c;
        o.x += br * old.x - bi * old.y;
        o.y += br * old.y + bi * old.x;
      }
      *c = o;
    }
  }
}

}  // namespace

int gemm_plain_tn(int dtk, int64_t M, int64_t N, int64_t K, const void* A, int64_t lda, const void* B,
                  int64_t ldb, void* C, int64_t ldc, double ar, double ai, double br, double bi, int lconj,
                  int rconj, cudaStream_t s) {
  if (M <= 0 || N <= 0) return 0;
  if (M > INT32_MAX || N > INT32_MAX || K > INT32_MAX) { set_error("gemm_plain_tn: size too large"); return TB_ERR_LIMIT; }
  switch (dtk) {
    case kR8: {
      const size_t smem = (size_t)D_ST * (D_BM + D_BN) * D_LD * sizeof(double);
      static DeviceOnce attr16, attr8;
      TB_CUDA(smem_limit_once(attr16, dgemm_tn_kernel<true>, (int)smem));
      TB_CUDA(smem_limit_once(attr8, dgemm_tn_kernel<false>, (int)smem));
      dim3 grid((unsigned)((N + D_BN - 1) / D_BN), (unsigned)((M + D_BM - 1) / D_BM));
      const bool v16 = (lda % 2 == 0) && (ldb % 2 == 0) && ((uintptr_t)A % 16 == 0) && ((uintptr_t)B % 16 == 0);
      if (v16)
        dgemm_tn_kernel<true><<<grid, 256, smem, s>>>((int)M, (int)N, (int)K, (const double*)A, lda,
                                                     (const double*)B, ldb, (double*)C, ldc, ar, br);
      else
        dgemm_tn_kernel<false><<<grid, 256, smem, s>>>((int)M, (int)N, (int)K, (const double*)A, lda,
                                                      (const double*)B, ldb, (double*)C, ldc, ar, br);
      break;
    }
    case kC8: {
      const size_t smem = (size_t)Z_ST * (Z_BM + Z_BN) * Z_LD * sizeof(double2);
      static DeviceOnce attr;
      TB_CUDA(smem_limit_once(attr, zgemm_tn_kernel, (int)smem));
      dim3 grid((unsigned)((N + Z_BN - 1) / Z_BN), (unsigned)((M + Z_BM - 1) / Z_BM));
      zgemm_tn_kernel<<<grid, 256, smem, s>>>((int)M, (int)N, (int)K, (const double2*)A, lda, (const double2*)B,
                                             ldb, (double2*)C, ldc, ar, ai, br, bi, lconj, rconj);
      break;
    }
    case kR4: {
      dim3 grid((unsigned)((N + S_BN - 1) / S_BN), (unsigned)((M + S_BM - 1) / S_BM));
      sgemm_tn_kernel<<<grid, 256, 0, s>>>((int)M, (int)N, (int)K, (const float*)A, lda, (const float*)B, ldb,
                                          (float*)C, ldc, (float)ar, (float)br);
      break;
    }
    case kC4: {
      dim3 grid((unsigned)((N + 63) / 64), (unsigned)((M + 63) / 64));
      cgemm_tn_kernel<<<grid, 256, 0, s>>>((int)M, (int)N, (int)K, (const float2*)A, lda, (const float2*)B, ldb,
                                          (float2*)C, ldc, (float)ar, (float)ai, (float)br, (float)bi, lconj,
                                          rconj);
      break;
    }
    default:
      return TB_ERR_INVALID_ARGS;
  }
  TB_CHECK_LAUNCH();
  return 0;
}

}  // namespace tb
