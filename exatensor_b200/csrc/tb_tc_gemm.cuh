// tb_tc_gemm.cuh -- persistent tcgen05 GEMM with multi-pass accumulation and
// a fused tensor epilogue.
//
//   C[m][n] = sum over passes p of  scale_p(m,n) * sum_{(a,b,k0,k1) in p} sum_{k0<=k<k1} A_a[m][k] * B_b[n][k]
//   D[dm[m] + dn[n]] = beta*D + alpha*C    (dm/dn: the output permutation)
//
// A_a / B_b are planes of K-major operands (INT8 slices of FP64 data, or
// BF16 high/low parts of FP32 data) prepared by tb_tc.cu.  One 128 x BN output
// tile per CTA iteration; 192 threads:
//   warp 0      TMA producer (one elected lane), kStagesTC-deep smem ring
//   warp 1      TMEM allocator and single-thread tcgen05.mma issuer
//   warps 2..5  epilogue: tcgen05.ld of the finished accumulator, scaling,
//               read-modify-write of D through the offset tables
// Two TMEM accumulators (2*BN columns) let the epilogue of pass p overlap the
// MMAs of pass p+1.  Every wait is bounded (tb_sm100.cuh).
#pragma once
#include "tb_common.cuh"
#include "tb_sm100.cuh"

namespace tb {

constexpr int kStagesTC = 4;
constexpr int kMaxProducts = 64;  // entries (plane pair and K range) over all passes
constexpr int kTcThreads = 192;

enum TcEpilogue { EPI_OZAKI_R = 0, EPI_OZAKI_C = 1, EPI_BF16_R = 2, EPI_BF16_C = 3 };

struct __align__(64) TcGemmParams {
  CUtensorMap tmA;            // 3-D: (K elements, rows, planes)
  CUtensorMap tmB;
  int M, N;                   // valid rows of A and of B (real-expanded)
  int mtiles, ntiles;         // tiles of 128 rows x BN columns
  int kblocks;                // 128-byte K blocks
  int npass;
  int pass_first[kMaxProducts + 1];  // entries of pass p: [pass_first[p], pass_first[p+1])
  int prod_a[kMaxProducts], prod_b[kMaxProducts];    // plane of A and of B
  int prod_kb0[kMaxProducts], prod_kb1[kMaxProducts];  // K-block range
  int pass_shift[kMaxProducts];      // INT8 slices: the pass's weight is 2^-pass_shift
  void* D;
  const int64_t* dm;          // D offset of row m (elements of D's data kind)
  const int64_t* dn;          // D offset of column n (complex: of column pair n/2)
  const int* rowexp;          // INT8 slices: row scale exponents
  const int* colexp;          // INT8 slices: column scale exponents
  double ar, ai, br, bi;      // alpha, beta
  unsigned int* err;
};

struct TcSmemBarriers {
  uint64_t full[kStagesTC];
  uint64_t empty[kStagesTC];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint32_t tmem_base;
};

template <int BN>
__host__ __device__ constexpr size_t tc_smem_bytes() {
  return 1024 /*alignment slack*/ + (size_t)kStagesTC * (128 * 128 + BN * 128) + sizeof(TcSmemBarriers) + 64;
}

__device__ __forceinline__ double pow2d(int e) {
  // exact 2^e for -1022 <= e <= 1023 (clamped outside)
  e = e < -1022 ? -1022 : (e > 1023 ? 1023 : e);
  return __longlong_as_double((long long)(e + 1023) << 52);
}
// x * 2^e with one rounding, also when the result is subnormal (e >= -2100).
__device__ __forceinline__ double scale2(double x, int e) {
  return e >= -1022 ? x * pow2d(e) : (x * pow2d(e + 1022)) * pow2d(-1022);
}

template <int BN, bool I8, int EPI>
__global__ void __launch_bounds__(kTcThreads, 1) tc_gemm_kernel(const __grid_constant__ TcGemmParams P) {
  using namespace sm100;
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* smA = base;                                    // [stages][128 rows][128 B]
  unsigned char* smB = base + (size_t)kStagesTC * 128 * 128;    // [stages][BN rows][128 B]
  TcSmemBarriers* bars = (TcSmemBarriers*)(smB + (size_t)kStagesTC * BN * 128);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntile_total = P.mtiles * P.ntiles;
  const int nprod = P.pass_first[P.npass];

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesTC; ++s) { mbar_init(&bars->full[s], 1); mbar_init(&bars->empty[s], 1); }
    for (int a = 0; a < 2; ++a) { mbar_init(&bars->acc_full[a], 1); mbar_init(&bars->acc_empty[a], 4); }
    fence_barrier_init();
    prefetch_tmap(&P.tmA);
    prefetch_tmap(&P.tmB);
  }
  if (warp == 1) {
    tmem_alloc(&bars->tmem_base, 2 * BN);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = bars->tmem_base;
  bool ok = true;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      uint32_t it = 0;
      const uint32_t bytes = 128 * 128 + BN * 128;
      for (int t = blockIdx.x; t < ntile_total && ok; t += gridDim.x) {
        const int mb = t / P.ntiles, nb = t - mb * P.ntiles;
        for (int q = 0; q < nprod && ok; ++q) {
          for (int kb = P.prod_kb0[q]; kb < P.prod_kb1[q]; ++kb, ++it) {
            const int s = it % kStagesTC;
            const uint32_t ph = (it / kStagesTC) & 1;
            if (!(ok = mbar_wait(&bars->empty[s], ph ^ 1, P.err))) break;
            mbar_expect_tx(&bars->full[s], bytes);
            tma_load_3d(smA + (size_t)s * 128 * 128, &P.tmA, kb * (I8 ? 128 : 64), mb * 128, P.prod_a[q],
                        &bars->full[s]);
            tma_load_3d(smB + (size_t)s * BN * 128, &P.tmB, kb * (I8 ? 128 : 64), nb * BN, P.prod_b[q],
                        &bars->full[s]);
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t kIdesc = idesc(I8, BN);
      uint32_t it = 0, acc_it = 0;
      for (int t = blockIdx.x; t < ntile_total && ok; t += gridDim.x) {
        for (int p = 0; p < P.npass && ok; ++p, ++acc_it) {
          const int a = acc_it & 1;
          const uint32_t aph = (acc_it >> 1) & 1;
          if (!(ok = mbar_wait(&bars->acc_empty[a], aph ^ 1, P.err))) break;
          tc_fence_after();
          const uint32_t dcol = tmem + (uint32_t)(a * BN);
          bool first = true;
          for (int q = P.pass_first[p]; q < P.pass_first[p + 1] && ok; ++q) {
            for (int kb = P.prod_kb0[q]; kb < P.prod_kb1[q]; ++kb, ++it) {
              const int s = it % kStagesTC;
              const uint32_t ph = (it / kStagesTC) & 1;
              if (!(ok = mbar_wait(&bars->full[s], ph, P.err))) break;
              tc_fence_after();
              const uint32_t sa = smem_u32(smA + (size_t)s * 128 * 128);
              const uint32_t sb = smem_u32(smB + (size_t)s * BN * 128);
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                mma<I8>(dcol, sdesc_k128(sa + kk * 32), sdesc_k128(sb + kk * 32), kIdesc,
                        (first && kk == 0) ? 0u : 1u);
              }
              first = false;
              mma_commit(&bars->empty[s]);
            }
          }
          mma_commit(&bars->acc_full[a]);
        }
      }
    }
  } else {
    // ---------------- epilogue (warps 2..5) ----------------
    const int quad = warp & 3;  // TMEM lanes 32*quad .. 32*quad+31
    uint32_t acc_it = 0;
    for (int t = blockIdx.x; t < ntile_total && ok; t += gridDim.x) {
      const int mb = t / P.ntiles, nb = t - mb * P.ntiles;
      const int m = mb * 128 + quad * 32 + lane;
      const bool mval = m < P.M;
      const int64_t dmo = mval ? P.dm[m] : 0;
      const int re = (EPI == EPI_OZAKI_R || EPI == EPI_OZAKI_C) && mval ? P.rowexp[m] : 0;
      for (int p = 0; p < P.npass && ok; ++p, ++acc_it) {
        const int a = acc_it & 1;
        const uint32_t aph = (acc_it >> 1) & 1;
        if (!(ok = mbar_wait(&bars->acc_full[a], aph, P.err))) break;
        tc_fence_after();
        const bool first = (p == 0);
        const int shift = (EPI == EPI_OZAKI_R || EPI == EPI_OZAKI_C) ? P.pass_shift[p] : 0;
#pragma unroll 1
        for (int c = 0; c < BN / 32; ++c) {
          uint32_t r[32];
          tmem_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * BN + c * 32), r);
          const int n0 = nb * BN + c * 32;
          if (!mval) continue;
          if (EPI == EPI_OZAKI_R) {
            double* D = (double*)P.D;
#pragma unroll 8
            for (int j = 0; j < 32; ++j) {
              const int n = n0 + j;
              if (n >= P.N) break;
              const double v = P.ar * scale2((double)(int)r[j], re + P.colexp[n] - shift);
              double* dp = D + dmo + P.dn[n];
              *dp = first ? (P.br == 0.0 ? v : fma(P.br, *dp, v)) : (*dp + v);
            }
          } else if (EPI == EPI_OZAKI_C) {
            double2* D = (double2*)P.D;
#pragma unroll 4
            for (int j = 0; j < 32; j += 2) {
              const int n = n0 + j;
              if (n >= P.N) break;
              const int e = re + P.colexp[n] - shift;
              const double xr = scale2((double)(int)r[j], e), xi = scale2((double)(int)r[j + 1], e);
              double2 v = make_double2(P.ar * xr - P.ai * xi, P.ar * xi + P.ai * xr);
              double2* dp = D + dmo + P.dn[n >> 1];
              double2 d = *dp;
              if (first) {
                v.x += P.br * d.x - P.bi * d.y;
                v.y += P.br * d.y + P.bi * d.x;
              } else {
                v.x += d.x; v.y += d.y;
              }
              *dp = v;
            }
          } else if (EPI == EPI_BF16_R) {
            float* D = (float*)P.D;
            const float ar = (float)P.ar, br = (float)P.br;
#pragma unroll 8
            for (int j = 0; j < 32; ++j) {
              const int n = n0 + j;
              if (n >= P.N) break;
              const float v = ar * __uint_as_float(r[j]);
              float* dp = D + dmo + P.dn[n];
              *dp = first ? (br == 0.f ? v : fmaf(br, *dp, v)) : (*dp + v);
            }
          } else {
            float2* D = (float2*)P.D;
            const float ar = (float)P.ar, ai = (float)P.ai, br = (float)P.br, bi = (float)P.bi;
#pragma unroll 4
            for (int j = 0; j < 32; j += 2) {
              const int n = n0 + j;
              if (n >= P.N) break;
              const float xr = __uint_as_float(r[j]), xi = __uint_as_float(r[j + 1]);
              float2 v = make_float2(ar * xr - ai * xi, ar * xi + ai * xr);
              float2* dp = D + dmo + P.dn[n >> 1];
              float2 d = *dp;
              if (first) {
                v.x += br * d.x - bi * d.y;
                v.y += br * d.y + bi * d.x;
              } else {
                v.x += d.x; v.y += d.y;
              }
              *dp = v;
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&bars->acc_empty[a]);
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * BN);
  }
}

}  // namespace tb
