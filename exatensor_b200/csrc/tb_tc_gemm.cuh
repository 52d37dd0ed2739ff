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

#include <type_traits>

namespace tb {

constexpr int kStagesTC = 4;
// The epilogue warps wait a whole accumulator pass (tens of microseconds) for
// their next accumulator; they poll every this many nanoseconds, so that the
// warps sharing their schedulers with the TMA and MMA threads do not take
// issue slots from them.
constexpr unsigned kEpilogueSleepNs = 200;
constexpr int kMaxProducts = 64;  // entries (plane pair and K range) over all passes
constexpr int kTcThreads = 192;

// EPI_RESID: modular residues (Ozaki scheme II) -- each pass is one modulus
// (pass_shift holds it) and the epilogue stores acc mod m as one byte per
// element into residue plane `pass` (layout [pass][column][row], rows fastest);
// crt_kernel later rebuilds D from all planes.
enum TcEpilogue { EPI_OZAKI_R = 0, EPI_OZAKI_C = 1, EPI_BF16_R = 2, EPI_BF16_C = 3, EPI_RESID = 4 };

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
  int pass_shift[kMaxProducts];      // INT8 slices: the pass's weight is 2^-pass_shift; residues: the modulus
  int pass_magic[kMaxProducts];      // residues: floor(2^32 / modulus), for the epilogue's reduction
  void* D;
  const int64_t* dm;          // D offset of row m (elements of D's data kind)
  const int64_t* dn;          // D offset of column n (complex: of column pair n/2)
  const int* rowexp;          // INT8 slices: row scale exponents
  const int* colexp;          // INT8 slices: column scale exponents
  double ar, ai, br, bi;      // alpha, beta
  unsigned int* err;
  int nf_skip;                // 1: leave entries of flagged rows / columns to the non-finite fix-up
  uint8_t* res;               // EPI_RESID: residue planes
  int64_t res_ld, res_plane;  // EPI_RESID: column stride and plane stride (bytes)
  int res_nch;                // EPI_RESID: passes per modulus (K chunks of at most
                              // 1023 blocks each, added up mod m by the epilogue)
  unsigned int* sched;        // single-SM kernel: zeroed work-unit counter (dynamic
                              // scheduling), or null for a static round robin
  int l2hint;                 // 1: A tiles are loaded evict-first and B tiles
                              // evict-last (B planes are re-read by every m-tile)
};

// Work units of the GEMMs.  EPI_RESID: one (modulus, tile) per unit with the
// moduli outermost -- every modulus has its own output plane, so all CTAs
// work on one modulus at a time and its B plane can stay in L2; the unit's
// passes are that modulus's K chunks, in order.  Other epilogues: one tile
// with all its passes (they accumulate into D in order).
template <int EPI>
__host__ __device__ __forceinline__ int gemm_units(const TcGemmParams& P) {
  return EPI == EPI_RESID ? (P.npass / P.res_nch) * P.mtiles * P.ntiles : P.mtiles * P.ntiles;
}
struct GemmUnit { int t, p0, p1; };
template <int EPI>
__device__ __forceinline__ GemmUnit gemm_unit(const TcGemmParams& P, int u) {
  const int nt = P.mtiles * P.ntiles;
  if (EPI == EPI_RESID) {
    const int i = u / nt;
    return {u - i * nt, i * P.res_nch, (i + 1) * P.res_nch};
  }
  return {u, 0, P.npass};
}

// A row or column whose exponent entry exceeds this holds a NaN or an
// infinity (exponent field 2047, minus 1021): with nf_skip the epilogue leaves
// its D entries untouched for the non-finite fix-up kernel.
constexpr int kNonFiniteExp = 2047 - 1021;

// Epilogue view of one output block: what epilogue_pass reads besides TMEM.
struct EpiView {
  void* D;
  const int64_t* dn;
  const int* colexp;
  int N;
  double ar, ai, br, bi;
  int nf_skip;
};

// Ring through which the producer hands work units to the MMA and epilogue
// warps (one arrival from the MMA thread and one from each epilogue warp
// frees an entry).
constexpr int kUnitRing = 4;
constexpr int kUnitConsumers = 5;

struct TcSmemBarriers {
  uint64_t full[kStagesTC];
  uint64_t empty[kStagesTC];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint64_t unit_full[kUnitRing];
  uint64_t unit_empty[kUnitRing];
  int unit[kUnitRing];
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

// One accumulator pass of the epilogue for the row held by this thread (EP
// provides D, dn, colexp, N and alpha/beta: TcGemmParams or EpiView): reads
// the BN accumulator columns of TMEM lane `tcol` (lane and column base
// encoded) 32 at a time, scales them and updates D through the offset tables.
// Column metadata (D offset, scale exponent) is loaded once per 32 columns, one
// column per lane, and broadcast with shuffles; all 32 loads of D of a chunk
// are issued before any of them is used, so that a warp keeps 1024 loads in
// flight instead of waiting on each one.
template <int BN, int EPI, class EP>
__device__ __forceinline__ void epilogue_pass(const EP& P, uint32_t tcol, bool mval, int64_t dmo, int re, int nb,
                                              bool first, int shift, int magic = 0) {
  using namespace sm100;
  constexpr bool OZ = EPI == EPI_OZAKI_R || EPI == EPI_OZAKI_C;
  constexpr bool CPLX = EPI == EPI_OZAKI_C || EPI == EPI_BF16_C;
  const int lane = threadIdx.x & 31;
  const bool load_d = !(first && P.br == 0.0 && P.bi == 0.0);
#pragma unroll 1
  for (int c = 0; c < BN / 32; ++c) {
    uint32_t r[32];
    tmem_ld32(tcol + (uint32_t)(c * 32), r);
    const int n0 = nb * BN + c * 32;
    if constexpr (EPI == EPI_RESID) {
      // residues of the exact INT32 sums: shift is the modulus m, and the
      // caller passes this pass's plane through P.res / res_plane.  v mod m
      // by a multiply-high with magic = floor(2^32 / m): the quotient estimate
      // is off by at most one either way, so two conditional corrections give
      // the residue in [0, m) (integer pipes only; no division).  Later K
      // chunks of a modulus (!first) add their residue to the stored one.
      if constexpr (std::is_same<EP, TcGemmParams>::value) {
        if (mval) {
          uint8_t* col = P.res + dmo;  // dmo: this modulus's plane offset + row
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (n0 + j >= P.N) break;
            const int v = (int)r[j];
            int rr = v - __mulhi(v, magic) * shift;
            rr += rr < 0 ? shift : 0;
            rr -= rr >= shift ? shift : 0;
            uint8_t* dst = col + (int64_t)(n0 + j) * P.res_ld;
            if (!first) {
              rr += *dst;
              rr -= rr >= shift ? shift : 0;
            }
            *dst = (uint8_t)rr;
          }
        }
      }
      continue;
    }
    // lane j: metadata of column n0 + j (complex: of column pair (n0 + j) / 2)
    const int nl = n0 + lane;
    const bool lvalid = nl < P.N;
    const int64_t dn_l = lvalid ? P.dn[CPLX ? (nl >> 1) : nl] : 0;
    const int ce_l = ((OZ || P.nf_skip) && lvalid) ? P.colexp[nl] : 0;
    // columns left to the non-finite fix-up
    const unsigned skipc = __ballot_sync(0xffffffffu, P.nf_skip && ce_l >= kNonFiniteExp);
    if (!CPLX) {
      using T = typename std::conditional<OZ, double, float>::type;
      T* D = (T*)P.D;
      T old[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int64_t dn = __shfl_sync(0xffffffffu, dn_l, j);
        old[j] = (load_d && mval && n0 + j < P.N) ? D[dmo + dn] : (T)0;
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int64_t dn = __shfl_sync(0xffffffffu, dn_l, j);
        const int ce = __shfl_sync(0xffffffffu, ce_l, j);
        if (!mval || n0 + j >= P.N || ((skipc >> j) & 1u)) continue;
        T v;
        if (OZ) v = (T)(P.ar * scale2((double)(int)r[j], re + ce - shift));
        else v = (T)P.ar * __uint_as_float(r[j]);
        T o;
        if (!first) o = old[j] + v;
        else if (P.br == 0.0) o = v;
        else if (OZ) o = fma((double)P.br, (double)old[j], (double)v);
        else o = fmaf((float)P.br, (float)old[j], (float)v);
        D[dmo + dn] = o;
      }
    } else {
      using T2 = typename std::conditional<OZ, double2, float2>::type;
      using T = typename std::conditional<OZ, double, float>::type;
      T2* D = (T2*)P.D;
      T2 old[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int64_t dn = __shfl_sync(0xffffffffu, dn_l, 2 * j);
        T2 z; z.x = 0; z.y = 0;
        old[j] = (load_d && mval && n0 + 2 * j < P.N) ? D[dmo + dn] : z;
      }
      const T ar = (T)P.ar, ai = (T)P.ai, br = (T)P.br, bi = (T)P.bi;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int64_t dn = __shfl_sync(0xffffffffu, dn_l, 2 * j);
        const int ce = __shfl_sync(0xffffffffu, ce_l, 2 * j);
        if (!mval || n0 + 2 * j >= P.N || ((skipc >> (2 * j)) & 1u)) continue;
        T xr, xi;
        if (OZ) {
          const int e = re + ce - shift;
          xr = (T)scale2((double)(int)r[2 * j], e);
          xi = (T)scale2((double)(int)r[2 * j + 1], e);
        } else {
          xr = __uint_as_float(r[2 * j]);
          xi = __uint_as_float(r[2 * j + 1]);
        }
        T2 v;
        v.x = ar * xr - ai * xi;
        v.y = ar * xi + ai * xr;
        const T2 d = old[j];
        if (first) {
          v.x += br * d.x - bi * d.y;
          v.y += br * d.y + bi * d.x;
        } else {
          v.x += d.x; v.y += d.y;
        }
        D[dmo + dn] = v;
      }
    }
  }
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
  const int nunits = gemm_units<EPI>(P);

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesTC; ++s) { mbar_init(&bars->full[s], 1); mbar_init(&bars->empty[s], 1); }
    for (int a = 0; a < 2; ++a) { mbar_init(&bars->acc_full[a], 1); mbar_init(&bars->acc_empty[a], 4); }
    for (int r = 0; r < kUnitRing; ++r) {
      mbar_init(&bars->unit_full[r], 1);
      mbar_init(&bars->unit_empty[r], kUnitConsumers);
    }
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

  // Next work unit from the ring (-1: no more).  Every consumer takes every
  // unit, in order, and frees the entry after reading it.
  auto take_unit = [&](uint32_t j, bool warp_wide) -> int {
    const int r = (int)(j % kUnitRing);
    const uint32_t ph = (j / kUnitRing) & 1;
    const bool got = warp_wide ? mbar_wait_warp(&bars->unit_full[r], ph, P.err, 1u, kEpilogueSleepNs)
                               : mbar_wait(&bars->unit_full[r], ph, P.err);
    if (!got) { ok = false; return -1; }
    const int u = *(volatile int*)&bars->unit[r];
    if (warp_wide) {
      __syncwarp();  // every lane has read the entry before the warp frees it
      if (lane == 0) mbar_arrive(&bars->unit_empty[r]);
    } else {
      mbar_arrive(&bars->unit_empty[r]);
    }
    return u;
  };

  if (warp == 0) {
    // ---------------- TMA producer and scheduler ----------------
    if (lane == 0) {
      uint64_t pol_a = 0, pol_b = 0;
      if (P.l2hint) { pol_a = l2_policy_evict_first(); pol_b = l2_policy_evict_last(); }
      uint32_t it = 0;
      const uint32_t bytes = 128 * 128 + BN * 128;
      for (uint32_t j = 0; ok; ++j) {
        int u = P.sched ? (int)atomicAdd(P.sched, 1u) : (int)(blockIdx.x + j * gridDim.x);
        if (u >= nunits) u = -1;
        const int r = (int)(j % kUnitRing);
        if (!(ok = mbar_wait(&bars->unit_empty[r], ((j / kUnitRing) & 1) ^ 1, P.err))) break;
        *(volatile int*)&bars->unit[r] = u;
        mbar_arrive(&bars->unit_full[r]);
        if (u < 0) break;
        const GemmUnit w = gemm_unit<EPI>(P, u);
        const int mb = w.t / P.ntiles, nb = w.t - mb * P.ntiles;
        for (int q = P.pass_first[w.p0]; q < P.pass_first[w.p1] && ok; ++q) {
          for (int kb = P.prod_kb0[q]; kb < P.prod_kb1[q]; ++kb, ++it) {
            const int s = it % kStagesTC;
            const uint32_t ph = (it / kStagesTC) & 1;
            if (!(ok = mbar_wait(&bars->empty[s], ph ^ 1, P.err))) break;
            mbar_expect_tx(&bars->full[s], bytes);
            const int kx = kb * (I8 ? 128 : 64);
            if (P.l2hint) {
              tma_load_3d_hint(smA + (size_t)s * 128 * 128, &P.tmA, kx, mb * 128, P.prod_a[q], &bars->full[s], pol_a);
              tma_load_3d_hint(smB + (size_t)s * BN * 128, &P.tmB, kx, nb * BN, P.prod_b[q], &bars->full[s], pol_b);
            } else {
              tma_load_3d(smA + (size_t)s * 128 * 128, &P.tmA, kx, mb * 128, P.prod_a[q], &bars->full[s]);
              tma_load_3d(smB + (size_t)s * BN * 128, &P.tmB, kx, nb * BN, P.prod_b[q], &bars->full[s]);
            }
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t kIdesc = idesc(I8, BN);
      uint32_t it = 0, acc_it = 0;
      for (uint32_t j = 0; ok; ++j) {
        const int u = take_unit(j, false);
        if (u < 0) break;
        const GemmUnit w = gemm_unit<EPI>(P, u);
        for (int p = w.p0; p < w.p1 && ok; ++p, ++acc_it) {
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
    for (uint32_t j = 0; ok; ++j) {
      const int u = take_unit(j, true);
      if (u < 0) break;
      const GemmUnit w = gemm_unit<EPI>(P, u);
      const int mb = w.t / P.ntiles, nb = w.t - mb * P.ntiles;
      const int m = mb * 128 + quad * 32 + lane;
      const int re = ((EPI == EPI_OZAKI_R || EPI == EPI_OZAKI_C) || P.nf_skip) && m < P.M ? P.rowexp[m] : 0;
      const bool mval = m < P.M && !(P.nf_skip && re >= kNonFiniteExp);  // flagged rows: the fix-up's
      const int64_t dmo = mval ? P.dm[m] : 0;
      for (int p = w.p0; p < w.p1 && ok; ++p, ++acc_it) {
        const int a = acc_it & 1;
        const uint32_t aph = (acc_it >> 1) & 1;
        if (!(ok = mbar_wait_warp(&bars->acc_full[a], aph, P.err, 1u, kEpilogueSleepNs))) break;
        tc_fence_after();
        const bool first = EPI == EPI_RESID ? (p - w.p0 == 0) : (p == 0);
        const int shift = (EPI == EPI_OZAKI_R || EPI == EPI_OZAKI_C || EPI == EPI_RESID) ? P.pass_shift[p] : 0;
        const int64_t dmp = EPI == EPI_RESID ? (int64_t)(p / P.res_nch) * P.res_plane + m : dmo;
        epilogue_pass<BN, EPI>(P, tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * BN),
                               EPI == EPI_RESID ? m < P.M : mval, dmp, re, nb, first, shift,
                               EPI == EPI_RESID ? P.pass_magic[p] : 0);
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

// ---------------------------------------------------------------------------
// CTA-pair variant (cluster of 2, tcgen05 cta_group::2): one 256 x BN output
// tile per pair iteration.  CTA r of the pair stages rows [128r, 128r+128) of
// the A tile and rows [r*BN/2, (r+1)*BN/2) of the B tile in its own shared
// memory; CTA 0's MMA thread issues M = 256 MMAs that read both CTAs' halves
// and accumulate rows 128r.. into CTA r's TMEM.  Each CTA stages half as many
// B bytes per MMA as the single-CTA kernel, which halves the L2-to-SM traffic
// for B and leaves room for deeper pipelines.  Barriers:
//   full[s]     CTA 0 only: CTA 0's expect_tx (both halves) + both CTAs' TMA
//   empty[s]    both CTAs: the MMA commit arrives on both (multicast commit)
//   acc_full[a] both CTAs: MMA commit multicast at the end of a pass
//   acc_empty[a] CTA 0: one arrival from each epilogue warp of both CTAs
// TMA loads carry no multicast; every wait is bounded.
template <int BN>
__host__ __device__ constexpr int pair_stages() { return BN == 256 ? 6 : 8; }

struct TcPairBarriers {
  uint64_t full[8];
  uint64_t empty[8];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint32_t tmem_base;
};

template <int BN>
__host__ __device__ constexpr size_t tc2_smem_bytes() {
  return 1024 + (size_t)pair_stages<BN>() * (128 * 128 + (BN / 2) * 128) + sizeof(TcPairBarriers) + 64;
}

template <int BN, bool I8, int EPI>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kTcThreads, 1)
    tc_gemm2_kernel(const __grid_constant__ TcGemmParams P) {
  using namespace sm100;
  constexpr int ST = pair_stages<BN>();
  constexpr uint32_t kA = 128 * 128, kB = (BN / 2) * 128;
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* smA = base;                          // [ST][128 rows][128 B]
  unsigned char* smB = base + (size_t)ST * kA;        // [ST][BN/2 rows][128 B]
  TcPairBarriers* bars = (TcPairBarriers*)(smB + (size_t)ST * kB);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int pair = (int)(blockIdx.x >> 1), npairs = (int)(gridDim.x >> 1);
  const int nunits = gemm_units<EPI>(P);  // mtiles counts 256-row tiles here

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) { mbar_init(&bars->full[s], 1); mbar_init(&bars->empty[s], 1); }
    for (int a = 0; a < 2; ++a) { mbar_init(&bars->acc_full[a], 1); mbar_init(&bars->acc_empty[a], 8); }
    fence_barrier_init();
    prefetch_tmap(&P.tmA);
    prefetch_tmap(&P.tmB);
  }
  if (warp == 1) {
    tmem_alloc2(&bars->tmem_base, 2 * BN);
    tmem_relinquish2();
  }
  tc_fence_before();
  cluster_sync();  // both CTAs' barriers initialised, TMEM allocated
  tc_fence_after();
  const uint32_t tmem = bars->tmem_base;
  bool ok = true;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      const uint32_t full0 = mapa_shared(smem_u32(&bars->full[0]), 0);  // CTA 0's full barriers
      uint32_t it = 0;
      for (int u = pair; u < nunits && ok; u += npairs) {
        const GemmUnit w = gemm_unit<EPI>(P, u);
        const int mb = w.t / P.ntiles, nb = w.t - mb * P.ntiles;
        for (int q = P.pass_first[w.p0]; q < P.pass_first[w.p1] && ok; ++q) {
          for (int kb = P.prod_kb0[q]; kb < P.prod_kb1[q]; ++kb, ++it) {
            const int s = (int)(it % ST);
            const uint32_t ph = (it / ST) & 1;
            if (!(ok = mbar_wait(&bars->empty[s], ph ^ 1, P.err))) break;
            if (rank == 0) mbar_expect_tx(&bars->full[s], 2 * (kA + kB));
            const uint32_t fb = full0 + (uint32_t)(s * sizeof(uint64_t));
            tma_load_3d_pair(smA + (size_t)s * kA, &P.tmA, kb * (I8 ? 128 : 64), mb * 256 + (int)rank * 128,
                             P.prod_a[q], fb);
            tma_load_3d_pair(smB + (size_t)s * kB, &P.tmB, kb * (I8 ? 128 : 64), nb * BN + (int)rank * (BN / 2),
                             P.prod_b[q], fb);
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (CTA 0 only) ----------------
    if (rank == 0 && lane == 0) {
      constexpr uint32_t kIdesc = idesc(I8, BN, 256);
      uint32_t it = 0, acc_it = 0;
      for (int u = pair; u < nunits && ok; u += npairs) {
        const GemmUnit w = gemm_unit<EPI>(P, u);
        for (int p = w.p0; p < w.p1 && ok; ++p, ++acc_it) {
          const int a = acc_it & 1;
          const uint32_t aph = (acc_it >> 1) & 1;
          if (!(ok = mbar_wait(&bars->acc_empty[a], aph ^ 1, P.err))) break;
          tc_fence_after();
          const uint32_t dcol = tmem + (uint32_t)(a * BN);
          bool first = true;
          for (int q = P.pass_first[p]; q < P.pass_first[p + 1] && ok; ++q) {
            for (int kb = P.prod_kb0[q]; kb < P.prod_kb1[q]; ++kb, ++it) {
              const int s = (int)(it % ST);
              const uint32_t ph = (it / ST) & 1;
              if (!(ok = mbar_wait(&bars->full[s], ph, P.err))) break;
              tc_fence_after();
              const uint32_t sa = smem_u32(smA + (size_t)s * kA);
              const uint32_t sb = smem_u32(smB + (size_t)s * kB);
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                mma2<I8>(dcol, sdesc_k128(sa + kk * 32), sdesc_k128(sb + kk * 32), kIdesc,
                         (first && kk == 0) ? 0u : 1u);
              }
              first = false;
              mma_commit2_both(&bars->empty[s]);
            }
          }
          mma_commit2_both(&bars->acc_full[a]);
        }
      }
    }
  } else {
    // ---------------- epilogue (warps 2..5 of both CTAs) ----------------
    const int quad = warp & 3;
    const uint32_t acc_empty0 = mapa_shared(smem_u32(&bars->acc_empty[0]), 0);
    uint32_t acc_it = 0;
    for (int u = pair; u < nunits && ok; u += npairs) {
      const GemmUnit w = gemm_unit<EPI>(P, u);
      const int mb = w.t / P.ntiles, nb = w.t - mb * P.ntiles;
      const int m = mb * 256 + (int)rank * 128 + quad * 32 + lane;
      const int re = ((EPI == EPI_OZAKI_R || EPI == EPI_OZAKI_C) || P.nf_skip) && m < P.M ? P.rowexp[m] : 0;
      const bool mval = m < P.M && !(P.nf_skip && re >= kNonFiniteExp);  // flagged rows: the fix-up's
      const int64_t dmo = mval ? P.dm[m] : 0;
      for (int p = w.p0; p < w.p1 && ok; ++p, ++acc_it) {
        const int a = acc_it & 1;
        const uint32_t aph = (acc_it >> 1) & 1;
        if (!(ok = mbar_wait_warp(&bars->acc_full[a], aph, P.err, 1u, kEpilogueSleepNs))) break;
        tc_fence_after();
        const int shift = (EPI == EPI_OZAKI_R || EPI == EPI_OZAKI_C || EPI == EPI_RESID) ? P.pass_shift[p] : 0;
        const int64_t dmp = EPI == EPI_RESID ? (int64_t)(p / P.res_nch) * P.res_plane + m : dmo;
        epilogue_pass<BN, EPI>(P, tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * BN),
                               EPI == EPI_RESID ? m < P.M : mval, dmp, re, nb,
                               EPI == EPI_RESID ? (p - w.p0 == 0) : (p == 0), shift,
                               EPI == EPI_RESID ? P.pass_magic[p] : 0);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(acc_empty0 + (uint32_t)(a * sizeof(uint64_t)));
      }
    }
  }
  __syncthreads();
  tc_fence_before();
  cluster_sync();  // neither CTA touches the other's barriers or TMEM after this
  tc_fence_after();
  if (warp == 1) tmem_dealloc2(tmem, 2 * BN);
}

}  // namespace tb
