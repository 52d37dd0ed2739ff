// tb_bsc_gemm.cuh -- persistent grouped tcgen05 GEMM for block-sparse
// contractions: every output block D_d accumulates the products of its
// (L block, R block) pairs,
//   D_d = beta*D_d + alpha * sum_{p in pairs(d)} L_p * R_p,
// with the operands already converted to K-major planes (INT8 slices of FP64
// data or BF16 parts of FP32 data, one tensor map per operand block).
//
// Work items are (output block, 128-row tile, BN-column tile), ordered by
// decreasing cost; CTAs take them from a device-side queue (one atomic counter)
// so that the uneven blocks balance across the SMs.  A work item sums all its
// pairs inside each TMEM accumulator pass (the operand blocks of an output
// block share row and column scales, so that INT32 sums over several pairs
// stay exact) and hands each pass to the epilogue, which adds it into the
// output tile; pairs that share an output block therefore never race.  The
// host flattens each output block's passes into runs (one pair's K range in
// one plane pair, with its tensor maps), so that the producer and the MMA
// issuer read one record per run, fetched two runs ahead, instead of chasing
// pass -> chunk -> pair -> operand records at every pair boundary.  Roles as
// in tc_gemm_kernel:
//   warp 0   queue + TMA producer (one lane); it publishes every item it takes
//            in a small shared-memory ring read by the other roles
//   warp 1   TMEM allocation and the single MMA-issuing thread
//   warps 2-5 epilogue
// Every wait is bounded; one that gives up records its site in the device
// error word: 11/12 producer (item slot, stage), 13/14/15 MMA issuer (item,
// accumulator, stage), 16/17 epilogue (item, accumulator).
#pragma once
#include "tb_tc_gemm.cuh"

namespace tb {

struct __align__(16) BscDBlk {  // output block
  void* D;
  const int64_t* dm;            // D offset of row m
  const int64_t* dn;            // D offset of column n
  const int* rowexp;            // INT8 slices: per-row scale exponents (shared by the block's A blocks)
  const int* colexp;            // INT8 slices: per-column scale exponents (shared by its B blocks)
  int M, N;
  int pass0, npass;             // its accumulator passes: passes[pass0 .. pass0 + npass)
  int run0, nrun;               // its runs: runs[run0 .. run0 + nrun), pass after pass
};
struct BscItem { int d, mt, nt, pad_; };
// A pass is one exact TMEM accumulator that the epilogue adds into the output
// tile.  INT8 slices: its weight is 2^-shift; the operand blocks of one output
// block share their row (column) scales, so products of several block pairs
// add up exactly in INT32 within a pass.
struct BscPass { int run0, nrun, shift, pad_; };
// A run is what the producer streams without looking anything up: K blocks
// [kb0, kb1) of plane a of one A block and plane b of one B block (tensor maps
// for both N tiles).  The runs of an output block are flat, pass after pass;
// flags mark the first and the last run of each pass.
constexpr int kBscRunFirst = 1, kBscRunLast = 2;
struct __align__(16) BscRun {
  const CUtensorMap* amap;      // (Kpad, Mpad, planes)
  const CUtensorMap* bmap[2];   // (Kpad, Npad, planes), boxes for BN = 128 / 256
  int a, b;                     // planes
  int kb0, kb1;                 // 128-byte K blocks
  int flags;
  int pad_;
};

constexpr int kBscRing = 4;

struct __align__(64) BscParams {
  const BscDBlk* dblks;
  const BscItem* items;
  const BscPass* passes;
  const BscRun* runs;
  unsigned int* queue;          // next item (zeroed before every launch)
  int nitems;
  double ar, ai, br, bi;        // beta applies to the first pass of each tile
  unsigned int* err;
};

struct BscSmemBarriers {
  uint64_t full[kStagesTC];
  uint64_t empty[kStagesTC];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint64_t item_full[kBscRing];
  uint64_t item_empty[kBscRing];
  int ring[kBscRing];
  uint32_t tmem_base;
};

template <int BN>
__host__ __device__ constexpr size_t bsc_smem_bytes() {
  return 1024 + (size_t)kStagesTC * (128 * 128 + BN * 128) + sizeof(BscSmemBarriers) + 64;
}

template <int BN, bool I8, int EPI>
__global__ void __launch_bounds__(kTcThreads, 1) bsc_gemm_kernel(const __grid_constant__ BscParams P) {
  using namespace sm100;
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* smA = base;
  constexpr int kStages = kStagesTC;
  unsigned char* smB = base + (size_t)kStages * 128 * 128;
  BscSmemBarriers* bars = (BscSmemBarriers*)(smB + (size_t)kStages * BN * 128);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) { mbar_init(&bars->full[s], 1); mbar_init(&bars->empty[s], 1); }
    for (int a = 0; a < 2; ++a) { mbar_init(&bars->acc_full[a], 1); mbar_init(&bars->acc_empty[a], 4); }
    for (int s = 0; s < kBscRing; ++s) { mbar_init(&bars->item_full[s], 1); mbar_init(&bars->item_empty[s], 5); }
    fence_barrier_init();
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
    // ---------------- queue + TMA producer ----------------
    if (lane == 0) {
      uint32_t it = 0;
      for (uint32_t k = 0; ok; ++k) {
        const int slot = (int)(k % kBscRing);
        if (!(ok = mbar_wait(&bars->item_empty[slot], ((k / kBscRing) & 1) ^ 1, P.err, 11u))) break;
        const int item = (int)atomicAdd(P.queue, 1u);
        const int cur = item < P.nitems ? item : -1;
        bars->ring[slot] = cur;
        mbar_arrive(&bars->item_full[slot]);  // release: the ring entry is visible to the waiters
        if (cur < 0) break;
        const BscItem I = P.items[cur];
        const BscDBlk Dd = P.dblks[I.d];
        // software pipeline over the runs: the record of run r + 1 was loaded
        // during run r - 1 and its tensor maps are prefetched now; the record
        // of run r + 2 loads while run r streams
        const int rend = Dd.run0 + Dd.nrun;
        BscRun ru = P.runs[Dd.run0];
        BscRun n1 = Dd.nrun > 1 ? P.runs[Dd.run0 + 1] : ru;
        prefetch_tmap(ru.amap);
        prefetch_tmap(ru.bmap[BN == 256]);
        for (int r = Dd.run0; r < rend && ok; ++r) {
          if (r + 1 < rend) {
            prefetch_tmap(n1.amap);
            prefetch_tmap(n1.bmap[BN == 256]);
          }
          const BscRun n2 = r + 2 < rend ? P.runs[r + 2] : n1;
          const CUtensorMap* bmap = ru.bmap[BN == 256];
          for (int kb = ru.kb0; kb < ru.kb1; ++kb, ++it) {
            const int s = (int)(it % kStages);
            const uint32_t ph = (it / kStages) & 1;
            if (!(ok = mbar_wait(&bars->empty[s], ph ^ 1, P.err, 12u))) break;
            mbar_expect_tx(&bars->full[s], 128 * 128 + BN * 128);
            tma_load_3d(smA + (size_t)s * 128 * 128, ru.amap, kb * (I8 ? 128 : 64), I.mt * 128, ru.a, &bars->full[s]);
            tma_load_3d(smB + (size_t)s * BN * 128, bmap, kb * (I8 ? 128 : 64), I.nt * BN, ru.b, &bars->full[s]);
          }
          ru = n1;
          n1 = n2;
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t kIdesc = idesc(I8, BN);
      uint32_t it = 0, acc_it = 0;
      for (uint32_t k = 0; ok; ++k) {
        const int slot = (int)(k % kBscRing);
        if (!(ok = mbar_wait(&bars->item_full[slot], (k / kBscRing) & 1, P.err, 13u))) break;
        const int cur = bars->ring[slot];
        if (cur < 0) break;
        const BscDBlk Dd = P.dblks[P.items[cur].d];
        const int rend = Dd.run0 + Dd.nrun;
        int2 ru = make_int2(0, 0), n1 = ru;  // (kb1 - kb0, flags) of runs r and r + 1
        {
          const BscRun x = P.runs[Dd.run0];
          ru = make_int2(x.kb1 - x.kb0, x.flags);
          if (Dd.nrun > 1) { const BscRun y = P.runs[Dd.run0 + 1]; n1 = make_int2(y.kb1 - y.kb0, y.flags); }
        }
        uint32_t dcol = 0;
        bool first = true;
        for (int r = Dd.run0; r < rend && ok; ++r) {
          int2 n2 = n1;
          if (r + 2 < rend) { const BscRun z = P.runs[r + 2]; n2 = make_int2(z.kb1 - z.kb0, z.flags); }
          const int a = acc_it & 1;
          if (ru.y & kBscRunFirst) {
            const uint32_t aph = (acc_it >> 1) & 1;
            if (!(ok = mbar_wait(&bars->acc_empty[a], aph ^ 1, P.err, 14u))) break;
            tc_fence_after();
            dcol = tmem + (uint32_t)(a * BN);
            first = true;
          }
          for (int kb = 0; kb < ru.x; ++kb, ++it) {
            const int s = (int)(it % kStages);
            const uint32_t ph = (it / kStages) & 1;
            if (!(ok = mbar_wait(&bars->full[s], ph, P.err, 15u))) break;
            tc_fence_after();
            const uint32_t sa = smem_u32(smA + (size_t)s * 128 * 128);
            const uint32_t sb = smem_u32(smB + (size_t)s * BN * 128);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
              mma<I8>(dcol, sdesc_k128(sa + kk * 32), sdesc_k128(sb + kk * 32), kIdesc, (first && kk == 0) ? 0u : 1u);
            first = false;
            mma_commit(&bars->empty[s]);
          }
          if (ok && (ru.y & kBscRunLast)) {
            mma_commit(&bars->acc_full[a]);
            ++acc_it;
          }
          ru = n1;
          n1 = n2;
        }
        mbar_arrive(&bars->item_empty[slot]);
      }
    }
  } else {
    // ---------------- epilogue (warps 2..5) ----------------
    const int quad = warp & 3;
    uint32_t acc_it = 0;
    for (uint32_t k = 0; ok; ++k) {
      const int slot = (int)(k % kBscRing);
      if (!(ok = mbar_wait_warp(&bars->item_full[slot], (k / kBscRing) & 1, P.err, 16u))) break;
      const int cur = bars->ring[slot];
      if (cur < 0) break;
      const BscItem I = P.items[cur];
      const BscDBlk Dd = P.dblks[I.d];
      const int m = I.mt * 128 + quad * 32 + lane;
      const bool mval = m < Dd.M;
      const int64_t dmo = mval ? Dd.dm[m] : 0;
      // all pairs of an output block share its row and column scales
      const int re = (EPI == EPI_OZAKI_R) && mval ? Dd.rowexp[m] : 0;
      const EpiView V{Dd.D, Dd.dn, Dd.colexp, Dd.N, P.ar, P.ai, P.br, P.bi, 0};
      for (int p = Dd.pass0; p < Dd.pass0 + Dd.npass && ok; ++p, ++acc_it) {
        const int a = acc_it & 1;
        const uint32_t aph = (acc_it >> 1) & 1;
        if (!(ok = mbar_wait_warp(&bars->acc_full[a], aph, P.err, 17u, kEpilogueSleepNs))) break;
        tc_fence_after();
        const int shift = (EPI == EPI_OZAKI_R) ? P.passes[p].shift : 0;
        epilogue_pass<BN, EPI>(V, tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * BN), mval, dmo, re, I.nt,
                               p == Dd.pass0, shift);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&bars->acc_empty[a]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars->item_empty[slot]);
    }
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * BN);
  }
}

}  // namespace tb
