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
// output tile; pairs that share an output block therefore never race.  Roles as in tc_gemm_kernel:
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

struct __align__(16) BscLOp {   // left operand block (A planes)
  const CUtensorMap* map;       // (Kpad, Mpad, planes)
  const int* rowexp;            // INT8 slices: per-row scale exponents
  int kblocks;                  // 128-byte K blocks
  int pad_;
};
struct __align__(16) BscROp {   // right operand block (B planes)
  const CUtensorMap* map;       // (Kpad, Npad, planes)
  const int* colexp;
  int kblocks;
  int pad_;
};
struct __align__(16) BscDBlk {  // output block
  void* D;
  const int64_t* dm;            // D offset of row m
  const int64_t* dn;            // D offset of column n
  int M, N;
  int pass0, npass;             // its accumulator passes: passes[pass0 .. pass0 + npass)
};
struct BscPair { int l, r; };
struct BscItem { int d, mt, nt, pad_; };
// A pass is one exact TMEM accumulator: chunks[chunk0 .. chunk0 + nchunk),
// each the product of plane a of A and plane b of B summed over the pairs
// pairs[p0 .. p1) of the output block (all their K blocks).  INT8 slices: the
// pass's weight is 2^-shift; the operand blocks of one output block share
// their row (column) scales, so their products add up exactly in INT32.
struct BscPass { int chunk0, nchunk, shift, pad_; };
// kb1 > 0: the chunk covers only pair p0, over its K blocks [kb0, kb1)
// (split-BF16 passes end inside a pair's K range); else all K blocks of the
// pairs p0 .. p1 - 1.
struct BscChunk { int a, b, p0, p1, kb0, kb1; };

constexpr int kBscRing = 4;

struct __align__(64) BscParams {
  const BscLOp* lops;
  const BscROp* rops;
  const BscDBlk* dblks;
  const BscPair* pairs;
  const BscItem* items;
  const BscPass* passes;
  const BscChunk* chunks;
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
  unsigned char* smB = base + (size_t)kStagesTC * 128 * 128;
  BscSmemBarriers* bars = (BscSmemBarriers*)(smB + (size_t)kStagesTC * BN * 128);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesTC; ++s) { mbar_init(&bars->full[s], 1); mbar_init(&bars->empty[s], 1); }
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
        for (int p = Dd.pass0; p < Dd.pass0 + Dd.npass && ok; ++p) {
          const BscPass ps = P.passes[p];
          for (int c = ps.chunk0; c < ps.chunk0 + ps.nchunk && ok; ++c) {
            const BscChunk ch = P.chunks[c];
            for (int pp = ch.p0; pp < ch.p1 && ok; ++pp) {
              const BscPair pr = P.pairs[pp];
              const BscLOp lo = P.lops[pr.l];
              const CUtensorMap* rmap = P.rops[pr.r].map;
              const int kbeg = ch.kb1 > 0 ? ch.kb0 : 0, kend = ch.kb1 > 0 ? ch.kb1 : lo.kblocks;
              for (int kb = kbeg; kb < kend; ++kb, ++it) {
                const int s = (int)(it % kStagesTC);
                const uint32_t ph = (it / kStagesTC) & 1;
                if (!(ok = mbar_wait(&bars->empty[s], ph ^ 1, P.err, 12u))) break;
                mbar_expect_tx(&bars->full[s], 128 * 128 + BN * 128);
                tma_load_3d(smA + (size_t)s * 128 * 128, lo.map, kb * (I8 ? 128 : 64), I.mt * 128, ch.a,
                            &bars->full[s]);
                tma_load_3d(smB + (size_t)s * BN * 128, rmap, kb * (I8 ? 128 : 64), I.nt * BN, ch.b,
                            &bars->full[s]);
              }
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
      for (uint32_t k = 0; ok; ++k) {
        const int slot = (int)(k % kBscRing);
        if (!(ok = mbar_wait(&bars->item_full[slot], (k / kBscRing) & 1, P.err, 13u))) break;
        const int cur = bars->ring[slot];
        if (cur < 0) break;
        const BscItem I = P.items[cur];
        const BscDBlk Dd = P.dblks[I.d];
        for (int p = Dd.pass0; p < Dd.pass0 + Dd.npass && ok; ++p, ++acc_it) {
          const BscPass ps = P.passes[p];
          const int a = acc_it & 1;
          const uint32_t aph = (acc_it >> 1) & 1;
          if (!(ok = mbar_wait(&bars->acc_empty[a], aph ^ 1, P.err, 14u))) break;
          tc_fence_after();
          const uint32_t dcol = tmem + (uint32_t)(a * BN);
          bool first = true;
          for (int c = ps.chunk0; c < ps.chunk0 + ps.nchunk && ok; ++c) {
            const BscChunk ch = P.chunks[c];
            for (int pp = ch.p0; pp < ch.p1 && ok; ++pp) {
              const int kblocks = P.lops[P.pairs[pp].l].kblocks;
              const int kbeg = ch.kb1 > 0 ? ch.kb0 : 0, kend = ch.kb1 > 0 ? ch.kb1 : kblocks;
              for (int kb = kbeg; kb < kend; ++kb, ++it) {
                const int s = (int)(it % kStagesTC);
                const uint32_t ph = (it / kStagesTC) & 1;
                if (!(ok = mbar_wait(&bars->full[s], ph, P.err, 15u))) break;
                tc_fence_after();
                const uint32_t sa = smem_u32(smA + (size_t)s * 128 * 128);
                const uint32_t sb = smem_u32(smB + (size_t)s * BN * 128);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                  mma<I8>(dcol, sdesc_k128(sa + kk * 32), sdesc_k128(sb + kk * 32), kIdesc,
                          (first && kk == 0) ? 0u : 1u);
                first = false;
                mma_commit(&bars->empty[s]);
              }
            }
          }
          mma_commit(&bars->acc_full[a]);
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
      const BscPair pr0 = P.pairs[P.chunks[P.passes[Dd.pass0].chunk0].p0];
      const int re = (EPI == EPI_OZAKI_R) && mval ? P.lops[pr0.l].rowexp[m] : 0;
      const EpiView V{Dd.D, Dd.dn, P.rops[pr0.r].colexp, Dd.N, P.ar, P.ai, P.br, P.bi, 0};
      for (int p = Dd.pass0; p < Dd.pass0 + Dd.npass && ok; ++p, ++acc_it) {
        const int a = acc_it & 1;
        const uint32_t aph = (acc_it >> 1) & 1;
        if (!(ok = mbar_wait_warp(&bars->acc_full[a], aph, P.err, 17u))) break;
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
