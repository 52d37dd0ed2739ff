// tb_permute.cuh -- tiled permutation engine (plan builder + kernel template).
//
// A permutation moves every element of a dense tensor to a new position.  The
// kernel stages one tile of the tensor in shared memory: the tile is a box
// whose input-fastest dimensions give contiguous input runs of at least
// 128 bytes ("load chunks") and whose output-fastest dimensions give
// contiguous output runs of at least 128 bytes ("store chunks"), so that
// both the HBM reads and the HBM writes are full-line coalesced whatever the
// permutation.  Chunk base offsets and the shared-memory transposition map
// are precomputed on the host once per plan and passed as a kernel parameter.
// The store side is a functor, so the same engine performs plain copies,
// conjugating copies, the fused permute+add, and the gather/convert passes
// that feed the tensor-core contraction.
#pragma once
#include "tb_common.cuh"
#include "tb_perm_plan.h"
#include "tb_sm100.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>

namespace tb {

constexpr int kPermThreads = 256;

// ---------------------------------------------------------------------------
// Pipelined kernel.  Each CTA walks its tiles through kStages shared-memory
// buffers.  Loads are asynchronous so that many bytes are in flight per SM:
//   BULK:  one thread issues a TMA bulk copy (cp.async.bulk) per load row,
//          completion counted in bytes on the stage's mbarrier;
//   !BULK: every thread issues element-sized cp.async copies (any alignment),
//          completion tracked with cp.async groups.
// The store phase reads the tile in output order and hands each element to
// the Store functor:  __device__ void operator()(int64_t out_off, const Elem&).
// ---------------------------------------------------------------------------
constexpr int kStages = 3;

struct PermSmem {
  int64_t ld_base[kMaxChunks];
  int64_t st_base[kMaxChunks];
  int32_t st_ebase[kMaxChunks];
  int32_t ejf[kMaxEjf];
  int16_t ld_dpb[kMaxChunks];
  int16_t st_dpa[kMaxChunks];
  unsigned long long mbar[kStages];
};

inline size_t perm_smem_bytes(const PermParams& P) {
  return ((sizeof(PermSmem) + 127) & ~size_t(127)) + (size_t)kStages * (size_t)perm_stage_bytes(P) + 128;
}

struct TileOrigin {
  int64_t in_base, out_base;
  int rem_a, rem_b;
  bool full;
};

__device__ __forceinline__ TileOrigin tile_origin(const PermParams& P, int64_t tile) {
  TileOrigin o{0, 0, 1 << 30, 1 << 30, true};
  uint64_t r = (uint64_t)tile;
  for (int g = 0; g < P.ngd; ++g) {
    const uint64_t q = P.gd32 ? (uint64_t)fdiv32((uint32_t)r, P.gmag[g], P.gsh[g]) : P.gdiv[g].div(r);
    const int64_t x = (int64_t)(r - q * (uint64_t)P.gext[g]);
    r = q;
    const int d = P.gdim[g];
    const int64_t org = x * P.tile[d];
    o.in_base += org * P.sin[d];
    o.out_base += org * P.sout[d];
    const int64_t rem = P.dims[d] - org;
    if (d == P.pa) o.rem_a = (int)(rem < P.tile[d] ? rem : P.tile[d]);
    if (d == P.pb) o.rem_b = (int)(rem < P.tile[d] ? rem : P.tile[d]);
  }
  o.full = (P.pa < 0 || o.rem_a >= P.tile[P.pa]) && (P.pb < 0 || o.rem_b >= P.tile[P.pb]);
  return o;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Loads one tile into a stage buffer (see the BULK / !BULK note above).
// !BULK: each warp copies whole rows (lanes along the row, 16-byte copies
// when rows are 16-byte aligned, element copies otherwise).
template <typename Elem, bool BULK, bool COMMIT = true>
__device__ __forceinline__ void perm_issue(const PermParams& P, const PermSmem& T, const Elem* in, Elem* stage,
                                           unsigned long long* bar, int64_t tile) {
  const TileOrigin o = tile_origin(P, tile);
  int len = P.LA;  // valid row length (elements) of this tile
  if (!o.full && P.pa >= 0) len = P.prodA * (P.pb == P.pa ? min(o.rem_a, o.rem_b) : o.rem_a);
  const bool rowcheck = !o.full && P.pb >= 0 && P.pb != P.pa;
  if (BULK) {
    if (threadIdx.x != 0) return;
    const uint32_t bytes = (uint32_t)(((int64_t)len * (int64_t)sizeof(Elem) + 15) & ~int64_t(15));
    uint32_t total = 0;
    for (int c = 0; c < P.nA; ++c)
      if (!rowcheck || T.ld_dpb[c] < o.rem_b) total += bytes;
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(total)
                 : "memory");
    for (int c = 0; c < P.nA; ++c) {
      if (rowcheck && T.ld_dpb[c] >= o.rem_b) continue;
      const Elem* src = in + o.in_base + T.ld_base[c];
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
              smem_addr(stage + (size_t)c * P.lap)),
          "l"(src), "r"(bytes), "r"(smem_addr(bar))
          : "memory");
    }
  } else {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int kW = kPermThreads / 32, kU = 4;  // copies per lane per unit
    // vector copies need rows that are whole vectors (the plan) on an aligned tensor
    const bool vec = P.tma_ok && sizeof(Elem) < 16 && (uintptr_t)in % 16 == 0;
    const bool vec8 = !vec && P.vec8 && sizeof(Elem) < 8 && (uintptr_t)in % 8 == 0;
    constexpr int VW = sizeof(Elem) < 16 ? 16 / sizeof(Elem) : 1;
    constexpr int VW8 = sizeof(Elem) < 8 ? 8 / sizeof(Elem) : 1;
    const int w = vec ? VW : (vec8 ? VW8 : 1);         // elements per copy
    const int nvec = (len + w - 1) / w;                // copies per row (vector rows round up)
    const int nseg = (nvec + 32 * kU - 1) / (32 * kU);
    const int units = P.nA * nseg;
    for (int u = warp; u < units; u += kW) {
      const int c = u / nseg, sg = u - c * nseg;
      if (rowcheck && T.ld_dpb[c] >= o.rem_b) continue;
      const Elem* src = in + o.in_base + T.ld_base[c];
      Elem* dst = stage + (size_t)c * P.lap;
#pragma unroll
      for (int uu = 0; uu < kU; ++uu) {
        const int v = (sg * kU + uu) * 32 + lane;
        if (v >= nvec) break;
        const int j = v * w;
        if (vec || sizeof(Elem) == 16)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst + j)), "l"(src + j)
                       : "memory");
        else if (vec8)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(dst + j)), "l"(src + j)
                       : "memory");
        else
          asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_addr(dst + j)), "l"(src + j),
                       "n"(sizeof(Elem))
                       : "memory");
      }
    }
    if (COMMIT) asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
}

// Store phase.  Work units are (store chunk, block of positions); lanes are
// grouped LPC to a unit and step through the block LPC positions at a time.
// Position j of a chunk lives at ejf[j % prodB] + (j / prodB) * stride; the
// common single-dimension store block (prodB == 1) needs one multiply.
constexpr int kStoreBlock = 512;

struct StoreLanes {
  int lpc, sub, l, cpw;  // lanes per unit, unit slot in the warp, lane in unit, units per warp step
  int blk, nblk;         // positions per block (a multiple of prodB), blocks per chunk
};

__device__ __forceinline__ void store_lanes_init(const PermParams& P, StoreLanes& S) {
  const int lane = threadIdx.x & 31;
  S.lpc = P.LB >= 24 ? 32 : (P.LB >= 12 ? 16 : 8);
  S.cpw = 32 / S.lpc;
  S.sub = lane / S.lpc;
  S.l = lane % S.lpc;
  S.blk = P.LB <= kStoreBlock ? P.LB : (kStoreBlock / P.ejf_n) * P.ejf_n;
  S.nblk = (P.LB + S.blk - 1) / S.blk;
}

template <typename Elem, typename Store>
__device__ __forceinline__ void perm_store(const PermParams& P, const PermSmem& T, const StoreLanes& S,
                                           const Elem* stage, int64_t tile, const Store& st) {
  const TileOrigin o = tile_origin(P, tile);
  const int warp = threadIdx.x >> 5;
  constexpr int kW = kPermThreads / 32;
  const int LB = P.LB, pB = P.ejf_n, stride = P.ej_pb_stride;
  const int qlim = (!o.full && P.pb >= 0) ? (P.pa == P.pb ? min(o.rem_a, o.rem_b) : o.rem_b) : (1 << 30);
  const bool dpa_check = !o.full && P.pa >= 0 && P.pa != P.pb;
  const int units = P.nB * S.nblk;
  for (int u = warp * S.cpw + S.sub; u < units; u += kW * S.cpw) {
    const int c = S.nblk == 1 ? u : u / S.nblk;
    const int j0 = (u - c * S.nblk) * S.blk;
    if (dpa_check && T.st_dpa[c] >= o.rem_a) continue;
    const int64_t ob = o.out_base + T.st_base[c];
    const Elem* sb = stage + T.st_ebase[c];
    const int jmax = min(j0 + S.blk, LB);
    if (pB == 1) {
      const int jlim = min(jmax, qlim);
#pragma unroll 4
      for (int j = j0 + S.l; j < jlim; j += S.lpc) st(ob + j, sb[j * stride]);
    } else {
#pragma unroll 2
      for (int j = j0 + S.l; j < jmax; j += S.lpc) {
        const int q = (int)fdiv32((uint32_t)j, P.pb_magic, P.pb_shift);
        if (q >= qlim) break;  // q is non-decreasing in j
        st(ob + j, sb[T.ejf[j - q * pB] + q * stride]);
      }
    }
  }
}

template <typename Elem, typename Store, bool BULK>
__global__ void __launch_bounds__(kPermThreads)
perm_pipe_kernel(const __grid_constant__ PermParams P, const Elem* __restrict__ in, Store st, unsigned int* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PermSmem& T = *reinterpret_cast<PermSmem*>(smem_raw);
  Elem* bufs = reinterpret_cast<Elem*>(smem_raw + ((sizeof(PermSmem) + 127) & ~size_t(127)));
  const size_t stage_elems = (size_t)P.nA * P.lap;
  const int tid = threadIdx.x;
  for (int i = tid; i < P.nA; i += kPermThreads) { T.ld_base[i] = P.ld_base[i]; T.ld_dpb[i] = P.ld_dpb[i]; }
  for (int i = tid; i < P.nB; i += kPermThreads) {
    T.st_base[i] = P.st_base[i]; T.st_ebase[i] = P.st_ebase[i]; T.st_dpa[i] = P.st_dpa[i];
  }
  for (int i = tid; i < P.ejf_n; i += kPermThreads) T.ejf[i] = P.ejf[i];
  if (BULK && tid == 0) {
    for (int s = 0; s < kStages; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(&T.mbar[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  StoreLanes SL;
  store_lanes_init(P, SL);
  const int64_t first = blockIdx.x, step = gridDim.x;
  const int64_t mine = first < P.ntiles ? (P.ntiles - 1 - first) / step + 1 : 0;
  for (int k = 0; k < kStages - 1; ++k) {
    if (k < mine) perm_issue<Elem, BULK>(P, T, in, bufs + (size_t)k * stage_elems, &T.mbar[k], first + k * step);
    else if (!BULK) asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  bool failed = false;
  int64_t k = 0;
  for (; k < mine; ++k) {
    const int stg = (int)(k % kStages);
    if (BULK) {
      // Every thread waits for the stage itself (its wait makes the bulk
      // copies' bytes visible to it); the wait is bounded in time (about two
      // seconds on the global timer) and the decision to give up is taken for
      // the whole CTA at once, so that no thread leaves the others behind at
      // a barrier.
      const uint32_t parity = (uint32_t)((k / kStages) & 1);
      const bool ok = sm100::mbar_wait(reinterpret_cast<uint64_t*>(&T.mbar[stg]), parity, nullptr);
      if (__syncthreads_or(ok ? 0 : 1)) { failed = true; break; }
    } else {
      asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 2) : "memory");
      __syncthreads();
    }
    const int64_t nk = k + kStages - 1;
    const int nstg = (int)(nk % kStages);
    if (nk < mine) perm_issue<Elem, BULK>(P, T, in, bufs + (size_t)nstg * stage_elems, &T.mbar[nstg], first + nk * step);
    else if (!BULK) asm volatile("cp.async.commit_group;\n" ::: "memory");
    perm_store<Elem, Store>(P, T, SL, bufs + (size_t)stg * stage_elems, first + k * step, st);
  }
  if (failed) {
    // leave no bulk copy in flight into this CTA's shared memory: wait, again
    // bounded, for the stages still loading (tiles k .. k + kStages - 2)
    if (threadIdx.x == 0)
      for (int64_t j = k; j < mine && j < k + kStages - 1; ++j)
        sm100::mbar_wait(reinterpret_cast<uint64_t*>(&T.mbar[j % kStages]), (uint32_t)((j / kStages) & 1), nullptr);
    __syncthreads();
    record_device_error(err, 1u);
    return;
  }
  if (!BULK) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Two-dimensional tiles (PermParams::lin2d): every load row and every store
// chunk is one step of a single dimension, so their offsets are c * stride and
// the kernel needs no chunk tables.
//
// Full tiles (all but those at the tensor's edges) run on per-thread offset
// lists (perm_list_entry): a thread's copies sit at the same tile-relative
// offsets in every full tile, so the kernel computes them once, keeps them in
// registers and its loops are unrolled loads and stores at base + offset.
// One thread computes each tile's origin, one tile ahead, into a ring of
// headers in shared memory.  Partial tiles, and plans whose lists do not fit
// (perm2d_list_entries == 0), take the general code:
//   perm2d_issue / perm2d_store    warps take whole rows (lanes along the row)
//                                  and whole chunks (lanes along the run);
//   perm2dv_issue                  the CTA walks (row, vector) pairs;
//   perm2dv_store                  each lane reads VB bytes = VB / es adjacent
//                                  columns (store chunks) of one row and writes
//                                  that many output runs.
// Rows in shared memory are an odd number of 16-byte units long where the
// plan allows it, so a warp's vector reads down a column spread over the banks.
// ---------------------------------------------------------------------------
template <typename Elem>
__device__ __forceinline__ void perm2d_issue(const PermParams& P, const Elem* in, Elem* stage, const TileOrigin& o) {
  int len = P.LA;
  if (!o.full && P.pa >= 0) len = P.prodA * (P.pb == P.pa ? min(o.rem_a, o.rem_b) : o.rem_a);
  int rows = P.nA;
  if (!o.full && P.pb >= 0 && P.pb != P.pa && P.row_is_pb) rows = min(rows, o.rem_b);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kW = kPermThreads / 32;
  // vector copies need rows that are whole vectors (the plan) on an aligned tensor
  const bool vec = P.tma_ok && sizeof(Elem) < 16 && (uintptr_t)in % 16 == 0;
  const bool vec8 = !vec && P.vec8 && sizeof(Elem) < 8 && (uintptr_t)in % 8 == 0;
  constexpr int VW = sizeof(Elem) < 16 ? 16 / sizeof(Elem) : 1;
  constexpr int VW8 = sizeof(Elem) < 8 ? 8 / sizeof(Elem) : 1;
  const int w = vec ? VW : (vec8 ? VW8 : 1);
  const int nvec = (len + w - 1) / w;
  for (int r = warp; r < rows; r += kW) {
    const Elem* src = in + o.in_base + (int64_t)r * P.row_sin;
    Elem* dst = stage + (size_t)r * P.lap;
    for (int v = lane; v < nvec; v += 32) {
      const int j = v * w;
      if (vec || sizeof(Elem) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst + j)), "l"(src + j) : "memory");
      else if (vec8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(dst + j)), "l"(src + j) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_addr(dst + j)), "l"(src + j),
                     "n"(sizeof(Elem))
                     : "memory");
    }
  }
}

template <typename Elem, typename Store>
__device__ __forceinline__ void perm2d_store(const PermParams& P, const Elem* stage, const TileOrigin& o,
                                             const Store& st) {
  const int qlim = (!o.full && P.pb >= 0) ? (P.pa == P.pb ? min(o.rem_a, o.rem_b) : o.rem_b) : (1 << 30);
  int chunks = P.nB;
  if (!o.full && P.pa >= 0 && P.pa != P.pb && P.chunk_is_pa) chunks = min(chunks, o.rem_a);
  const int jlim = min(P.LB, qlim);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kW = kPermThreads / 32;
  const int pstride = P.ej_pb_stride;
  for (int c = warp; c < chunks; c += kW) {
    const int64_t ob = o.out_base + (int64_t)c * P.chunk_sout;
    const Elem* sb = stage + (size_t)c * P.chunk_eb;
#pragma unroll 2
    for (int j = lane; j < jlim; j += 32) st(ob + j, sb[j * pstride]);
  }
}

template <typename Elem, int VB>
__device__ __forceinline__ void perm2dv_issue(const PermParams& P, const Elem* in, Elem* stage, const TileOrigin& o) {
  int len = P.LA;
  if (!o.full && P.pa >= 0) len = P.prodA * (P.pb == P.pa ? min(o.rem_a, o.rem_b) : o.rem_a);
  int rows = P.nA;
  if (!o.full && P.pb >= 0 && P.pb != P.pa && P.row_is_pb) rows = min(rows, o.rem_b);
  constexpr int VW = VB / (int)sizeof(Elem);
  const int nv = (len + VW - 1) / VW;  // valid vectors of a row in this tile
  const int total = rows * P.nvec;
  const Elem* src0 = in + o.in_base;
  for (int v = threadIdx.x; v < total; v += kPermThreads) {
    const int r = (int)fdiv32((uint32_t)v, P.nv_magic, P.nv_shift);
    const int x = v - r * P.nvec;
    if (x >= nv) continue;
    const Elem* src = src0 + (int64_t)r * P.row_sin + x * VW;
    Elem* dst = stage + (size_t)r * P.lap + x * VW;
    if (VB == 16)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
  }
}

template <typename Elem, typename Store, int VB>
__device__ __forceinline__ void perm2dv_store(const PermParams& P, const Elem* stage, const TileOrigin& o,
                                              const Store& st) {
  constexpr int VW = VB / (int)sizeof(Elem);
  using V = typename std::conditional<VB == 16, uint4, uint2>::type;
  const int qlim = (!o.full && P.pb >= 0) ? (P.pa == P.pb ? min(o.rem_a, o.rem_b) : o.rem_b) : (1 << 30);
  int chunks = P.nB;
  if (!o.full && P.pa >= 0 && P.pa != P.pb && P.chunk_is_pa) chunks = min(chunks, o.rem_a);
  const int jlim = min(P.LB, qlim);
  const int groups = (chunks + VW - 1) / VW;
  const int total = groups * P.LB;
  const int pstride = P.ej_pb_stride;
  for (int e = threadIdx.x; e < total; e += kPermThreads) {
    const int g = (int)fdiv32((uint32_t)e, P.lb_magic, P.lb_shift);
    const int j = e - g * P.LB;
    if (j >= jlim) continue;
    const int c0 = g * VW;
    union { V q; Elem v[VW]; } u;
    u.q = *reinterpret_cast<const V*>(stage + (size_t)j * pstride + c0);
    const int64_t ob = o.out_base + j;
#pragma unroll
    for (int t = 0; t < VW; ++t)
      if (c0 + t < chunks) st(ob + (int64_t)(c0 + t) * P.chunk_sout, u.v[t]);
  }
}

// A thread's full-tile offset list (N entries, n of them valid).
template <int N>
struct PermList {
  uint32_t a[N];  // shared-memory byte offset
  int32_t b[N];   // global element offset from the tile origin
  int n;
  __device__ __forceinline__ void build(int nq, int np, uint32_t Aq, uint32_t Ap, int32_t Bq, int32_t Bp) {
    const int total = nq * np, tid = threadIdx.x;
    n = tid < total ? min(N, (total - 1 - tid) / kPermThreads + 1) : 0;
#pragma unroll
    for (int i = 0; i < N; ++i) perm_list_entry(tid + i * kPermThreads, nq, Aq, Ap, Bq, Bp, &a[i], &b[i]);
  }
};

// Store functors that can write a whole vector of adjacent elements.
template <class S, class = void>
struct has_vec_store : std::false_type {};
template <class S>
struct has_vec_store<S, std::void_t<decltype(S::kVecStore)>> : std::true_type {};

// Store functors that read the output they update (the fused add): they
// expose load(o) -> Old and put(o, v, old), so that the list kernels can
// issue a batch of output loads before any of the writes that depend on them
// (one element at a time, each load's latency would serialise the stores).
template <class S, class = void>
struct is_rmw_store : std::false_type {};
template <class S>
struct is_rmw_store<S, std::void_t<decltype(S::kRMW)>> : std::true_type {};
template <class S, class E, bool = is_rmw_store<S>::value>
struct rmw_old { using type = E; };
template <class S, class E>
struct rmw_old<S, E, true> { using type = typename S::Old; };

constexpr int kHdrRing = kStages + 1;  // tile headers: issued, in flight, stored, being written

// VB: vector bytes of the vector paths (0: scalar general code only).
// ROWS: row copies (PermParams::rows2d), else column-group transposes.
// N: entries of the full-tile offset lists (0: general code only).
template <typename Elem, typename Store, int VB, bool ROWS, int N>
__global__ void __launch_bounds__(kPermThreads, N >= 16 ? 2 : (N > 0 ? 3 : 1))
perm2d_kernel(const __grid_constant__ PermParams P, const Elem* __restrict__ in, Store st, int flags) {
  constexpr bool VEC = VB > 0;
  constexpr bool LISTS = VEC && N > 0;
  constexpr int VBv = VB ? VB : 16;
  constexpr int es = (int)sizeof(Elem);
  constexpr int VW = VBv / es > 0 ? VBv / es : 1;
  constexpr int NL = N > 0 ? N : 1;
  using V = typename std::conditional<VBv == 16, uint4, uint2>::type;
  // flags: bit 0 = the functor's vector stores (row copies), bit 1 = full
  // tiles through the general code as well (a tuning/diagnostic switch)
  const bool vstore = (flags & 1) != 0;
  const bool lists = LISTS && (flags & 2) == 0;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ TileOrigin org[kHdrRing];
  Elem* bufs = reinterpret_cast<Elem*>(smem_raw);
  const size_t stage_elems = (size_t)P.nA * P.lap;
  const int64_t first = blockIdx.x, step = gridDim.x;
  const int mine = first < P.ntiles ? (int)((P.ntiles - 1 - first) / step + 1) : 0;
  PermList<NL> ldl, stl;
  if (LISTS) {
    ldl.build(P.nvec, P.nA, VBv, (uint32_t)(P.lap * es), VW, (int32_t)P.row_sin);
    if (ROWS)
      stl.build(P.nvec, P.nB, VBv, (uint32_t)(P.chunk_eb * es), VW, (int32_t)P.chunk_sout);
    else
      stl.build(P.LB, P.nB / VW, (uint32_t)(P.ej_pb_stride * es), VBv, 1, (int32_t)(VW * P.chunk_sout));
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < kStages && k < mine; ++k) org[k] = tile_origin(P, first + k * step);
  __syncthreads();

  auto issue = [&](int k) {
    const TileOrigin o = org[k % kHdrRing];
    Elem* stage = bufs + (size_t)(k % kStages) * stage_elems;
    if (lists && o.full) {
      const Elem* src = in + o.in_base;
      const uint32_t sb = smem_addr(stage);
#pragma unroll
      for (int i = 0; i < NL; ++i) {
        if (i < ldl.n) {
          if (VBv == 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sb + ldl.a[i]), "l"(src + ldl.b[i])
                         : "memory");
          else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sb + ldl.a[i]), "l"(src + ldl.b[i])
                         : "memory");
        }
      }
    } else if (VEC) {
      perm2dv_issue<Elem, VBv>(P, in, stage, o);
    } else {
      perm2d_issue<Elem>(P, in, stage, o);
    }
  };
  auto store = [&](int k) {
    const TileOrigin o = org[k % kHdrRing];
    const Elem* stage = bufs + (size_t)(k % kStages) * stage_elems;
    bool done = false;
    if constexpr (is_rmw_store<Store>::value) {
     if (lists && o.full) {
      // read-modify-write stores in batches of kRmwBatch list entries: the
      // output loads of a batch are all issued before its writes
      done = true;
      Store s2 = st;
      s2.out += o.out_base;
      const unsigned char* sb = reinterpret_cast<const unsigned char*>(stage);
      const int32_t cs = ROWS ? 1 : (int32_t)P.chunk_sout;
      constexpr int kRmwBatch = 4;
      using Old = typename rmw_old<Store, Elem>::type;
#pragma unroll
      for (int i0 = 0; i0 < NL; i0 += kRmwBatch) {
        Old old[kRmwBatch][VW];
#pragma unroll
        for (int g = 0; g < kRmwBatch; ++g) {
          const int i = i0 + g;
          if (i < NL && i < stl.n) {
#pragma unroll
            for (int t = 0; t < VW; ++t) old[g][t] = s2.load(stl.b[i] + t * cs);
          }
        }
#pragma unroll
        for (int g = 0; g < kRmwBatch; ++g) {
          const int i = i0 + g;
          if (i < NL && i < stl.n) {
            union { V q; Elem v[VW]; } u;
            u.q = *reinterpret_cast<const V*>(sb + stl.a[i]);
#pragma unroll
            for (int t = 0; t < VW; ++t) s2.put(stl.b[i] + t * cs, u.v[t], old[g][t]);
          }
        }
      }
     }
    }
    if (done) {
    } else if (lists && o.full) {
      Store s2 = st;
      s2.out += o.out_base;
      const unsigned char* sb = reinterpret_cast<const unsigned char*>(stage);
      const int32_t cs = (int32_t)P.chunk_sout;
#pragma unroll
      for (int i = 0; i < NL; ++i) {
        if (i < stl.n) {
          union { V q; Elem v[VW]; } u;
          u.q = *reinterpret_cast<const V*>(sb + stl.a[i]);
          if (ROWS) {
            bool done = false;
            if constexpr (has_vec_store<Store>::value) {
              if (vstore) { s2.template vec<V>(stl.b[i], u.q); done = true; }
            }
            if (!done) {
#pragma unroll
              for (int t = 0; t < VW; ++t) s2(stl.b[i] + t, u.v[t]);
            }
          } else {
#pragma unroll
            for (int t = 0; t < VW; ++t) s2(stl.b[i] + t * cs, u.v[t]);
          }
        }
      }
    } else if (VEC && !ROWS) {
      perm2dv_store<Elem, Store, VBv>(P, stage, o, st);
    } else {
      perm2d_store<Elem, Store>(P, stage, o, st);
    }
  };

  for (int k = 0; k < kStages - 1; ++k) {
    if (k < mine) issue(k);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int k = 0; k < mine; ++k) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 2) : "memory");
    __syncthreads();
    const int nk = k + kStages - 1;
    if (nk < mine) issue(nk);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    // the header slot of tile k + kStages last held tile k - 1, whose store
    // finished before the barrier above; it is read after the next barrier
    if (threadIdx.x == 0 && k + kStages < mine) org[(k + kStages) % kHdrRing] = tile_origin(P, first + (int64_t)(k + kStages) * step);
    store(k);
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// General plans on per-thread offset lists (perm_glist_kernel).  A plan of
// any shape -- several dimensions in the load or the store block, chunk
// tables -- moves every full tile with the same tile-relative offsets, so each
// thread computes its copies once, from the plan's tables: up to kGListN
// vector loads (VB bytes of a load row: 16, 8 or one element) and up to
// kGListN element stores, kept in registers.  Full tiles then run as unrolled
// base-plus-offset copies: a cp.async per load entry, a shared-memory read
// and a global store per store entry.  Store functors that read the output
// (the fused add) load a whole tile's worth of a thread's outputs before
// writing any.  Tiles at the tensor's edges (partial tiles) take the
// table-driven code of the pipelined kernel.  The host launches this kernel
// only for plans whose tile has at most kGListN * 256 elements and load
// vectors, and whose tile-relative offsets fit in 32 bits (glist_ok).
constexpr int kGListN = kGListEntries;

template <typename Elem, typename Store, int VB, int ST>
__global__ void __launch_bounds__(kPermThreads, 2)
perm_glist_kernel(const __grid_constant__ PermParams P, const Elem* __restrict__ in, Store st) {
  constexpr int es = (int)sizeof(Elem);
  constexpr int VW = VB / es;  // elements per load copy
  constexpr int kRing = ST + 1;  // tile headers: issued, in flight, stored, being written
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PermSmem& T = *reinterpret_cast<PermSmem*>(smem_raw);
  Elem* bufs = reinterpret_cast<Elem*>(smem_raw + ((sizeof(PermSmem) + 127) & ~size_t(127)));
  __shared__ TileOrigin org[kRing];
  const size_t stage_elems = (size_t)P.nA * P.lap;
  const int tid = threadIdx.x;
  for (int i = tid; i < P.nA; i += kPermThreads) { T.ld_base[i] = P.ld_base[i]; T.ld_dpb[i] = P.ld_dpb[i]; }
  for (int i = tid; i < P.nB; i += kPermThreads) {
    T.st_base[i] = P.st_base[i]; T.st_ebase[i] = P.st_ebase[i]; T.st_dpa[i] = P.st_dpa[i];
  }
  for (int i = tid; i < P.ejf_n; i += kPermThreads) T.ejf[i] = P.ejf[i];
  const int64_t first = blockIdx.x, step = gridDim.x;
  const int mine = first < P.ntiles ? (int)((P.ntiles - 1 - first) / step + 1) : 0;
  if (tid == 0)
    for (int k = 0; k < ST && k < mine; ++k) org[k] = tile_origin(P, first + k * step);
  __syncthreads();
  // this thread's full-tile copies: load vector v = (row c, vector x), store
  // element e = (store chunk c', position j) with consecutive e along a chunk
  const int nvec = P.LA / VW;
  const int nld_all = P.nA * nvec;
  const int nld = tid < nld_all ? min(kGListN, (nld_all - 1 - tid) / kPermThreads + 1) : 0;
  const int nst = tid < P.V ? min(kGListN, (P.V - 1 - tid) / kPermThreads + 1) : 0;
  uint32_t la[kGListN], sa[kGListN];
  int32_t lb[kGListN], sb[kGListN];
#pragma unroll
  for (int i = 0; i < kGListN; ++i) {
    int v = tid + i * kPermThreads;
    if (v >= nld_all) v = 0;
    const int c = v / nvec, x = v - c * nvec;
    la[i] = (uint32_t)((c * P.lap + x * VW) * es);
    lb[i] = (int32_t)(T.ld_base[c] + x * VW);
    int e = tid + i * kPermThreads;
    if (e >= P.V) e = 0;
    const int cc = e / P.LB, j = e - cc * P.LB;
    const int q = j / P.prodB;
    sa[i] = (uint32_t)((T.st_ebase[cc] + T.ejf[j - q * P.prodB] + q * P.ej_pb_stride) * es);
    sb[i] = (int32_t)(T.st_base[cc] + j);
  }
  StoreLanes SL;
  store_lanes_init(P, SL);

  auto issue = [&](int k) {
    const TileOrigin o = org[k % kRing];
    Elem* stage = bufs + (size_t)(k % ST) * stage_elems;
    if (o.full) {
      const Elem* src = in + o.in_base;
      const uint32_t sbase = smem_addr(stage);
#pragma unroll
      for (int i = 0; i < kGListN; ++i) {
        if (i < nld) {
          if (VB == 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sbase + la[i]), "l"(src + lb[i])
                         : "memory");
          else
            asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sbase + la[i]), "l"(src + lb[i]),
                         "n"(VB)
                         : "memory");
        }
      }
    } else {
      perm_issue<Elem, false, false>(P, T, in, stage, nullptr, first + (int64_t)k * step);
    }
  };
  auto store = [&](int k) {
    const TileOrigin o = org[k % kRing];
    const Elem* stage = bufs + (size_t)(k % ST) * stage_elems;
    if (!o.full) {
      perm_store<Elem, Store>(P, T, SL, stage, first + (int64_t)k * step, st);
      return;
    }
    Store s2 = st;
    s2.out += o.out_base;
    const unsigned char* sbase = reinterpret_cast<const unsigned char*>(stage);
    if constexpr (is_rmw_store<Store>::value) {
      constexpr int kBatch = 8;  // output loads in flight per thread before their writes
#pragma unroll
      for (int h = 0; h < kGListN; h += kBatch) {
        typename Store::Old old[kBatch];
#pragma unroll
        for (int g = 0; g < kBatch; ++g)
          if (h + g < nst) old[g] = s2.load(sb[h + g]);
#pragma unroll
        for (int g = 0; g < kBatch; ++g)
          if (h + g < nst) s2.put(sb[h + g], *reinterpret_cast<const Elem*>(sbase + sa[h + g]), old[g]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < kGListN; ++i)
        if (i < nst) s2(sb[i], *reinterpret_cast<const Elem*>(sbase + sa[i]));
    }
  };

  for (int k = 0; k < ST - 1; ++k) {
    if (k < mine) issue(k);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int k = 0; k < mine; ++k) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(ST - 2) : "memory");
    __syncthreads();
    const int nk = k + ST - 1;
    if (nk < mine) issue(nk);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    // the header slot of tile k + ST last held tile k - 1, whose store
    // finished before the barrier above; it is read after the next barrier
    if (tid == 0 && k + ST < mine) org[(k + ST) % kRing] = tile_origin(P, first + (int64_t)(k + ST) * step);
    store(k);
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Load vector bytes of the list kernel for a plan and input pointer, or 0
// when the plan does not fit its lists.
template <typename Elem>
inline int glist_vector_bytes(const PermParams& P, const Elem* in) {
  const uintptr_t a = (uintptr_t)in;
  return perm_glist_vector_bytes(P, a % 16 == 0 ? 16 : (a % 8 == 0 ? 8 : (int)sizeof(Elem)), kPermThreads);
}

// Pipeline depth of the list kernel: small tiles keep six in flight (two
// CTAs per SM still fit), larger ones three.
constexpr int kGListDeep = 6;

template <typename Elem, typename Store, int VB>
void launch_glist(const PermParams& P, const Elem* in, const Store& st, cudaStream_t s) {
  static DeviceOnce attr3, attr6;
  const size_t tables = ((sizeof(PermSmem) + 127) & ~size_t(127)) + 128;
  const size_t stage = (size_t)perm_stage_bytes(P);
  const bool deep = tables + kGListDeep * stage <= 110 * 1024;
  const size_t smem = tables + (deep ? kGListDeep : kStages) * stage;
  int per_sm = (int)((224 * 1024) / (smem + 1024));
  per_sm = std::max(1, std::min(per_sm, 2));  // launch bound: 2 CTAs of 256 threads per SM (register lists)
  const unsigned grid = (unsigned)std::min<int64_t>((int64_t)num_sms() * per_sm, P.ntiles);
  if (deep) {
    smem_limit_once(attr6, perm_glist_kernel<Elem, Store, VB, kGListDeep>, 220 * 1024);
    perm_glist_kernel<Elem, Store, VB, kGListDeep><<<grid, kPermThreads, smem, s>>>(P, in, st);
  } else {
    smem_limit_once(attr3, perm_glist_kernel<Elem, Store, VB, kStages>, 220 * 1024);
    perm_glist_kernel<Elem, Store, VB, kStages><<<grid, kPermThreads, smem, s>>>(P, in, st);
  }
}

// ---------------------------------------------------------------------------
// Row copies without shared memory (perm_rowcopy_kernel): plans whose store
// chunks are the load rows themselves (the fastest dimension stays fastest,
// as rows2d) but whose rows are not whole vectors (rows2d needs 8- or 16-byte
// rows) need no transposition at all, so each row moves directly from global
// to global memory: one warp per (tile, row), lanes along the row, kRowBatch
// loads in flight per lane before their stores (with the output loads of
// functors that read the output).
constexpr int kRowBatch = 8;

template <typename Elem, typename Store>
__global__ void __launch_bounds__(kPermThreads)
perm_rowcopy_kernel(const __grid_constant__ PermParams P, const Elem* __restrict__ in, Store st) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t units = P.ntiles * P.nA;
  for (int64_t u = warp; u < units; u += nwarps) {
    const int64_t tile = u / P.nA;
    const int c = (int)(u - tile * P.nA);
    const TileOrigin o = tile_origin(P, tile);
    if (!o.full && P.pb >= 0 && P.pb != P.pa && P.row_is_pb && c >= o.rem_b) continue;
    int len = P.LA;
    if (!o.full && P.pa >= 0) len = P.prodA * (P.pb == P.pa ? min(o.rem_a, o.rem_b) : o.rem_a);
    const Elem* src = in + o.in_base + (int64_t)c * P.row_sin;
    const int64_t ob = o.out_base + (int64_t)c * P.chunk_sout;
    for (int j0 = 0; j0 < len; j0 += 32 * kRowBatch) {
      Elem v[kRowBatch];
      typename rmw_old<Store, Elem>::type old[kRowBatch];
#pragma unroll
      for (int t = 0; t < kRowBatch; ++t) {
        const int j = j0 + t * 32 + lane;
        if (j < len) v[t] = src[j];
      }
      if constexpr (is_rmw_store<Store>::value) {
#pragma unroll
        for (int t = 0; t < kRowBatch; ++t) {
          const int j = j0 + t * 32 + lane;
          if (j < len) old[t] = st.load(ob + j);
        }
      }
#pragma unroll
      for (int t = 0; t < kRowBatch; ++t) {
        const int j = j0 + t * 32 + lane;
        if (j >= len) continue;
        if constexpr (is_rmw_store<Store>::value) st.put(ob + j, v[t], old[t]);
        else st(ob + j, v[t]);
      }
    }
  }
}

// Row-copy-shaped plans (load row c is store chunk c, same run).
inline bool row_copy_shape(const PermParams& P) {
  return P.lin2d && P.nA == P.nB && P.LA == P.LB && P.ej_pb_stride == 1 && (P.chunk_eb == P.lap || P.nA == 1);
}

// Whether a store functor writes vectors of vbytes to an aligned output
// (functors without vector stores: no; StoreCopy overloads this below).
template <typename S>
inline bool store_vec_ok(const S&, int) { return false; }

// One 2-D kernel variant; N = list entries (0, 8 or 16).  The grid is the
// number of CTAs resident at once (tiles are dealt to CTAs round robin).
template <typename Elem, typename Store, int VB, bool ROWS>
void launch_2d(int N, int64_t ntiles, size_t smem, cudaStream_t s, const PermParams& P, const Elem* in,
               const Store& st, int flags) {
  using Kern = void (*)(PermParams, const Elem*, Store, int);
  const int idx = VB > 0 ? (N == 16 ? 2 : (N == 8 ? 1 : 0)) : 0;
  const Kern kern = idx == 2 ? (Kern)perm2d_kernel<Elem, Store, VB, ROWS, (VB > 0 ? 16 : 0)>
                  : idx == 1 ? (Kern)perm2d_kernel<Elem, Store, VB, ROWS, (VB > 0 ? 8 : 0)>
                             : (Kern)perm2d_kernel<Elem, Store, VB, ROWS, 0>;
  // per variant and device: the shared-memory limit, and the resident CTAs
  // per SM of the last shared-memory size (packed as smem << 8 | blocks)
  static DeviceOnce attr[3];
  static std::atomic<unsigned long long> occ[3][64];
  const int dev = current_device();
  smem_limit_once(attr[idx], kern, 220 * 1024);
  unsigned long long o = occ[idx][dev].load(std::memory_order_relaxed);
  int blocks = (int)(o & 0xFF);
  if ((o >> 8) != (unsigned long long)smem || blocks < 1) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, kPermThreads, smem) != cudaSuccess || b < 1) {
      cudaGetLastError();
      b = 1;
    }
    blocks = std::min(b, 255);
    occ[idx][dev].store(((unsigned long long)smem << 8) | (unsigned long long)blocks, std::memory_order_relaxed);
  }
  const unsigned grid = (unsigned)std::min<int64_t>((int64_t)num_sms() * blocks, ntiles);
  kern<<<grid, kPermThreads, smem, s>>>(P, in, st, flags);
}

// Launches the pipelined kernel with a grid sized to the SM count.
template <typename Elem, typename Store>
int launch_perm(const PermParams& P, const Elem* in, const Store& st, cudaStream_t s) {
  if (P.ntiles <= 0) return 0;
  const size_t smem = perm_smem_bytes(P);
  // TB_PERM_LOADS=async|bulk|tables|auto selects the load mechanism (tuning
  // knob; all produce identical results).  auto: bulk copies for long rows,
  // the 2-D kernel for other 2-D tiles.
  static int mode = [] {
    const char* e = getenv("TB_PERM_LOADS");
    if (!e) return 0;
    if (!strcmp(e, "bulk")) return 1;
    if (!strcmp(e, "async")) return 2;
    if (!strcmp(e, "tables")) return 3;  // the table-driven kernel even for 2-D tiles
    if (!strcmp(e, "scalar2d")) return 4;  // the 2-D kernel without 16-byte column groups
    if (!strcmp(e, "norows")) return 5;    // row copies through the scalar 2-D store
    return 0;
  }();
  const bool eligible = P.tma_ok && ((uintptr_t)in % 16 == 0);
  // TB_PERM_GLIST=0: general plans through the table-driven kernel (tuning
  // and diagnostic switch; results are identical)
  static const bool glist_on = [] { const char* e = getenv("TB_PERM_GLIST"); return !(e && e[0] == '0'); }();
  // long rows move as bulk copies, except row copies (rows2d), whose 2-D
  // kernel stores whole vectors (TB_PERM_LONGROWS=bulk: those too)
  static const bool longrows_bulk = [] { const char* e = getenv("TB_PERM_LONGROWS"); return e && !strcmp(e, "bulk"); }();
  const bool bulk = eligible && (mode == 1 || (mode == 0 && (int64_t)P.LA * P.es >= 4096 &&
                                               (!P.rows2d || longrows_bulk || P.bulk_rows)));
  static DeviceOnce attr_bulk, attr_async;
  smem_limit_once(attr_bulk, perm_pipe_kernel<Elem, Store, true>, 220 * 1024);
  smem_limit_once(attr_async, perm_pipe_kernel<Elem, Store, false>, 220 * 1024);
  if (smem > 220 * 1024) { set_error("permutation tile too large for shared memory"); return TB_ERR_LIMIT; }
  // TB_PERM_TRACE=1: one line per launch on stderr (plan shape and kernel; diagnostics)
  static const bool trace = [] { const char* e = getenv("TB_PERM_TRACE"); return e && e[0] == '1'; }();
  if (trace) {
    const int gvb = glist_vector_bytes(P, in);
    fprintf(stderr, "perm es=%d rank=%d V=%d LA=%d nA=%d LB=%d nB=%d prodB=%d lin2d=%d vec2d=%d rows2d=%d tma=%d "
                    "vec8=%d tiles=%lld kernel=%s\n",
            P.es, P.rank, P.V, P.LA, P.nA, P.LB, P.nB, P.prodB, P.lin2d, P.vec2d, P.rows2d, P.tma_ok, P.vec8,
            (long long)P.ntiles,
            bulk ? "bulk" : (P.lin2d && mode != 3 && (P.vec2d || P.rows2d) && P.vbytes && (uintptr_t)in % P.vbytes == 0)
                                ? "2d-vector"
                                : (P.lin2d && mode == 0 && glist_on && row_copy_shape(P)) ? "rowcopy"
                                : (mode == 0 && glist_on && gvb) ? (gvb == 16 ? "glist16" : gvb == 8 ? "glist8" : "glist1")
                                : P.lin2d && mode != 3 ? "2d-scalar" : "tables");
  }
  int per_sm = (int)((224 * 1024) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 2048 / kPermThreads) per_sm = 2048 / kPermThreads;
  int64_t grid = (int64_t)num_sms() * per_sm;
  if (grid > P.ntiles) grid = P.ntiles;
  if (!bulk && P.lin2d && mode != 3) {
    // two-dimensional tiles: no chunk tables in shared memory, so more CTAs fit
    const size_t smem2 = (size_t)kStages * (size_t)perm_stage_bytes(P) + 128;
    const bool in_ok = P.vbytes && (uintptr_t)in % (uintptr_t)P.vbytes == 0 && mode != 4;
    const bool vec = P.vec2d && in_ok;
    const bool rows = P.rows2d && in_ok && mode != 5;  // TB_PERM_LOADS=norows: row copies as scalar stores
    // TB_PERM_FAST=0: full tiles through the general code too (diagnostic)
    static const int nowalk = [] { const char* e = getenv("TB_PERM_FAST"); return e && e[0] == '0' ? 2 : 0; }();
    constexpr int V8 = sizeof(Elem) <= 8 ? 8 : 16;
    if (rows || vec) {
      const int N = perm2d_list_entries(P, rows, kPermThreads);
      const int flags = (rows && P.out_vec && store_vec_ok(st, P.vbytes) ? 1 : 0) | nowalk;
      if (rows && P.vbytes == 16) launch_2d<Elem, Store, 16, true>(N, P.ntiles, smem2, s, P, in, st, flags);
      else if (rows) launch_2d<Elem, Store, V8, true>(N, P.ntiles, smem2, s, P, in, st, flags);
      else if (P.vbytes == 16) launch_2d<Elem, Store, 16, false>(N, P.ntiles, smem2, s, P, in, st, flags);
      else launch_2d<Elem, Store, V8, false>(N, P.ntiles, smem2, s, P, in, st, flags);
    } else if (mode == 0 && glist_on && row_copy_shape(P)) {
      const unsigned grid = (unsigned)std::min<int64_t>((int64_t)num_sms() * 8, (P.ntiles * P.nA + 7) / 8);
      perm_rowcopy_kernel<Elem, Store><<<std::max(1u, grid), kPermThreads, 0, s>>>(P, in, st);
    } else if (const int gvb = (mode == 0 && glist_on) ? glist_vector_bytes(P, in) : 0) {
      if (gvb == 16) launch_glist<Elem, Store, (sizeof(Elem) < 16 ? 16 : sizeof(Elem))>(P, in, st, s);
      else if (gvb == 8) launch_glist<Elem, Store, (sizeof(Elem) < 8 ? 8 : sizeof(Elem))>(P, in, st, s);
      else launch_glist<Elem, Store, sizeof(Elem)>(P, in, st, s);
    } else {
      launch_2d<Elem, Store, 0, false>(0, P.ntiles, smem2, s, P, in, st, 0);
    }
  } else if (!bulk && mode == 0 && glist_on && glist_vector_bytes(P, in)) {
    const int gvb = glist_vector_bytes(P, in);
    if (gvb == 16) launch_glist<Elem, Store, (sizeof(Elem) < 16 ? 16 : sizeof(Elem))>(P, in, st, s);
    else if (gvb == 8) launch_glist<Elem, Store, (sizeof(Elem) < 8 ? 8 : sizeof(Elem))>(P, in, st, s);
    else launch_glist<Elem, Store, sizeof(Elem)>(P, in, st, s);
  } else if (bulk)
    perm_pipe_kernel<Elem, Store, true><<<(unsigned)grid, kPermThreads, smem, s>>>(P, in, st, device_error_word());
  else
    perm_pipe_kernel<Elem, Store, false><<<(unsigned)grid, kPermThreads, smem, s>>>(P, in, st, device_error_word());
  TB_CHECK_LAUNCH();
  return 0;
}

// ---- element types and store functors --------------------------------------
struct alignas(16) u128 { uint64_t lo, hi; };

template <typename E>
struct StoreCopy {
  E* out;
  static constexpr bool kVecStore = true;
  __device__ __forceinline__ void operator()(int64_t o, const E& v) const { out[o] = v; }
  // adjacent elements o, o+1, ... as one vector (o * sizeof(E) aligned to V)
  template <typename V>
  __device__ __forceinline__ void vec(int64_t o, const V& v) const { *reinterpret_cast<V*>(out + o) = v; }
};
template <typename E>
inline bool store_vec_ok(const StoreCopy<E>& st, int vbytes) {
  return vbytes > 0 && (uintptr_t)st.out % (uintptr_t)vbytes == 0;
}
// Conjugating copies: flip the sign bit of the imaginary part.
struct StoreConjC4 {  // complex float as one 64-bit word (re low, im high)
  uint64_t* out;
  __device__ __forceinline__ void operator()(int64_t o, const uint64_t& v) const {
    out[o] = v ^ 0x8000000000000000ull;
  }
};
struct StoreConjC8 {
  u128* out;
  __device__ __forceinline__ void operator()(int64_t o, const u128& v) const {
    u128 w = v; w.hi ^= 0x8000000000000000ull; out[o] = w;
  }
};

}  // namespace tb
