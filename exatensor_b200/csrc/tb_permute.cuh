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
constexpr uint32_t kWaitLimit = 1u << 26;  // bounded mbarrier polling

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
    const uint64_t q = P.gdiv[g].div(r);
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
template <typename Elem, bool BULK>
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
    const bool vec = P.tma_ok && sizeof(Elem) < 16;
    const bool vec8 = !vec && P.vec8 && sizeof(Elem) < 8;
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
    asm volatile("cp.async.commit_group;\n" ::: "memory");
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
  for (int64_t k = 0; k < mine; ++k) {
    const int stg = (int)(k % kStages);
    if (BULK) {
      const uint32_t parity = (uint32_t)((k / kStages) & 1);
      uint32_t done = 0, it = 0;
      while (!done) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(&T.mbar[stg])), "r"(parity)
            : "memory");
        if (!done && ++it > kWaitLimit) { failed = true; break; }
      }
    } else {
      asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 2) : "memory");
    }
    if (failed) break;
    __syncthreads();
    const int64_t nk = k + kStages - 1;
    const int nstg = (int)(nk % kStages);
    if (nk < mine) perm_issue<Elem, BULK>(P, T, in, bufs + (size_t)nstg * stage_elems, &T.mbar[nstg], first + nk * step);
    else if (!BULK) asm volatile("cp.async.commit_group;\n" ::: "memory");
    perm_store<Elem, Store>(P, T, SL, bufs + (size_t)stg * stage_elems, first + k * step, st);
  }
  if (failed) {
    record_device_error(err, 1u);
    return;
  }
  if (!BULK) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Two-dimensional tiles (PermParams::lin2d): every load row and every store
// chunk is one step of a single dimension, so their offsets are c * stride and
// the kernel needs no chunk tables.  Warps take whole rows (loads: 16-byte or
// element cp.async, lanes along the row) and whole chunks (stores: lanes along
// the output run), which keeps the instruction count per element low; the
// 3-stage cp.async pipeline is the same as perm_pipe_kernel's !BULK path.
template <typename Elem>
__device__ __forceinline__ void perm2d_issue(const PermParams& P, const Elem* in, Elem* stage, int64_t tile) {
  const TileOrigin o = tile_origin(P, tile);
  int len = P.LA;
  if (!o.full && P.pa >= 0) len = P.prodA * (P.pb == P.pa ? min(o.rem_a, o.rem_b) : o.rem_a);
  int rows = P.nA;
  if (!o.full && P.pb >= 0 && P.pb != P.pa && P.row_is_pb) rows = min(rows, o.rem_b);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kW = kPermThreads / 32;
  const bool vec = P.tma_ok && sizeof(Elem) < 16;
  const bool vec8 = !vec && P.vec8 && sizeof(Elem) < 8;
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
__device__ __forceinline__ void perm2d_store(const PermParams& P, const Elem* stage, int64_t tile, const Store& st) {
  const TileOrigin o = tile_origin(P, tile);
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

// Vectorised 2-D tiles (PermParams::vec2d): the load phase walks (row,
// 16-byte vector) pairs over the whole CTA, and the store phase gives each
// lane 16 / es adjacent columns (= store chunks) of one row: one 16-byte
// shared-memory read feeds 16 / es output runs, and consecutive lanes take
// consecutive rows, i.e. consecutive positions of those runs.  Rows are an
// odd number of 16-byte units long, so a warp's 16-byte reads of one column
// group spread over all banks.  The tile's store bounds are computed by
// thread 0 when the tile is issued and kept in shared memory until its store.
struct Perm2dHdr {
  int64_t out_base;
  int chunks, jlim;
};

template <typename Elem, int VB>
__device__ __forceinline__ void perm2dv_issue(const PermParams& P, const Elem* in, Elem* stage, int64_t tile,
                                              Perm2dHdr* hdr) {
  const TileOrigin o = tile_origin(P, tile);
  int len = P.LA;
  if (!o.full && P.pa >= 0) len = P.prodA * (P.pb == P.pa ? min(o.rem_a, o.rem_b) : o.rem_a);
  int rows = P.nA;
  if (!o.full && P.pb >= 0 && P.pb != P.pa && P.row_is_pb) rows = min(rows, o.rem_b);
  if (threadIdx.x == 0) {
    const int qlim = (!o.full && P.pb >= 0) ? (P.pa == P.pb ? min(o.rem_a, o.rem_b) : o.rem_b) : (1 << 30);
    int chunks = P.nB;
    if (!o.full && P.pa >= 0 && P.pa != P.pb && P.chunk_is_pa) chunks = min(chunks, o.rem_a);
    hdr->out_base = o.out_base;
    hdr->chunks = chunks;
    hdr->jlim = min(P.LB, qlim);
  }
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
__device__ __forceinline__ void perm2dv_store(const PermParams& P, const Elem* stage, const Perm2dHdr& h,
                                              const Store& st) {
  constexpr int VW = VB / (int)sizeof(Elem);
  using V = typename std::conditional<VB == 16, uint4, uint2>::type;
  const int groups = (h.chunks + VW - 1) / VW;
  const int total = groups * P.LB;
  const int pstride = P.ej_pb_stride;
  for (int e = threadIdx.x; e < total; e += kPermThreads) {
    const int g = (int)fdiv32((uint32_t)e, P.lb_magic, P.lb_shift);
    const int j = e - g * P.LB;
    if (j >= h.jlim) continue;
    const int c0 = g * VW;
    union { V q; Elem v[VW]; } u;
    u.q = *reinterpret_cast<const V*>(stage + (size_t)j * pstride + c0);
    const int64_t ob = h.out_base + j;
#pragma unroll
    for (int t = 0; t < VW; ++t)
      if (c0 + t < h.chunks) st(ob + (int64_t)(c0 + t) * P.chunk_sout, u.v[t]);
  }
}

template <typename Elem, typename Store, int VB>  // VB: vector bytes of the vectorised path, 0 = scalar
__global__ void __launch_bounds__(kPermThreads)
perm2d_kernel(const __grid_constant__ PermParams P, const Elem* __restrict__ in, Store st) {
  constexpr bool VEC = VB > 0;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ Perm2dHdr hdr[kStages];
  Elem* bufs = reinterpret_cast<Elem*>(smem_raw);
  const size_t stage_elems = (size_t)P.nA * P.lap;
  const int64_t first = blockIdx.x, step = gridDim.x;
  const int64_t mine = first < P.ntiles ? (P.ntiles - 1 - first) / step + 1 : 0;
  for (int k = 0; k < kStages - 1; ++k) {
    if (k < mine) {
      if (VEC) perm2dv_issue<Elem, VB ? VB : 16>(P, in, bufs + (size_t)k * stage_elems, first + k * step, &hdr[k]);
      else perm2d_issue<Elem>(P, in, bufs + (size_t)k * stage_elems, first + k * step);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int64_t k = 0; k < mine; ++k) {
    const int stg = (int)(k % kStages);
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 2) : "memory");
    __syncthreads();
    const int64_t nk = k + kStages - 1;
    const int nstg = (int)(nk % kStages);
    if (nk < mine) {
      if (VEC) perm2dv_issue<Elem, VB ? VB : 16>(P, in, bufs + (size_t)nstg * stage_elems, first + nk * step, &hdr[nstg]);
      else perm2d_issue<Elem>(P, in, bufs + (size_t)nstg * stage_elems, first + nk * step);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    if (VEC) perm2dv_store<Elem, Store, VB ? VB : 16>(P, bufs + (size_t)stg * stage_elems, hdr[stg], st);
    else perm2d_store<Elem, Store>(P, bufs + (size_t)stg * stage_elems, first + k * step, st);
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
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
    return 0;
  }();
  const bool eligible = P.tma_ok && ((uintptr_t)in % 16 == 0);
  const bool bulk = eligible && (mode == 1 || (mode == 0 && (int64_t)P.LA * P.es >= 4096));
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(perm_pipe_kernel<Elem, Store, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    cudaFuncSetAttribute(perm_pipe_kernel<Elem, Store, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    attr_set = true;
  }
  if (smem > 220 * 1024) { set_error("permutation tile too large for shared memory"); return TB_ERR_LIMIT; }
  int per_sm = (int)((224 * 1024) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 2048 / kPermThreads) per_sm = 2048 / kPermThreads;
  int64_t grid = (int64_t)num_sms() * per_sm;
  if (grid > P.ntiles) grid = P.ntiles;
  if (!bulk && P.lin2d && mode != 3) {
    // two-dimensional tiles: no chunk tables in shared memory, so more CTAs fit
    const size_t smem2 = (size_t)kStages * (size_t)perm_stage_bytes(P) + 128;
    static bool attr2 = false;
    if (!attr2) {
      cudaFuncSetAttribute(perm2d_kernel<Elem, Store, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
      cudaFuncSetAttribute(perm2d_kernel<Elem, Store, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
      if (sizeof(Elem) <= 8)
        cudaFuncSetAttribute(perm2d_kernel<Elem, Store, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
      attr2 = true;
    }
    int per2 = (int)((224 * 1024) / (smem2 + 1024));
    per2 = std::max(1, std::min(per2, 2048 / kPermThreads));
    int64_t grid2 = std::min<int64_t>((int64_t)num_sms() * per2, P.ntiles);
    const bool vec = P.vec2d && (uintptr_t)in % (uintptr_t)P.vbytes == 0 && mode != 4;
    if (vec && P.vbytes == 16)
      perm2d_kernel<Elem, Store, 16><<<(unsigned)grid2, kPermThreads, smem2, s>>>(P, in, st);
    else if (vec && P.vbytes == 8 && sizeof(Elem) <= 8)
      perm2d_kernel<Elem, Store, (sizeof(Elem) <= 8 ? 8 : 16)><<<(unsigned)grid2, kPermThreads, smem2, s>>>(P, in, st);
    else
      perm2d_kernel<Elem, Store, 0><<<(unsigned)grid2, kPermThreads, smem2, s>>>(P, in, st);
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
  __device__ __forceinline__ void operator()(int64_t o, const E& v) const { out[o] = v; }
};
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
