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

namespace tb {

constexpr int kPermThreads = 256;

// ---------------------------------------------------------------------------
// Kernel template.  Elem: the staged element type; Store: functor with
//   __device__ void operator()(int64_t out_offset, const Elem& v) const;
// ---------------------------------------------------------------------------
struct PermSmem {
  int64_t ld_base[kMaxChunks];
  int64_t st_base[kMaxChunks];
  int32_t st_ebase[kMaxChunks];
  int32_t ejf[kMaxEjf];
  int16_t ld_dpb[kMaxChunks];
  int16_t st_dpa[kMaxChunks];
};

template <typename Elem>
__host__ __device__ inline size_t perm_smem_bytes(int V, int pad_shift) {
  return sizeof(PermSmem) + (size_t)(V + (V >> pad_shift) + 1) * sizeof(Elem) + 16;
}

template <typename Elem, typename Store>
__global__ void __launch_bounds__(kPermThreads)
perm_tile_kernel(const __grid_constant__ PermParams P, const Elem* __restrict__ in, Store st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PermSmem& T = *reinterpret_cast<PermSmem*>(smem_raw);
  Elem* buf = reinterpret_cast<Elem*>(smem_raw + ((sizeof(PermSmem) + 15) & ~size_t(15)));
  const int tid = threadIdx.x;
  for (int i = tid; i < P.nA; i += kPermThreads) { T.ld_base[i] = P.ld_base[i]; T.ld_dpb[i] = P.ld_dpb[i]; }
  for (int i = tid; i < P.nB; i += kPermThreads) {
    T.st_base[i] = P.st_base[i]; T.st_ebase[i] = P.st_ebase[i]; T.st_dpa[i] = P.st_dpa[i];
  }
  for (int i = tid; i < P.ejf_n; i += kPermThreads) T.ejf[i] = P.ejf[i];
  __syncthreads();
  const int V = P.V, LA = P.LA, LB = P.LB;
  const int ps = P.pad_shift;
  for (int64_t tile = blockIdx.x; tile < P.ntiles; tile += gridDim.x) {
    // tile origin
    int64_t in_base = 0, out_base = 0;
    int rem_a = 1 << 30, rem_b = 1 << 30;
    {
      uint64_t r = (uint64_t)tile;
      for (int g = 0; g < P.ngd; ++g) {
        uint64_t q = P.gdiv[g].div(r);
        int64_t x = (int64_t)(r - q * (uint64_t)P.gext[g]);
        r = q;
        const int d = P.gdim[g];
        const int64_t org = x * P.tile[d];
        in_base += org * P.sin[d];
        out_base += org * P.sout[d];
        const int64_t rem = P.dims[d] - org;
        if (d == P.pa) rem_a = (int)(rem < P.tile[d] ? rem : P.tile[d]);
        if (d == P.pb) rem_b = (int)(rem < P.tile[d] ? rem : P.tile[d]);
      }
    }
    const bool full = (P.pa < 0 || rem_a >= P.tile[P.pa]) && (P.pb < 0 || rem_b >= P.tile[P.pb]);
    // ---- load phase: input-order tile index e = j + LA*c
    if (full) {
#pragma unroll 4
      for (int e = tid; e < V; e += kPermThreads) {
        const int c = (int)fdiv32((uint32_t)e, P.la_magic, P.la_shift);
        const int j = e - c * LA;
        buf[e + (e >> ps)] = in[in_base + T.ld_base[c] + j];
      }
    } else {
      for (int e = tid; e < V; e += kPermThreads) {
        const int c = (int)fdiv32((uint32_t)e, P.la_magic, P.la_shift);
        const int j = e - c * LA;
        bool ok = true;
        if (P.pa >= 0) {
          const int da = j / P.prodA;
          ok = da < rem_a;
          if (P.pb == P.pa) ok = ok && da < rem_b;
        }
        if (P.pb >= 0 && P.pb != P.pa) ok = ok && T.ld_dpb[c] < rem_b;
        if (ok) buf[e + (e >> ps)] = in[in_base + T.ld_base[c] + j];
      }
    }
    __syncthreads();
    // ---- store phase: output-order tile index f = j' + LB*c'
    if (full) {
#pragma unroll 4
      for (int f = tid; f < V; f += kPermThreads) {
        const int c = (int)fdiv32((uint32_t)f, P.lb_magic, P.lb_shift);
        const int j = f - c * LB;
        const int q = (int)fdiv32((uint32_t)j, P.pb_magic, P.pb_shift);
        const int e = T.st_ebase[c] + T.ejf[j - q * P.ejf_n] + q * P.ej_pb_stride;
        st(out_base + T.st_base[c] + j, buf[e + (e >> ps)]);
      }
    } else {
      for (int f = tid; f < V; f += kPermThreads) {
        const int c = (int)fdiv32((uint32_t)f, P.lb_magic, P.lb_shift);
        const int j = f - c * LB;
        const int q = (int)fdiv32((uint32_t)j, P.pb_magic, P.pb_shift);
        bool ok = true;
        if (P.pb >= 0) {
          ok = q < rem_b;
          if (P.pa == P.pb) ok = ok && q < rem_a;
        }
        if (P.pa >= 0 && P.pa != P.pb) ok = ok && T.st_dpa[c] < rem_a;
        if (ok) {
          const int e = T.st_ebase[c] + T.ejf[j - q * P.ejf_n] + q * P.ej_pb_stride;
          st(out_base + T.st_base[c] + j, buf[e + (e >> ps)]);
        }
      }
    }
    __syncthreads();
  }
}

// Launches perm_tile_kernel with a grid sized to the SM count.
template <typename Elem, typename Store>
int launch_perm(const PermParams& P, const Elem* in, const Store& st, cudaStream_t s) {
  if (P.ntiles <= 0) return 0;
  const size_t smem = perm_smem_bytes<Elem>(P.V, P.pad_shift);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(perm_tile_kernel<Elem, Store>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         96 * 1024);
    attr_set = true;
  }
  int per_sm = (int)((200 * 1024) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 8) per_sm = 8;
  int64_t grid = (int64_t)num_sms() * per_sm;
  if (grid > P.ntiles) grid = P.ntiles;
  perm_tile_kernel<Elem, Store><<<(unsigned)grid, kPermThreads, smem, s>>>(P, in, st);
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
