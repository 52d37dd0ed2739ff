// tb_perm_tma.cuh -- permutation tiles staged by TMA tensor loads.
//
// For a permutation whose output-fastest dimension b is not the input-fastest
// dimension 0 (a transpose in the two fastest dimensions of the output), the
// input is described once as a tensor map (the plan's reduced dims, up to 5)
// and each tile is up to four boxes side by side along dim 0: a box is 128
// bytes along dim 0 times B indices along dim b (B = the extent of b up to
// 128, so that short b dims do not load wasted rows), one index along every
// other dim.  One thread issues the box loads (cp.async.bulk.tensor,
// SWIZZLE_128B, no multicast) into a pipeline stage; completion is counted in
// bytes on the stage's mbarrier.  A box lands as B rows (one per b index) of
// 128 bytes whose 16-byte chunks are permuted by XOR with the row index mod 8,
// so that the store phase -- each lane reading one 16-byte chunk of its own
// row, 32 consecutive rows per warp -- reads shared memory without bank
// conflicts.  Each lane then holds 16 bytes
// along dim 0 for one b index, and the warp writes 16/es output runs of 32
// consecutive elements along b.  Out-of-range parts of edge boxes are filled
// with zeros by the TMA unit and not stored.
//
// Requirements (checked by tma_perm_plan): reduced rank 2..5, b != 0, every
// input stride of dims >= 1 a multiple of 16 bytes, a 16-byte aligned input.
#pragma once
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "tb_common.cuh"
#include "tb_perm_plan.h"
#include "tb_sm100.cuh"

namespace tb {

constexpr int kTmaPermStages = 3;
constexpr int kTmaBoxBytes = 128;     // along input dim 0
constexpr int kTmaBoxRowsMax = 128;   // along the output-fastest dim b
constexpr int kTmaStageMax = 36 * 1024;  // two CTAs per SM with three stages
constexpr int kTmaMaxRank = 5;

struct alignas(64) TmaPermParams {
  CUtensorMap map;                 // input as bytes along dim 0, elements along the others
  int rank, es, b;
  int A;                           // elements of a box along dim 0 (128 / es)
  int B;                           // box rows along dim b
  int nbx;                         // boxes side by side along dim 0 per tile
  int region;                      // shared-memory bytes per box (1024-aligned)
  int64_t ext[kTmaMaxRank];
  int64_t sout[kTmaMaxRank];       // output strides (elements); sout[b] == 1
  int ord[kTmaMaxRank];            // tile-index digits, fastest first: b, then the others in output order
  int64_t cnt[kTmaMaxRank];        // tiles along ord[i]
  int64_t ntiles;
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
inline PFN_cuTensorMapEncodeTiled_v12000 perm_tma_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// Builds the TMA plan from a permutation plan's reduced view; false when the
// layout does not meet the requirements above.
inline bool tma_perm_plan(const PermParams& P, const void* in, TmaPermParams* T) {
  const int r = P.rank, es = P.es;
  if (r < 2 || r > kTmaMaxRank || (es != 4 && es != 8 && es != 16) || (uintptr_t)in % 16 != 0) return false;
  int b = -1;
  for (int d = 0; d < r; ++d)
    if (P.sout[d] == 1) b = d;
  if (b <= 0) return false;
  for (int d = 1; d < r; ++d)
    if ((P.sin[d] * es) % 16 != 0) return false;
  auto enc = perm_tma_encode();
  if (!enc) return false;
  std::memset(T, 0, sizeof(*T));
  T->rank = r; T->es = es; T->b = b; T->A = kTmaBoxBytes / es;
  T->B = (int)std::min<int64_t>(P.dims[b], kTmaBoxRowsMax);
  T->region = (kTmaBoxBytes * T->B + 1023) / 1024 * 1024;
  const int64_t row_boxes = (P.dims[0] * es + kTmaBoxBytes - 1) / kTmaBoxBytes;
  T->nbx = (int)std::max<int64_t>(1, std::min<int64_t>({4, row_boxes, kTmaStageMax / T->region}));
  cuuint64_t dims[kTmaMaxRank], strides[kTmaMaxRank - 1];
  cuuint32_t box[kTmaMaxRank], estr[kTmaMaxRank];
  for (int d = 0; d < r; ++d) {
    T->ext[d] = P.dims[d];
    T->sout[d] = P.sout[d];
    dims[d] = (cuuint64_t)(d == 0 ? P.dims[0] * es : P.dims[d]);
    if (d > 0) strides[d - 1] = (cuuint64_t)(P.sin[d] * es);
    box[d] = d == 0 ? kTmaBoxBytes : (d == b ? T->B : 1);
    estr[d] = 1;
  }
  if (enc(&T->map, CU_TENSOR_MAP_DATA_TYPE_UINT8, r, const_cast<void*>(in), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  // tile order: b fastest, then the other dims by increasing output stride
  int n = 0;
  T->ord[n] = b;
  T->cnt[n++] = (P.dims[b] + T->B - 1) / T->B;
  bool used[kTmaMaxRank] = {};
  used[b] = true;
  for (int k = 1; k < r; ++k) {
    int best = -1;
    for (int d = 0; d < r; ++d)
      if (!used[d] && (best < 0 || P.sout[d] < P.sout[best])) best = d;
    used[best] = true;
    T->ord[n] = best;
    T->cnt[n++] = best == 0 ? (P.dims[0] + (int64_t)T->nbx * T->A - 1) / ((int64_t)T->nbx * T->A) : P.dims[best];
  }
  T->ntiles = 1;
  for (int k = 0; k < r; ++k) T->ntiles *= T->cnt[k];
  return true;
}

namespace tmaperm {

__device__ __forceinline__ void load_box(void* dst, const CUtensorMap* map, int rank, const int* c, uint64_t* bar) {
  const uint32_t d = sm100::smem_u32(dst), mb = sm100::smem_u32(bar);
  const uint64_t m = (uint64_t)map;
  switch (rank) {
    case 2:
      asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(mb) : "memory");
      break;
    case 3:
      asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(mb) : "memory");
      break;
    case 4:
      asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(mb) : "memory");
      break;
    default:
      asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(mb) : "memory");
      break;
  }
}

struct TileHdr {
  int64_t out;     // output offset of the tile origin
  int ra, rb;      // valid extents along dim 0 and dim b
};

struct Smem {
  uint64_t full[kTmaPermStages];
  TileHdr hdr[kTmaPermStages];
};

// Origin of tile t: writes the box coordinates (bytes along dim 0) and the header.
__device__ __forceinline__ void origin(const TmaPermParams& P, int64_t t, int* c, TileHdr* h) {
  int64_t out = 0;
  int ra = P.nbx * P.A, rb = P.B;
  for (int k = 0; k < P.rank; ++k) {
    const int d = P.ord[k];
    const int64_t q = t / P.cnt[k];
    const int64_t digit = t - q * P.cnt[k];
    t = q;
    int64_t x = digit;
    if (d == 0) {
      x = digit * P.nbx * P.A;
      ra = (int)min((int64_t)P.nbx * P.A, P.ext[0] - x);
      c[0] = (int)(x * P.es);
    } else if (d == P.b) {
      x = digit * P.B;
      rb = (int)min((int64_t)P.B, P.ext[d] - x);
      c[d] = (int)x;
    } else {
      c[d] = (int)x;
    }
    out += x * P.sout[d];
  }
  h->out = out;
  h->ra = ra;
  h->rb = rb;
}

}  // namespace tmaperm

template <typename Elem, typename Store>
__global__ void __launch_bounds__(kPermThreads) perm_tma_kernel(const __grid_constant__ TmaPermParams P, Store st,
                                                                unsigned int* err) {
  using namespace tmaperm;
  extern __shared__ __align__(1024) unsigned char tma_smem_raw[];
  unsigned char* stages = (unsigned char*)(((uintptr_t)tma_smem_raw + 1023) & ~(uintptr_t)1023);
  const int stage_bytes = P.nbx * P.region;
  Smem* S = reinterpret_cast<Smem*>(stages + kTmaPermStages * stage_bytes);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int V = 16 / (int)sizeof(Elem);  // elements per 16-byte chunk
  if (tid == 0) {
    for (int s = 0; s < kTmaPermStages; ++s) sm100::mbar_init(&S->full[s], 1);
    sm100::fence_barrier_init();
    asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)&P.map) : "memory");
  }
  __syncthreads();
  const int64_t row_bytes = P.ext[0] * P.es;
  auto issue = [&](int64_t t, int s) {
    int c[kTmaMaxRank] = {0, 0, 0, 0, 0};
    origin(P, t, c, &S->hdr[s]);
    // boxes that start inside dim 0 (the last may run past its end: zero fill)
    const int nb = (int)min((int64_t)P.nbx, (row_bytes - c[0] + kTmaBoxBytes - 1) / kTmaBoxBytes);
    sm100::mbar_expect_tx(&S->full[s], (uint32_t)(nb * kTmaBoxBytes * P.B));
    const int c0 = c[0];
    for (int j = 0; j < nb; ++j) {
      c[0] = c0 + j * kTmaBoxBytes;
      load_box(stages + s * stage_bytes + j * P.region, &P.map, P.rank, c, &S->full[s]);
    }
  };
  if (tid == 0)
    for (int s = 0; s < kTmaPermStages; ++s) {
      const int64_t t = blockIdx.x + (int64_t)s * gridDim.x;
      if (t < P.ntiles) issue(t, s);
    }
  const int64_t sa = P.sout[0];
  constexpr int kChunks = kTmaBoxBytes / 16;  // 16-byte chunks per box row
  const int ntask = ((P.B + 31) / 32) * (P.nbx * kChunks);  // (row group, chunk) pairs
  int i = 0;
  for (int64_t t = blockIdx.x; t < P.ntiles; t += gridDim.x, ++i) {
    const int s = i % kTmaPermStages;
    const bool ok = sm100::mbar_wait(&S->full[s], (uint32_t)((i / kTmaPermStages) & 1), err, 21u);
    if (__syncthreads_or(!ok)) {
      // uniform: every thread leaves; first the other stages' loads still in
      // flight are waited for (bounded), so that none lands after the exit
      if (tid == 0)
        for (int k = 1; k < kTmaPermStages; ++k) {
          const int i2 = i + k;
          if (blockIdx.x + (int64_t)i2 * gridDim.x < P.ntiles)
            sm100::mbar_wait(&S->full[i2 % kTmaPermStages], (uint32_t)((i2 / kTmaPermStages) & 1), err, 21u);
        }
      break;
    }
    const TileHdr h = S->hdr[s];
    const unsigned char* sb = stages + s * stage_bytes;
    for (int task = warp; task < ntask; task += kPermThreads / 32) {
      const int g = task / (P.nbx * kChunks), qq = task - g * (P.nbx * kChunks);
      const int box = qq / kChunks, q = qq - box * kChunks;
      const int row = g * 32 + lane;  // index along b within the tile
      if (row < h.rb) {
        const uint4 v =
            *reinterpret_cast<const uint4*>(sb + box * P.region + row * kTmaBoxBytes + ((q ^ (row & 7)) << 4));
        const Elem* e = reinterpret_cast<const Elem*>(&v);
#pragma unroll
        for (int k = 0; k < V; ++k) {
          const int x = qq * V + k;
          if (x < h.ra) st(h.out + x * sa + row, e[k]);
        }
      }
    }
    __syncthreads();  // stage s read by every warp
    if (tid == 0) {
      const int64_t t2 = t + (int64_t)kTmaPermStages * gridDim.x;
      if (t2 < P.ntiles) issue(t2, s);
    }
  }
}

inline size_t perm_tma_smem_bytes(const TmaPermParams& T) {
  return 1024 + (size_t)kTmaPermStages * T.nbx * T.region + sizeof(tmaperm::Smem);
}

template <typename Elem, typename Store>
int launch_perm_tma(const TmaPermParams& T, const Store& st, cudaStream_t s) {
  if (T.ntiles <= 0) return 0;
  const size_t smem = perm_tma_smem_bytes(T);
  static DeviceOnce attr;
  const cudaError_t e =
      smem_limit_once(attr, perm_tma_kernel<Elem, Store>, (int)(1024 + kTmaPermStages * kTmaStageMax + 1024));
  if (e != cudaSuccess) { set_error("TMA permutation smem attribute: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
  static const bool trace = [] { const char* e = getenv("TB_PERM_TRACE"); return e && e[0] == '1'; }();
  if (trace)
    fprintf(stderr, "perm es=%d rank=%d b=%d B=%d boxes=%d tiles=%lld kernel=tma\n", T.es, T.rank, T.b, T.B, T.nbx,
            (long long)T.ntiles);
  const int per_sm = std::max(1, (int)((224 * 1024) / (smem + 1024)));
  const int64_t grid = std::min<int64_t>(T.ntiles, (int64_t)num_sms() * per_sm);
  perm_tma_kernel<Elem, Store><<<(unsigned)grid, kPermThreads, smem, s>>>(T, st, device_error_word());
  TB_CHECK_LAUNCH();
  return 0;
}

}  // namespace tb
