// tb_perm_plan.h -- host-side permutation plan (shared by the CUDA engine and
// the CPU emulation test of its index arithmetic).
//
// A permutation moves every element of a dense tensor to a new position.  The
// kernel stages one tile of the tensor in shared memory: the tile is a box
// whose input-fastest dimensions give contiguous input runs of at least
// 128 bytes ("load chunks") and whose output-fastest dimensions give
// contiguous output runs of at least 128 bytes ("store chunks").  Chunk base
// offsets and the shared-memory transposition map are computed here once per
// plan and passed to the kernel as a parameter.
#pragma once
#include <cstdint>
#include "tb_fastdiv.h"

namespace tb {

constexpr int kPlanMaxRank = 56;
constexpr int kMaxChunks = 256;   // load/store chunks per tile
constexpr int kMaxEjf = 64;       // entries of the store-chunk transposition table

// Device-side plan (passed by value as a __grid_constant__ kernel parameter).
struct PermParams {
  int rank;                  // reduced rank
  int es;                    // element bytes
  int V;                     // tile volume (elements)
  int LA, nA;                // load chunk length, number of load chunks
  int LB, nB;                // store chunk length, number of store chunks
  int pa, pb;                // partial dims (reduced indices) or -1
  int prodA, prodB;          // digit(pa) = j / prodA in a load chunk; digit(last store dim) = j' / prodB
  int ejf_n;                 // entries of ejf (= prodB)
  int ej_pb_stride;          // tile-index stride of the last store-block dim
  int lap;                   // shared-memory row stride (elements) of a load chunk
  int tma_ok;                // 1: load chunks can be moved by 16-byte-aligned bulk copies
  int64_t total;             // tensor volume (elements)
  int ngd;                   // grid dims
  int64_t ntiles;
  int64_t dims[kPlanMaxRank];
  int64_t tile[kPlanMaxRank];
  int64_t sin[kPlanMaxRank];
  int64_t sout[kPlanMaxRank];
  int gdim[kPlanMaxRank];        // reduced dim of each grid dim
  int64_t gext[kPlanMaxRank];    // tile positions along each grid dim
  FastDiv gdiv[kPlanMaxRank];    // divisors for gext
  // 32-bit magic divisors for gext, valid while ntiles < 2^31 (gd32 = 1): a
  // tile's origin then costs one 32x32->64 multiply and a shift per grid dim
  int gd32;
  uint32_t gmag[kPlanMaxRank];
  int gsh[kPlanMaxRank];
  uint32_t la_magic; int la_shift;   // 32-bit fast division by LA
  uint32_t lb_magic; int lb_shift;   // by LB
  uint32_t pb_magic; int pb_shift;   // by prodB
  int64_t ld_base[kMaxChunks];  // input offset of load chunk c (tile-relative)
  int16_t ld_dpb[kMaxChunks];   // digit of pb in load chunk c (-1: pb inside the chunk or none)
  int64_t st_base[kMaxChunks];  // output offset of store chunk c'
  int32_t st_ebase[kMaxChunks]; // shared-memory position base of store chunk c'
  int16_t st_dpa[kMaxChunks];   // digit of pa in store chunk c' (-1: pa inside the chunk or none)
  int32_t ejf[kMaxEjf];         // shared-memory position of j' % prodB inside a store chunk
  // Two-dimensional tiles (at most one dim outside the load block, at most one
  // outside the store block, single-dim store block): load row c starts at
  // c * row_sin in the input, store chunk c at c * chunk_sout in the output and
  // at c * chunk_eb in shared memory, and position j of a store chunk sits at
  // j * ej_pb_stride after it.  Lets the kernel skip the chunk tables.
  int lin2d;
  int row_is_pb, chunk_is_pa;   // the row (chunk) dim is the partial dim pb (pa)
  int64_t row_sin, chunk_sout;
  int32_t chunk_eb;
  // 2-D tiles whose store chunks are adjacent columns of vector-aligned rows
  // (chunk_eb == 1): the store phase reads vbytes (vbytes / es columns) per
  // lane and the load phase walks (row, vector) pairs.
  int vec2d;
  int vec8;                     // 4-byte elements: rows move as 8-byte copies (tma_ok: 16-byte)
  int vbytes;                   // vector bytes of the 2-D path: 16, 8 or 0
  int nvec;                     // vectors per full load row
  uint32_t nv_magic; int nv_shift;  // fast division by nvec
  // 2-D tiles whose store chunks are the load rows themselves (row copies:
  // the fastest dim stays fastest, one other dim moves): the store phase
  // moves whole vectors as well.  out_vec: every store run starts on a
  // vbytes boundary of the output (relative to an aligned output pointer).
  int rows2d;
  int out_vec;
  // Set by the caller, not the planner: long row copies (rows2d with rows of
  // 4 KB or more) run in the bulk-copy kernel instead of the 2-D kernel.
  int bulk_rows;
};

// Full-tile offset lists of the 2-D kernel.  A thread's i-th copy in a full
// tile is the linear position lin = tid + i * nthr of the tile's (outer p,
// inner q) grid in q-fastest order; it sits at shared-memory byte offset
// p*Ap + q*Aq and at global element offset p*Bp + q*Bq from the tile origin.
// The offsets are the same in every full tile, so the kernel computes them
// once.  The same function drives the CPU emulation of the kernel.
TB_HD void perm_list_entry(int lin, int nq, uint32_t Aq, uint32_t Ap, int32_t Bq, int32_t Bp, uint32_t* a,
                           int32_t* b) {
  const int p = lin / nq, q = lin - p * nq;
  *a = (uint32_t)p * Ap + (uint32_t)q * Aq;
  *b = (int32_t)((uint32_t)p * (uint32_t)Bp + (uint32_t)q * (uint32_t)Bq);
}

// Host-side plan builder.  dims/sin/sout describe the input dims (input
// strides, output strides), first dim fastest in the input.  Returns 0 or a
// TB_ERR code.  Dims of extent 1 are dropped and mergeable neighbours fused.
// vmin_kb / vmax_kb bound the tile's bytes (0: the defaults, 16 and 32 KB);
// min_run is the minimum contiguous run of the load and store blocks in bytes
// (0: the default, 256).
int build_perm_plan(int es, int rank, const int64_t* dims, const int64_t* sin, const int64_t* sout,
                    PermParams* p, int vmin_kb = 0, int vmax_kb = 0, int min_run = 0);
// Convenience: plain O2N permutation of a dense tensor (cptrn 1-based).
int build_perm_plan_o2n(int es, int rank, const int* dims, const int* cptrn, PermParams* p, int vmin_kb = 0,
                        int vmax_kb = 0, int min_run = 0);
// Entries per thread of the 2-D kernel's full-tile offset lists for a plan
// whose vector path is rows (row copies) or column groups (transposes): 8 or
// 16, or 0 when the lists would not cover a tile, an offset would not fit in
// 32 bits, or the last column group is ragged (the general code runs then).
int perm2d_list_entries(const PermParams& P, bool rows, int nthr);
// General-plan list kernel (perm_glist_kernel): entries per thread of its
// load and store lists, and the bytes of its load copies for a plan and an
// input pointer aligned to in_align bytes -- 16, 8 or one element -- or 0 when
// the plan does not fit the lists (more than kGListEntries * nthr elements or
// load copies per tile, or tile-relative offsets beyond 32 bits).
constexpr int kGListEntries = 16;
int perm_glist_vector_bytes(const PermParams& P, int in_align, int nthr);
// Bytes of one pipeline stage (a tile in shared memory).
inline int64_t perm_stage_bytes(const PermParams& P) { return (int64_t)P.nA * P.lap * P.es; }

}  // namespace tb
