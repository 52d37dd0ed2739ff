// tb_blocks.cpp -- block-task lists of block-sparse contractions, built from
// the tensors' segment metadata.
//
// ExaTENSOR splits every index of a hierarchical tensor into segments; a block
// (subtensor) is one combination of segments.  TensContractionSplitFunc
// (INTRAVIRT/tensor_recursive.F90:9202-9784) builds the descriptor lists of
// the subtensors of D, L and R and matches them into the list of subtensor
// contractions, which TAVP-WRK then runs one talsh_tensor_contract at a time
// (INTERVIRT/tavp_worker.F90:9420-9518).  tb_bsc_tasks_from_blocks does the
// matching here and emits the list as tb_block_task_t entries for
// tb_bsc_plan_create / tb_batch_add:
//   * left and right blocks meet when their contracted segments agree;
//   * their output block is the D block whose segments are the left block's
//     (for D indices taken from L) and the right block's (from R); a pair
//     whose output block D does not hold produces no task;
//   * block extents come from the segment tables, and every index's
//     segmentation must agree between the tensors that carry it.
// Tasks are emitted in left-block order, right blocks in their list order.
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "talsh_b200.h"
#include "tb_pattern.h"

namespace tb {
namespace {

struct ListView {
  int rank;
  std::vector<const int*> seg;  // segment extents of index k
  std::vector<int> nseg;
};

int view_of(const tb_block_list_t* b, int rank, ListView* v, const char* name) {
  if (!b || b->rank != rank || (b->nblocks > 0 && (!b->keys || !b->bodies)) || b->nblocks < 0 ||
      (rank > 0 && (!b->nseg || !b->seg_ext))) {
    set_error("tb_bsc_tasks_from_blocks: block list of %s does not match the pattern (rank %d)", name, rank);
    return TB_ERR_INVALID_ARGS;
  }
  v->rank = rank;
  v->seg.resize(rank);
  v->nseg.resize(rank);
  int64_t off = 0;
  for (int k = 0; k < rank; ++k) {
    if (b->nseg[k] < 1) {
      set_error("tb_bsc_tasks_from_blocks: index %d of %s has no segments", k, name);
      return TB_ERR_INVALID_ARGS;
    }
    v->seg[k] = b->seg_ext + off;
    v->nseg[k] = b->nseg[k];
    for (int s = 0; s < b->nseg[k]; ++s)
      if (v->seg[k][s] < 1) {
        set_error("tb_bsc_tasks_from_blocks: segment %d of index %d of %s has extent %d", s, k, name, v->seg[k][s]);
        return TB_ERR_INVALID_ARGS;
      }
    off += b->nseg[k];
  }
  for (int i = 0; i < b->nblocks; ++i)
    for (int k = 0; k < rank; ++k) {
      const int s = b->keys[(int64_t)i * rank + k];
      if (s < 0 || s >= v->nseg[k]) {
        set_error("tb_bsc_tasks_from_blocks: block %d of %s names segment %d of index %d (of %d)", i, name, s, k,
                  v->nseg[k]);
        return TB_ERR_INVALID_ARGS;
      }
    }
  return 0;
}

bool same_segments(const ListView& a, int ka, const ListView& b, int kb) {
  return a.nseg[ka] == b.nseg[kb] && std::memcmp(a.seg[ka], b.seg[kb], sizeof(int) * a.nseg[ka]) == 0;
}

std::string key_of(const int* k, int n) { return std::string((const char*)k, sizeof(int) * (size_t)n); }

}  // namespace
}  // namespace tb

using namespace tb;

extern "C" int tb_bsc_tasks_from_blocks(const char* pattern, const tb_block_list_t* d, const tb_block_list_t* l,
                                        const tb_block_list_t* r, int max_tasks, tb_block_task_t* tasks,
                                        int* ntasks) {
  if (!pattern || !ntasks || max_tasks < 0 || (max_tasks > 0 && !tasks)) {
    set_error("tb_bsc_tasks_from_blocks: bad arguments");
    return TB_ERR_INVALID_ARGS;
  }
  *ntasks = 0;
  ParsedPattern P;
  if (parse_pattern(pattern, &P) || P.rrank < 0) {
    set_error("tb_bsc_tasks_from_blocks: not a contraction pattern: %s", pattern);
    return TB_ERR_INVALID_ARGS;
  }
  if (P.hyper || P.drank > 8 || P.lrank > 8 || P.rrank > 8) {
    set_error("tb_bsc_tasks_from_blocks: block tasks hold ranks up to 8 without hyper-indices");
    return TB_ERR_NOT_IMPLEMENTED;
  }
  ListView D, L, R;
  if (int e = view_of(d, P.drank, &D, "D")) return e;
  if (int e = view_of(l, P.lrank, &L, "L")) return e;
  if (int e = view_of(r, P.rrank, &R, "R")) return e;
  // index map: L index i -> D position or R position, R index j likewise
  std::vector<int> lcon, rcon;             // contracted positions, paired in R order
  std::vector<int> dsrc_op(P.drank, -1), dsrc_pos(P.drank, -1);
  for (int i = 0; i < P.lrank; ++i) {
    const int c = P.cptrn[i];
    if (c > 0) { dsrc_op[c - 1] = 0; dsrc_pos[c - 1] = i; }
  }
  for (int j = 0; j < P.rrank; ++j) {
    const int c = P.cptrn[P.lrank + j];
    if (c > 0) {
      dsrc_op[c - 1] = 1; dsrc_pos[c - 1] = j;
    } else {
      lcon.push_back(-c - 1);
      rcon.push_back(j);
    }
  }
  for (int p = 0; p < P.drank; ++p) {
    const ListView& S = dsrc_op[p] == 0 ? L : R;
    if (dsrc_op[p] < 0 || !same_segments(D, p, S, dsrc_pos[p])) {
      set_error("tb_bsc_tasks_from_blocks: index %d of D is segmented unlike its source", p);
      return TB_ERR_INVALID_ARGS;
    }
  }
  for (size_t c = 0; c < lcon.size(); ++c)
    if (!same_segments(L, lcon[c], R, rcon[c])) {
      set_error("tb_bsc_tasks_from_blocks: contracted index %d of L is segmented unlike index %d of R", lcon[c],
                rcon[c]);
      return TB_ERR_INVALID_ARGS;
    }
  // output blocks by key; right blocks grouped by their contracted segments
  std::unordered_map<std::string, int> dby;
  dby.reserve((size_t)d->nblocks * 2);
  for (int i = 0; i < d->nblocks; ++i)
    if (!dby.emplace(key_of(d->keys + (int64_t)i * P.drank, P.drank), i).second) {
      set_error("tb_bsc_tasks_from_blocks: block %d of D repeats a key", i);
      return TB_ERR_INVALID_ARGS;
    }
  const int nc = (int)rcon.size();
  std::unordered_map<std::string, std::vector<int>> rby;
  std::vector<int> kbuf(std::max(nc, P.drank) + 1);
  for (int j = 0; j < r->nblocks; ++j) {
    const int* rk = r->keys + (int64_t)j * P.rrank;
    for (int c = 0; c < nc; ++c) kbuf[c] = rk[rcon[c]];
    rby[key_of(kbuf.data(), nc)].push_back(j);
  }
  int64_t n = 0;
  for (int i = 0; i < l->nblocks; ++i) {
    const int* lk = l->keys + (int64_t)i * P.lrank;
    for (int c = 0; c < nc; ++c) kbuf[c] = lk[lcon[c]];
    auto it = rby.find(key_of(kbuf.data(), nc));
    if (it == rby.end()) continue;
    for (int j : it->second) {
      const int* rk = r->keys + (int64_t)j * P.rrank;
      for (int p = 0; p < P.drank; ++p) kbuf[p] = dsrc_op[p] == 0 ? lk[dsrc_pos[p]] : rk[dsrc_pos[p]];
      auto dt = dby.find(key_of(kbuf.data(), P.drank));
      if (dt == dby.end()) continue;  // D holds no such block
      if (n < max_tasks) {
        tb_block_task_t& t = tasks[n];
        std::memset(&t, 0, sizeof(t));
        t.d = d->bodies[dt->second];
        t.l = l->bodies[i];
        t.r = r->bodies[j];
        for (int p = 0; p < P.drank; ++p) t.d_dims[p] = D.seg[p][kbuf[p]];
        for (int a = 0; a < P.lrank; ++a) t.l_dims[a] = L.seg[a][lk[a]];
        for (int b = 0; b < P.rrank; ++b) t.r_dims[b] = R.seg[b][rk[b]];
      }
      if (++n > INT32_MAX) {
        set_error("tb_bsc_tasks_from_blocks: more than 2^31 tasks");
        return TB_ERR_LIMIT;
      }
    }
  }
  *ntasks = (int)n;
  if (tasks && n > max_tasks) {
    set_error("tb_bsc_tasks_from_blocks: %lld tasks, room for %d", (long long)n, max_tasks);
    return TB_ERR_LIMIT;
  }
  return 0;
}
