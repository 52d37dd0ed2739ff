// tb_bsc.cu -- block-sparse contractions as one grouped tensor-core launch.
//
// A block-sparse contraction is a list of block tasks D_d += alpha * L * R
// under one index pattern, where several tasks may add into the same output
// block (ExaTENSOR's TAVP-WRK issues them one talsh_tensor_contract per block,
// INTERVIRT/tavp_worker.F90:9420-9518, call at :9467).  The plan built here
// converts every distinct operand block once (row maxima, then INT8 slices or
// BF16 parts, through per-block offset tables: two grouped launches over all
// blocks) and runs all (output tile, pair) work in one persistent grouped GEMM
// (tb_bsc_gemm.cuh) fed from a device-side queue.  The launch sequence is
// captured once in a CUDA graph and replayed.  An autotuner times the tile
// width and slice-count candidates on the plan's own data and keeps the
// fastest.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <unordered_map>
#include <vector>

#include "tb_bsc_gemm.cuh"
#include "tb_tc_prep.cuh"

namespace tb {
namespace {

int64_t rup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Host offset table: out[i] = sum_g digit_g(i) * (use_s2 ? s2 : s1)_g, first group fastest.
void host_offsets(const std::vector<MGroup>& gs, bool use_s2, std::vector<int64_t>& out) {
  int64_t n = 1;
  for (auto& g : gs) n *= g.ext;
  const size_t base = out.size();
  out.resize(base + (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    int64_t r = i, o = 0;
    for (auto& g : gs) {
      o += (r % g.ext) * (use_s2 ? g.s2 : g.s1);
      r /= g.ext;
    }
    out[base + (size_t)i] = o;
  }
}

struct OpBlock {          // one distinct operand block in the A (row) or B (column) role
  const void* ptr;
  std::vector<MGroup> rows, ks;
  int64_t R, K, Rpad, Kpad;
  size_t lm_off, lk_off, e_off;   // offsets into the table arrays (elements)
  size_t plane_off;               // bytes into the plane buffer
};

void* dalloc(size_t bytes, int* err) {
  void* p = nullptr;
  if (*err) return nullptr;
  if (cudaMalloc(&p, std::max<size_t>(bytes, 256)) != cudaSuccess) {
    cudaGetLastError();
    set_error("block-sparse plan: device allocation of %zu bytes failed", bytes);
    *err = TB_ERR_NO_MEMORY;
    return nullptr;
  }
  return p;
}

}  // namespace
}  // namespace tb

struct tb_bsc_plan_s {
  int dtk = 0;
  bool i8 = true;
  int slices = 6, bn = 256;        // current configuration
  int max_slices = 7;              // planes allocated for this many slices
  double ar = 1, ai = 0, br = 0, bi = 0;
  int n_a = 0, n_b = 0, n_d = 0, n_pairs = 0, n_items[2] = {0, 0};
  int64_t a_rowtiles = 0, b_rowtiles_max = 0;
  double flops = 0;
  int max_kblocks = 0;
  // device memory
  std::vector<void*> allocs;
  unsigned char* planes = nullptr;
  int64_t* tables = nullptr;       // lm/lk of every operand block, dm/dn of every output block
  unsigned* rowE = nullptr;        // exponent fields of every operand row (A rows then B rows)
  int* rowexp = nullptr;
  size_t n_erows = 0;
  tb::GatherParams* jobs = nullptr;  // A blocks then B blocks
  int2* rm_map = nullptr;          // rowmax grouped launch: (job, row tile)
  int2* g_map = nullptr;           // gather grouped launch
  int64_t rm_ctas = 0, g_ctas = 0;
  int rm_gy = 1, g_gy = 1;
  CUtensorMap* maps = nullptr;
  tb::BscDBlk* dblks = nullptr;
  tb::BscItem* items[2] = {nullptr, nullptr};  // items for BN = 128 / 256
  tb::BscPass* passes = nullptr;   // per output block, for the current slice count
  tb::BscRun* runs = nullptr;
  size_t passes_cap = 0, runs_cap = 0;
  std::vector<tb::BscDBlk> dblk_host;            // output blocks (pass and run ranges rewritten per slice count)
  std::vector<std::vector<int>> dpair_kb;       // K blocks of every pair of every output block
  std::vector<int> dpair0;                      // first global pair index of every output block
  std::vector<const CUtensorMap*> pair_maps;    // per global pair: A map, B map (BN 128), B map (BN 256)
  unsigned* queue = nullptr;
  // graph of the current configuration
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  float tune_ms[2][8] = {{0}};
};

namespace tb {
namespace {

template <int BN, bool I8, int EPI>
int launch_bsc(const BscParams& P, int grid, cudaStream_t s) {
  constexpr size_t smem = bsc_smem_bytes<BN>();
  static DeviceOnce attr;
  const cudaError_t e = smem_limit_once(attr, bsc_gemm_kernel<BN, I8, EPI>, (int)smem);
  if (e != cudaSuccess) { set_error("grouped GEMM smem attribute: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
  bsc_gemm_kernel<BN, I8, EPI><<<grid, kTcThreads, smem, s>>>(P);
  TB_CHECK_LAUNCH();
  return 0;
}

}  // namespace
}  // namespace tb

using namespace tb;

namespace {

// Queues the whole block-sparse contraction for the plan's current
// configuration on stream s (no allocation; capturable).
int bsc_enqueue(tb_bsc_plan_s* pl, cudaStream_t s) {
  const int bi = pl->bn == 256 ? 1 : 0;
  if (pl->i8) {
    if (cudaMemsetAsync(pl->rowE, 0, pl->n_erows * sizeof(unsigned), s) != cudaSuccess) return TB_ERR_CUDA;
    rowmax_grouped_kernel<false><<<dim3((unsigned)pl->rm_ctas, (unsigned)pl->rm_gy), kGThreads, 0, s>>>(pl->jobs,
                                                                                                       pl->rm_map);
    TB_CHECK_LAUNCH();
    exps_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)(pl->n_erows + 255) / 256, 4096)), 256, 0,
                  s>>>(pl->rowE, pl->rowexp, (int64_t)pl->n_erows, 1);
    TB_CHECK_LAUNCH();
  }
  // the gathers read the slice count from the jobs: keep them in sync with the configuration
  const cudaError_t ga = pl->i8 ? gather_grouped_prepare<G_SLICE_R8>() : gather_grouped_prepare<G_SPLIT_R4>();
  if (ga != cudaSuccess) { set_error("grouped gather smem attribute: %s", cudaGetErrorString(ga)); return TB_ERR_CUDA; }
  if (pl->i8)
    gather_grouped_kernel<G_SLICE_R8><<<dim3((unsigned)pl->g_ctas, (unsigned)pl->g_gy), kGThreads,
                                        gather_smem_bytes<G_SLICE_R8>(), s>>>(pl->jobs, pl->g_map);
  else
    gather_grouped_kernel<G_SPLIT_R4><<<dim3((unsigned)pl->g_ctas, (unsigned)pl->g_gy), kGThreads,
                                        gather_smem_bytes<G_SPLIT_R4>(), s>>>(pl->jobs, pl->g_map);
  TB_CHECK_LAUNCH();
  if (cudaMemsetAsync(pl->queue, 0, sizeof(unsigned), s) != cudaSuccess) return TB_ERR_CUDA;
  BscParams P;
  std::memset(&P, 0, sizeof(P));
  P.dblks = pl->dblks; P.items = pl->items[bi];
  P.queue = pl->queue; P.nitems = pl->n_items[bi];
  P.passes = pl->passes; P.runs = pl->runs;
  P.ar = pl->ar; P.ai = pl->ai; P.br = pl->br; P.bi = pl->bi;
  P.err = device_error_word();
  const int grid = std::max(1, std::min(P.nitems, num_sms()));
  int e;
  if (pl->bn == 256) e = pl->i8 ? launch_bsc<256, true, EPI_OZAKI_R>(P, grid, s) : launch_bsc<256, false, EPI_BF16_R>(P, grid, s);
  else e = pl->i8 ? launch_bsc<128, true, EPI_OZAKI_R>(P, grid, s) : launch_bsc<128, false, EPI_BF16_R>(P, grid, s);
  return e;
}

void drop_graph(tb_bsc_plan_s* pl) {
  if (pl->exec) cudaGraphExecDestroy(pl->exec);
  if (pl->graph) cudaGraphDestroy(pl->graph);
  pl->exec = nullptr;
  pl->graph = nullptr;
}

// Accumulator passes of every output block for the current slice count, and
// their runs (what the producer streams: one block pair's K range in one
// plane pair).
// INT8: slice pairs (i, j) of equal i + j share a pass while the K blocks
// summed into it stay within 1023 (each adds at most 128^3 = 2^21, so the
// INT32 sum is exact); a product over many pairs is split at pair boundaries.
// BF16: passes of at most kBscBf16PassKBlocks K blocks, each with the three
// products, over the pairs in order (a pass may end inside a pair's K range):
// the FP32 accumulation of the tensor cores loses accuracy with the length
// of the sum, and the epilogue adds each pass into D with one rounding.
constexpr int kBscBf16PassKBlocks = 32;
void plan_passes(const tb_bsc_plan_s* pl, int S, std::vector<BscPass>& passes, std::vector<BscRun>& runs,
                 std::vector<BscDBlk>* dbl) {
  passes.clear();
  runs.clear();
  const bool maps = !pl->pair_maps.empty();
  auto new_pass = [&](int shift) { passes.push_back(BscPass{(int)runs.size(), 0, shift, 0}); };
  // run of global pair q over K blocks [k0, k1) in planes (a, b), added to the last pass
  auto add_run = [&](int q, int a, int b, int k0, int k1) {
    BscRun r{};
    if (maps) {
      r.amap = pl->pair_maps[3 * (size_t)q];
      r.bmap[0] = pl->pair_maps[3 * (size_t)q + 1];
      r.bmap[1] = pl->pair_maps[3 * (size_t)q + 2];
    }
    r.a = a; r.b = b; r.kb0 = k0; r.kb1 = k1;
    runs.push_back(r);
    passes.back().nrun++;
  };
  for (size_t d = 0; d < pl->dpair_kb.size(); ++d) {
    const std::vector<int>& kb = pl->dpair_kb[d];
    const int p0 = pl->dpair0[d], np = (int)kb.size();
    const int pass0 = (int)passes.size(), run0 = (int)runs.size();
    if (!pl->i8) {
      int load = kBscBf16PassKBlocks;  // forces a new pass first
      for (int q = 0; q < np; ++q) {
        for (int k0 = 0; k0 < kb[q];) {
          if (load >= kBscBf16PassKBlocks) {
            new_pass(0);
            load = 0;
          }
          const int n = std::min(kBscBf16PassKBlocks - load, kb[q] - k0);
          const int terms[3][2] = {{0, 0}, {0, 1}, {1, 0}};
          for (auto& t : terms) add_run(p0 + q, t[0], t[1], k0, k0 + n);
          load += n;
          k0 += n;
        }
      }
    } else {
      for (int dsum = 2; dsum <= S + 1; ++dsum) {
        int load = 1 << 30;  // forces a new pass for every diagonal
        for (int i = 1; i < dsum; ++i) {
          const int j = dsum - i;
          if (i > S || j > S) continue;
          for (int q = 0; q < np; ++q) {
            if (load + kb[q] > 1023) {
              new_pass(8 * dsum - 2);
              load = 0;
            }
            add_run(p0 + q, i - 1, j - 1, 0, kb[q]);
            load += kb[q];
          }
        }
      }
    }
    for (size_t p = pass0; p < passes.size(); ++p) {
      runs[passes[p].run0].flags |= kBscRunFirst;
      runs[passes[p].run0 + passes[p].nrun - 1].flags |= kBscRunLast;
    }
    if (dbl) {
      (*dbl)[d].pass0 = pass0;
      (*dbl)[d].npass = (int)passes.size() - pass0;
      (*dbl)[d].run0 = run0;
      (*dbl)[d].nrun = (int)runs.size() - run0;
    }
  }
}

int build_passes(tb_bsc_plan_s* pl, cudaStream_t s) {
  std::vector<BscPass> passes;
  std::vector<BscRun> runs;
  plan_passes(pl, pl->slices, passes, runs, &pl->dblk_host);
  if (passes.size() > pl->passes_cap || runs.size() > pl->runs_cap) {
    set_error("block-sparse plan: pass table larger than allocated");
    return TB_ERR_LIMIT;
  }
  if (cudaMemcpyAsync(pl->passes, passes.data(), passes.size() * sizeof(BscPass), cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(pl->runs, runs.data(), runs.size() * sizeof(BscRun), cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(pl->dblks, pl->dblk_host.data(), pl->dblk_host.size() * sizeof(BscDBlk), cudaMemcpyHostToDevice,
                      s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    set_error("block-sparse plan: pass table upload failed");
    return TB_ERR_CUDA;
  }
  return 0;
}

// Sets the slice count used by the gathers (stored in the job table).
int set_slices(tb_bsc_plan_s* pl, int S, cudaStream_t s) {
  const int n = pl->n_a + pl->n_b;
  std::vector<GatherParams> J((size_t)n);
  if (cudaMemcpyAsync(J.data(), pl->jobs, sizeof(GatherParams) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return TB_ERR_CUDA;
  for (auto& j : J) j.slices = S;
  if (cudaMemcpyAsync(pl->jobs, J.data(), sizeof(GatherParams) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return TB_ERR_CUDA;
  pl->slices = S;
  return build_passes(pl, s);
}

}  // namespace

namespace {

void plan_free(tb_bsc_plan_s* pl) {
  drop_graph(pl);
  for (void* p : pl->allocs) cudaFree(p);
  delete pl;
}

template <typename T>
T* upload(tb_bsc_plan_s* pl, const std::vector<T>& v, int* err, cudaStream_t s) {
  T* d = (T*)dalloc(sizeof(T) * std::max<size_t>(1, v.size()), err);
  if (!d) return nullptr;
  pl->allocs.push_back(d);
  if (!v.empty() && cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s) != cudaSuccess) {
    cudaGetLastError();
    set_error("block-sparse plan: upload failed");
    *err = TB_ERR_CUDA;
  }
  return d;
}

int plan_create(const char* pattern, int dtk, int ntasks, const tb_block_task_t* tasks, double ar, double ai,
                int accumulative, const tb_plan_t* plan, tb_bsc_plan_s** out, cudaStream_t s) {
  *out = nullptr;
  if (!pattern || !tasks || ntasks < 1) { set_error("tb_bsc_plan_create: no tasks"); return TB_ERR_INVALID_ARGS; }
  if (dtk != kR8 && dtk != kR4) {
    set_error("tb_bsc_plan_create: data kind %d not supported (R4 and R8 only)", dtk);
    return TB_ERR_NOT_IMPLEMENTED;
  }
  ParsedPattern PP;
  if (parse_pattern(pattern, &PP) || PP.rrank < 0) {
    set_error("tb_bsc_plan_create: bad contraction pattern \"%s\"", pattern);
    return TB_ERR_PATTERN;
  }
  if (PP.hyper) { set_error("tb_bsc_plan_create: hyper-contractions are not supported"); return TB_ERR_NOT_IMPLEMENTED; }
  if (PP.drank > 8 || PP.lrank > 8 || PP.rrank > 8) { set_error("tb_bsc_plan_create: rank above 8"); return TB_ERR_LIMIT; }
  // Role of the operands: the one holding D's first (fastest) dimension gives the rows.
  bool swap = true;
  for (int i = 0; i < PP.lrank; ++i)
    if (PP.cptrn[i] == 1) swap = false;
  auto* pl = new tb_bsc_plan_s();
  pl->dtk = dtk;
  pl->i8 = dtk == kR8;
  {
    // attribute set here, before any graph capture of the plan's launches
    const cudaError_t ga = pl->i8 ? gather_grouped_prepare<G_SLICE_R8>() : gather_grouped_prepare<G_SPLIT_R4>();
    if (ga != cudaSuccess) {
      set_error("grouped gather smem attribute: %s", cudaGetErrorString(ga));
      delete pl;
      return TB_ERR_CUDA;
    }
  }
  pl->slices = pl->i8 ? ((plan && plan->slices >= 2 && plan->slices <= 7) ? plan->slices : 6) : 2;
  pl->max_slices = pl->i8 ? std::max(pl->slices, 6) : 2;  // planes allocated (the autotuner stays within them)
  pl->bn = (plan && plan->tile_n == 128) ? 128 : 256;
  pl->ar = std::abs(ai) > 0 ? (ar != 0.0 ? std::hypot(ar, ai) * (ar > 0 ? 1.0 : -1.0) : ai) : ar;
  pl->br = accumulative ? 1.0 : 0.0;
  // distinct blocks
  std::vector<OpBlock> A, B;
  std::unordered_map<const void*, int> amap, bmap, dmap;
  struct DInfo { void* ptr; std::vector<MGroup> mrows, nrows; int64_t M, N; std::vector<std::pair<int, int>> pairs; };
  std::vector<DInfo> Ds;
  auto by_d = [](const MGroup& x, const MGroup& y) { return x.s2 < y.s2; };
  for (int t = 0; t < ntasks; ++t) {
    const tb_block_task_t& T = tasks[t];
    Matricization Z;
    int e = matricize(PP.cptrn, PP.drank, T.d_dims, PP.lrank, T.l_dims, PP.rrank, T.r_dims, &Z);
    if (e || !T.d || !T.l || !T.r) {
      set_error("tb_bsc_plan_create: task %d does not match the pattern (code %d)", t, e);
      plan_free(pl);
      return e ? e : TB_ERR_INVALID_ARGS;
    }
    if (Z.m.empty() || Z.n.empty() || Z.k.empty()) {
      set_error("tb_bsc_plan_create: task %d is not a matrix product (empty row, column or contracted set)", t);
      plan_free(pl);
      return TB_ERR_NOT_IMPLEMENTED;
    }
    std::stable_sort(Z.m.begin(), Z.m.end(), by_d);
    std::stable_sort(Z.n.begin(), Z.n.end(), by_d);
    std::vector<MGroup> lk, rk;
    for (auto g : Z.k) { lk.push_back(g); MGroup h = g; h.s1 = g.s2; rk.push_back(h); }
    const void* aptr = swap ? T.r : T.l;
    const void* bptr = swap ? T.l : T.r;
    const std::vector<MGroup>& arows = swap ? Z.n : Z.m;
    const std::vector<MGroup>& brows = swap ? Z.m : Z.n;
    const std::vector<MGroup>& aks = swap ? rk : lk;
    const std::vector<MGroup>& bks = swap ? lk : rk;
    auto add = [&](std::vector<OpBlock>& V, std::unordered_map<const void*, int>& mp, const void* ptr,
                   const std::vector<MGroup>& rows, const std::vector<MGroup>& ks) -> int {
      int64_t R = 1, K = 1;
      for (auto& g : rows) R *= g.ext;
      for (auto& g : ks) K *= g.ext;
      auto it = mp.find(ptr);
      if (it != mp.end()) {
        const OpBlock& o = V[it->second];
        return (o.R == R && o.K == K) ? it->second : -1;
      }
      OpBlock o;
      o.ptr = ptr; o.rows = rows; o.ks = ks; o.R = R; o.K = K;
      V.push_back(o);
      mp[ptr] = (int)V.size() - 1;
      return (int)V.size() - 1;
    };
    const int ia = add(A, amap, aptr, arows, aks), ib = add(B, bmap, bptr, brows, bks);
    if (ia < 0 || ib < 0 || A[ia].K != B[ib].K) {
      set_error("tb_bsc_plan_create: task %d reuses a block with different extents", t);
      plan_free(pl);
      return TB_ERR_INVALID_ARGS;
    }
    auto dit = dmap.find(T.d);
    int id;
    if (dit == dmap.end()) {
      DInfo di;
      di.ptr = T.d;
      di.mrows = swap ? Z.n : Z.m;  // D strides (s2) of the A rows
      di.nrows = swap ? Z.m : Z.n;
      di.M = A[ia].R; di.N = B[ib].R;
      Ds.push_back(di);
      id = (int)Ds.size() - 1;
      dmap[T.d] = id;
    } else {
      id = dit->second;
      if (Ds[id].M != A[ia].R || Ds[id].N != B[ib].R) {
        set_error("tb_bsc_plan_create: task %d adds a product of another shape into an output block", t);
        plan_free(pl);
        return TB_ERR_INVALID_ARGS;
      }
    }
    Ds[id].pairs.push_back({ia, ib});
    pl->flops += 2.0 * (double)A[ia].R * (double)B[ib].R * (double)A[ia].K;
  }
  pl->n_a = (int)A.size(); pl->n_b = (int)B.size(); pl->n_d = (int)Ds.size(); pl->n_pairs = ntasks;
  // Operand blocks that meet in an output block must share row (column)
  // scales: union the A blocks (B blocks) of every output block.
  std::vector<int> ua(A.size()), ub(B.size());
  std::iota(ua.begin(), ua.end(), 0);
  std::iota(ub.begin(), ub.end(), 0);
  auto find = [](std::vector<int>& u, int x) {
    while (u[x] != x) x = u[x] = u[u[x]];
    return x;
  };
  for (auto& d : Ds)
    for (auto& pr : d.pairs) {
      ua[find(ua, pr.first)] = find(ua, d.pairs[0].first);
      ub[find(ub, pr.second)] = find(ub, d.pairs[0].second);
    }
  // sizes, tables, planes
  const int oes = pl->i8 ? 1 : 2;
  const int np = pl->i8 ? pl->max_slices : 2;
  std::vector<int64_t> tab;
  size_t plane_bytes = 0, erows = 0;
  int max_kb = 0;
  for (auto* V : {&A, &B}) {
    const bool isb = V == &B;
    std::vector<int>& u = isb ? ub : ua;
    std::vector<size_t> comp_off(V->size(), SIZE_MAX);
    for (size_t i = 0; i < V->size(); ++i) {
      OpBlock& o = (*V)[i];
      o.Rpad = rup(o.R, isb ? 256 : 128);
      o.Kpad = rup(o.K, 128);
      max_kb = std::max<int>(max_kb, (int)(o.Kpad * oes / 128));
      o.lm_off = tab.size(); host_offsets(o.rows, false, tab);
      o.lk_off = tab.size(); host_offsets(o.ks, false, tab);
      const int c = find(u, (int)i);  // exponent rows are per component (same row count by construction)
      if (comp_off[c] == SIZE_MAX) { comp_off[c] = erows; erows += (size_t)o.R; }
      o.e_off = comp_off[c];
      o.plane_off = plane_bytes;
      plane_bytes += (size_t)np * o.Rpad * o.Kpad * oes;
      plane_bytes = (plane_bytes + 255) & ~size_t(255);
    }
  }
  if (max_kb > 1023) { set_error("tb_bsc_plan_create: a block K above 130944"); plan_free(pl); return TB_ERR_LIMIT; }
  pl->max_kblocks = max_kb;
  std::vector<size_t> dm_off(Ds.size()), dn_off(Ds.size());
  for (size_t d = 0; d < Ds.size(); ++d) {
    dm_off[d] = tab.size(); host_offsets(Ds[d].mrows, true, tab);
    dn_off[d] = tab.size(); host_offsets(Ds[d].nrows, true, tab);
  }
  int err = 0;
  pl->tables = upload(pl, tab, &err, s);
  pl->planes = (unsigned char*)dalloc(plane_bytes, &err);
  if (pl->planes) pl->allocs.push_back(pl->planes);
  pl->n_erows = erows;
  pl->rowE = (unsigned*)dalloc(erows * sizeof(unsigned), &err);
  if (pl->rowE) pl->allocs.push_back(pl->rowE);
  pl->rowexp = (int*)dalloc(erows * sizeof(int), &err);
  if (pl->rowexp) pl->allocs.push_back(pl->rowexp);
  pl->queue = (unsigned*)dalloc(sizeof(unsigned), &err);
  if (pl->queue) pl->allocs.push_back(pl->queue);
  if (err) { plan_free(pl); return err; }
  // gather jobs (A blocks, then B blocks) and their CTA maps
  std::vector<GatherParams> jobs;
  std::vector<int2> rm_map, g_map;
  int64_t max_kt = 1;
  for (auto* V : {&A, &B}) {
    for (auto& o : *V) {
      GatherParams G{};
      G.src = o.ptr;
      G.lm = pl->tables + o.lm_off;
      G.lk = pl->tables + o.lk_off;
      G.rows = o.R; G.K = o.K; G.kpad = o.Kpad; G.pstride = o.Rpad * o.Kpad;
      G.planes = pl->planes + o.plane_off;
      G.rowE = pl->rowE + o.e_off;
      G.slices = pl->slices;
      G.lanes_on_k = (o.ks[0].s1 == 1 || o.rows[0].s1 != 1) ? 1 : 0;
      G.isign = 1.0;
      const int job = (int)jobs.size();
      jobs.push_back(G);
      for (int64_t t = 0; t < (o.R + 63) / 64; ++t) rm_map.push_back(make_int2(job, (int)t));
      for (int64_t t = 0; t < o.Rpad / 64; ++t) g_map.push_back(make_int2(job, (int)t));
      max_kt = std::max<int64_t>(max_kt, o.Kpad / kGK);
    }
  }
  pl->jobs = upload(pl, jobs, &err, s);
  pl->rm_map = upload(pl, rm_map, &err, s);
  pl->g_map = upload(pl, g_map, &err, s);
  pl->rm_ctas = (int64_t)rm_map.size();
  pl->g_ctas = (int64_t)g_map.size();
  const int64_t want = (int64_t)num_sms() * 16;
  pl->rm_gy = (int)std::max<int64_t>(1, std::min<int64_t>(max_kt, want / std::max<int64_t>(1, pl->rm_ctas)));
  pl->g_gy = (int)std::max<int64_t>(1, std::min<int64_t>(max_kt, want / std::max<int64_t>(1, pl->g_ctas)));
  if (pl->rm_ctas > INT32_MAX || pl->g_ctas > INT32_MAX) { plan_free(pl); return TB_ERR_LIMIT; }
  // tensor maps: A (128-row boxes), B for BN = 128 and 256
  std::vector<CUtensorMap> maps((size_t)A.size() + 2 * B.size());
  for (size_t i = 0; i < A.size() && !err; ++i)
    err = make_operand_map(&maps[i], pl->planes + A[i].plane_off, pl->i8, A[i].Kpad, A[i].Rpad, np, 128);
  for (size_t i = 0; i < B.size() && !err; ++i) {
    err = make_operand_map(&maps[A.size() + i], pl->planes + B[i].plane_off, pl->i8, B[i].Kpad, B[i].Rpad, np, 128);
    if (!err)
      err = make_operand_map(&maps[A.size() + B.size() + i], pl->planes + B[i].plane_off, pl->i8, B[i].Kpad,
                             B[i].Rpad, np, 256);
  }
  pl->maps = upload(pl, maps, &err, s);
  if (err) { plan_free(pl); return err; }
  // output blocks, their pairs (tensor maps and K blocks) and work items (largest first)
  std::vector<BscDBlk>& dbl = pl->dblk_host;
  dbl.assign(Ds.size(), BscDBlk{});
  pl->dpair_kb.assign(Ds.size(), {});
  pl->dpair0.assign(Ds.size(), 0);
  pl->pair_maps.clear();
  int npairs = 0;
  for (size_t d = 0; d < Ds.size(); ++d) {
    dbl[d].D = Ds[d].ptr;
    dbl[d].dm = pl->tables + dm_off[d];
    dbl[d].dn = pl->tables + dn_off[d];
    // the block's A (B) blocks share one exponent component
    dbl[d].rowexp = pl->rowexp + A[Ds[d].pairs[0].first].e_off;
    dbl[d].colexp = pl->rowexp + B[Ds[d].pairs[0].second].e_off;
    dbl[d].M = (int)Ds[d].M; dbl[d].N = (int)Ds[d].N;
    pl->dpair0[d] = npairs;
    for (auto& p : Ds[d].pairs) {
      pl->pair_maps.push_back(pl->maps + p.first);
      pl->pair_maps.push_back(pl->maps + A.size() + p.second);
      pl->pair_maps.push_back(pl->maps + A.size() + B.size() + p.second);
      pl->dpair_kb[d].push_back((int)(A[p.first].Kpad * oes / 128));
      ++npairs;
    }
  }
  {
    std::vector<BscPass> ps;
    std::vector<BscRun> rs;
    plan_passes(pl, pl->i8 ? pl->max_slices : 2, ps, rs, nullptr);  // the largest tables any slice count needs
    pl->passes_cap = ps.size();
    pl->runs_cap = rs.size();
    pl->passes = (BscPass*)dalloc(ps.size() * sizeof(BscPass), &err);
    if (pl->passes) pl->allocs.push_back(pl->passes);
    pl->runs = (BscRun*)dalloc(rs.size() * sizeof(BscRun), &err);
    if (pl->runs) pl->allocs.push_back(pl->runs);
  }
  pl->dblks = upload(pl, dbl, &err, s);
  if (!err) err = build_passes(pl, s);
  // Items of one output block go N tile by N tile, every M tile of an N tile
  // before the next N tile: the CTAs working at the same time share one B slab
  // and stream consecutive A slabs.  On the full block-sparse configuration
  // this order ran 1974 ms against 2051, 2113, 2196, 2269 and 2360 ms for
  // bands of 2, 3, 4, 6 and 12 N tiles (M tiles inner within a band) and
  // 2791 ms for M tile by M tile, all on one GPU.
  for (int bi = 0; bi < 2; ++bi) {
    const int BN = bi ? 256 : 128;
    std::vector<std::pair<int64_t, BscItem>> its;
    for (size_t d = 0; d < Ds.size(); ++d) {
      int64_t cost = 0;
      for (auto& p : Ds[d].pairs) cost += A[p.first].Kpad;
      const int mt = (int)((Ds[d].M + 127) / 128), nt = (int)((Ds[d].N + BN - 1) / BN);
      for (int y = 0; y < nt; ++y)
        for (int x = 0; x < mt; ++x) its.push_back({cost, BscItem{(int)d, x, y, 0}});
    }
    std::stable_sort(its.begin(), its.end(), [](const std::pair<int64_t, BscItem>& a, const std::pair<int64_t, BscItem>& b) {
      return a.first > b.first;
    });
    std::vector<BscItem> v;
    for (auto& x : its) v.push_back(x.second);
    pl->items[bi] = upload(pl, v, &err, s);
    pl->n_items[bi] = (int)v.size();
  }
  if (!err && cudaStreamSynchronize(s) != cudaSuccess) { cudaGetLastError(); err = TB_ERR_CUDA; }
  if (err) { plan_free(pl); return err; }
  *out = pl;
  return 0;
}

}  // namespace

namespace {

int bsc_prepare_attrs() {
  // attributes set outside any stream capture
  const size_t s128 = bsc_smem_bytes<128>(), s256 = bsc_smem_bytes<256>();
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(bsc_gemm_kernel<128, true, EPI_OZAKI_R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s128);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(bsc_gemm_kernel<256, true, EPI_OZAKI_R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s256);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(bsc_gemm_kernel<128, false, EPI_BF16_R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s128);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(bsc_gemm_kernel<256, false, EPI_BF16_R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s256);
  if (e != cudaSuccess) { cudaGetLastError(); set_error("grouped GEMM attributes: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
  return 0;
}

int kernels_per_run(const tb_bsc_plan_s* pl) { return pl->i8 ? 4 : 2; }

// Captures the current configuration into a CUDA graph (on a private stream).
int build_graph(tb_bsc_plan_s* pl) {
  drop_graph(pl);
  cudaStream_t cs;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) { cudaGetLastError(); return TB_ERR_CUDA; }
  int err = 0;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    err = TB_ERR_CUDA;
  } else {
    err = bsc_enqueue(pl, cs);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    if (!err && (e != cudaSuccess || !g)) { cudaGetLastError(); err = TB_ERR_CUDA; }
    if (!err) {
      pl->graph = g;
      if (cudaGraphInstantiate(&pl->exec, g, 0) != cudaSuccess) { cudaGetLastError(); err = TB_ERR_CUDA; }
    } else if (g) {
      cudaGraphDestroy(g);
    }
  }
  cudaStreamDestroy(cs);
  if (err) { set_error("block-sparse plan: graph capture failed"); drop_graph(pl); }
  return err;
}

}  // namespace

extern "C" int tb_bsc_plan_create(const char* pattern, int data_kind, int ntasks, const tb_block_task_t* tasks,
                                  double alpha_real, double alpha_imag, int accumulative, const tb_plan_t* plan,
                                  tb_bsc_plan_t** out, void* stream) {
  if (!out) { set_error("tb_bsc_plan_create: null output"); return TB_ERR_INVALID_ARGS; }
  if (!device_error_word()) { set_error("tb_bsc_plan_create: device error word unavailable"); return TB_ERR_CUDA; }
  if (int e = bsc_prepare_attrs()) return e;
  tb_bsc_plan_s* pl = nullptr;
  int e = plan_create(pattern, data_kind, ntasks, tasks, alpha_real, alpha_imag, accumulative, plan, &pl,
                      (cudaStream_t)stream);
  if (e) return e;
  *out = pl;
  return 0;
}

extern "C" int tb_bsc_execute(tb_bsc_plan_t* pl, void* stream) {
  if (!pl) { set_error("tb_bsc_execute: null plan"); return TB_ERR_INVALID_ARGS; }
  if (!pl->exec)
    if (int e = build_graph(pl)) return e;
  if (cudaGraphLaunch(pl->exec, (cudaStream_t)stream) != cudaSuccess) {
    cudaError_t e = cudaGetLastError();
    set_error("tb_bsc_execute: %s", cudaGetErrorString(e));
    return TB_ERR_CUDA;
  }
  for (int i = 0; i < kernels_per_run(pl); ++i) count_launch();
  return 0;
}

extern "C" int tb_bsc_execute_stream(tb_bsc_plan_t* pl, void* stream) {
  if (!pl) { set_error("tb_bsc_execute_stream: null plan"); return TB_ERR_INVALID_ARGS; }
  return bsc_enqueue(pl, (cudaStream_t)stream);
}

extern "C" int tb_bsc_autotune(tb_bsc_plan_t* pl, void* stream) {
  if (!pl) { set_error("tb_bsc_autotune: null plan"); return TB_ERR_INVALID_ARGS; }
  cudaStream_t s = (cudaStream_t)stream;
  // The timed runs use alpha = 0, beta = 1: the same work, D left unchanged.
  const double ar = pl->ar, ai = pl->ai, br = pl->br, bi = pl->bi;
  const int s0 = pl->slices, bn0 = pl->bn;
  pl->ar = 0.0; pl->ai = 0.0; pl->br = 1.0; pl->bi = 0.0;
  const int cand_s[2] = {6, 7};
  const int ns = pl->i8 ? (pl->max_slices >= 7 ? 2 : 1) : 1;
  float best = 1e30f;
  int bs = s0, bbn = bn0, err = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int si = 0; si < ns && !err; ++si) {
    if (pl->i8 && (err = set_slices(pl, cand_s[si], s))) break;
    for (int bi2 = 0; bi2 < 2 && !err; ++bi2) {
      pl->bn = bi2 ? 256 : 128;
      if ((err = bsc_enqueue(pl, s))) break;  // warm-up
      cudaEventRecord(e0, s);
      for (int r = 0; r < 2 && !err; ++r) err = bsc_enqueue(pl, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) { cudaGetLastError(); err = TB_ERR_CUDA; break; }
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= 2;
      pl->tune_ms[bi2][si] = ms;
      if (ms < best) { best = ms; bs = pl->i8 ? cand_s[si] : s0; bbn = pl->bn; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  pl->ar = ar; pl->ai = ai; pl->br = br; pl->bi = bi;
  pl->bn = err ? bn0 : bbn;
  if (pl->i8) {
    int e2 = set_slices(pl, err ? s0 : bs, s);
    if (!err) err = e2;
  }
  drop_graph(pl);
  return err;
}

extern "C" int tb_bsc_plan_info(const tb_bsc_plan_t* pl, tb_bsc_info_t* info) {
  if (!pl || !info) return TB_ERR_INVALID_ARGS;
  std::memset(info, 0, sizeof(*info));
  info->tasks = pl->n_pairs;
  info->left_blocks = pl->n_a;
  info->right_blocks = pl->n_b;
  info->out_blocks = pl->n_d;
  info->work_items = pl->n_items[pl->bn == 256 ? 1 : 0];
  info->slices = pl->i8 ? pl->slices : 0;
  info->tile_n = pl->bn;
  info->flops = pl->flops;
  for (int b = 0; b < 2; ++b)
    for (int s = 0; s < 2; ++s) info->tune_ms[b * 2 + s] = pl->tune_ms[b][s];
  return 0;
}

extern "C" int tb_bsc_plan_destroy(tb_bsc_plan_t* pl) {
  if (!pl) return 0;
  cudaDeviceSynchronize();
  plan_free(pl);
  return 0;
}
