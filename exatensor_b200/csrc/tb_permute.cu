// tb_permute.cu -- permutation plans, tiled and scatter permutation kernels,
// and the tb_tensor_copy / tb_tensor_add entry points.
#include "tb_permute.cuh"
#include "tb_perm_tma.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

namespace tb {

// ---------------------------------------------------------------------------
// Scatter permutation: one element per thread (the plain reference form).
// ---------------------------------------------------------------------------
struct ScatterParams {
  int rank;
  int64_t vol;
  FastDiv div[kMaxRank];
  int64_t dims[kMaxRank];
  int64_t sout[kMaxRank];
};

template <typename E, typename Store>
__global__ void scatter_kernel(const __grid_constant__ ScatterParams P, const E* __restrict__ in, Store st) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P.vol;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t r = (uint64_t)i;
    int64_t o = 0;
    for (int d = 0; d < P.rank; ++d) {
      uint64_t q = P.div[d].div(r);
      o += (int64_t)(r - q * (uint64_t)P.dims[d]) * P.sout[d];
      r = q;
    }
    st(o, in[i]);
  }
}

namespace {

int o2n_strides(int rank, const int* dims, const int* cptrn, int64_t* sout) {
  int seen[kMaxRank + 1] = {0};
  int64_t oe[kMaxRank], pos[kMaxRank];
  for (int i = 0; i < rank; ++i) {
    if (cptrn[i] < 1 || cptrn[i] > rank || seen[cptrn[i]]) return TB_ERR_PATTERN;
    seen[cptrn[i]] = 1;
    oe[cptrn[i] - 1] = dims[i];
  }
  int64_t s = 1;
  for (int q = 0; q < rank; ++q) { pos[q] = s; s *= oe[q]; }
  for (int i = 0; i < rank; ++i) sout[i] = pos[cptrn[i] - 1];
  return 0;
}

int check_dims(int rank, const int* dims, int64_t* vol) {
  if (rank < 0 || rank > kMaxRank || (rank > 0 && !dims)) return TB_ERR_INVALID_ARGS;
  int64_t v = 1;
  for (int i = 0; i < rank; ++i) { if (dims[i] <= 0) return TB_ERR_INVALID_ARGS; v *= dims[i]; }
  *vol = v;
  return 0;
}

template <typename E, typename Store>
int run_scatter(int rank, const int* dims, const int* cptrn, const E* in, const Store& st,
                cudaStream_t s) {
  ScatterParams P;
  std::memset(&P, 0, sizeof(P));
  int64_t vol;
  if (int e = check_dims(rank, dims, &vol)) return e;
  int64_t sout[kMaxRank];
  if (int e = o2n_strides(rank, dims, cptrn, sout)) return e;
  P.rank = rank; P.vol = vol;
  for (int i = 0; i < rank; ++i) { P.dims[i] = dims[i]; P.sout[i] = sout[i]; P.div[i].init(dims[i]); }
  int64_t blocks = std::min<int64_t>((vol + 255) / 256, (int64_t)num_sms() * 16);
  if (blocks < 1) blocks = 1;
  scatter_kernel<E, Store><<<(unsigned)blocks, 256, 0, s>>>(P, in, st);
  TB_CHECK_LAUNCH();
  return 0;
}

// Fused permute + add: d = d + v*a with two roundings (no FMA), complex
// products by the textbook formula, the left operand optionally conjugated.
// Each functor reads the output it updates: load(o) and put(o, v, old) let the
// list kernels issue a batch of output loads before the dependent writes.
template <typename R>
struct AddScalar {
  R* out; R a;
  static constexpr bool kRMW = true;
  using Old = R;
  __device__ __forceinline__ R load(int64_t o) const { return out[o]; }
  __device__ __forceinline__ void put(int64_t o, const R& v, const R& old) const;
  __device__ __forceinline__ void operator()(int64_t o, const R& v) const { put(o, v, out[o]); }
};
template <> __device__ __forceinline__ void AddScalar<float>::put(int64_t o, const float& v, const float& old) const {
  out[o] = __fadd_rn(old, __fmul_rn(v, a));
}
template <> __device__ __forceinline__ void AddScalar<double>::put(int64_t o, const double& v,
                                                                   const double& old) const {
  out[o] = __dadd_rn(old, __dmul_rn(v, a));
}
struct AddC4 {
  float2* out; float ar, ai; bool conj;
  static constexpr bool kRMW = true;
  using Old = float2;
  __device__ __forceinline__ float2 load(int64_t o) const { return out[o]; }
  __device__ __forceinline__ void put(int64_t o, const float2& v, const float2& old) const {
    const float vr = v.x, vi = conj ? -v.y : v.y;
    const float tr = __fsub_rn(__fmul_rn(vr, ar), __fmul_rn(vi, ai));
    const float ti = __fadd_rn(__fmul_rn(vr, ai), __fmul_rn(vi, ar));
    float2 d = old;
    d.x = __fadd_rn(d.x, tr); d.y = __fadd_rn(d.y, ti);
    out[o] = d;
  }
  __device__ __forceinline__ void operator()(int64_t o, const float2& v) const { put(o, v, out[o]); }
};
struct AddC8 {
  double2* out; double ar, ai; bool conj;
  static constexpr bool kRMW = true;
  using Old = double2;
  __device__ __forceinline__ double2 load(int64_t o) const { return out[o]; }
  __device__ __forceinline__ void put(int64_t o, const double2& v, const double2& old) const {
    const double vr = v.x, vi = conj ? -v.y : v.y;
    const double tr = __dsub_rn(__dmul_rn(vr, ar), __dmul_rn(vi, ai));
    const double ti = __dadd_rn(__dmul_rn(vr, ai), __dmul_rn(vi, ar));
    double2 d = old;
    d.x = __dadd_rn(d.x, tr); d.y = __dadd_rn(d.y, ti);
    out[o] = d;
  }
  __device__ __forceinline__ void operator()(int64_t o, const double2& v) const { put(o, v, out[o]); }
};

double cmplx8_to_real8(double re, double im) {
  // TALSH/tensor_algebra_cpu.F90:430-445
  if (re != 0.0) return std::hypot(re, im) * (re > 0 ? 1.0 : -1.0);
  return im;
}

}  // namespace

double real_scale_factor(double re, double im) { return cmplx8_to_real8(re, im); }

// ---- measured plan choice for copies ----------------------------------------
// Which tile size runs a permutation fastest depends on the permutation and
// the element size in ways no simple rule captured (some run 10% faster with
// smaller tiles, others 25% faster with larger ones).  The first copy of a
// tensor of at least kTuneMinBytes with a given shape, permutation and
// element size therefore times the distinct plans that the planner builds for
// a few tile-size bounds, once each after an untimed run, on the caller's
// stream, and keeps the fastest for later calls (the default unless another
// is more than 2% faster).  Long row copies also try the bulk-copy kernel.
// Every plan writes the same bits, so the choice changes speed only; the
// timed runs leave the copy done.  Not while the stream is being captured
// into a graph (the default plan runs then), and TB_PERM_TUNE=0 turns it
// off.  Only copies are timed: their output may be written several times,
// unlike an accumulation's.
// {8, 16} and {4, 16} with 128-byte minimum runs: small tiles, which general
// plans (several dimensions in a load or store block) run on the list
// kernel's registers (at most 4096 elements); with 256-byte runs a 4-byte
// tile that crosses two multi-dimension blocks cannot be that small.
struct TileBounds { int vmin_kb, vmax_kb, min_run; };
constexpr TileBounds kTileCandidates[] = {{0, 0, 0}, {8, 24, 0}, {24, 48, 0}, {8, 16, 0}, {4, 16, 128}};
constexpr int kNumTileCandidates = 5;
constexpr int kListCand = 3, kListCandShort = 4;
constexpr int64_t kTuneMinBytes = (int64_t)32 << 20;
// A further candidate for long row copies: the default plan in the bulk-copy
// kernel (measured faster for 4-byte elements, slower for 8-byte ones).
constexpr int kBulkRowsCand = kNumTileCandidates;
// the TMA-staged transpose kernel (tb_perm_tma.cuh) on the default plan's
// reduced view, where its layout requirements hold
constexpr int kTmaCand = kNumTileCandidates + 1;
constexpr int kNumPlanCandidates = kNumTileCandidates + 2;

bool long_row_copy(const PermParams& P) { return P.rows2d && P.tma_ok && (int64_t)P.LA * P.es >= 4096; }

std::mutex g_tune_mu;
std::map<std::vector<int>, int> g_tune;  // (es, rank, dims, cptrn) -> candidate
constexpr size_t kMaxTuned = 4096;       // past this many shapes the choices are forgotten (bounded memory)

void remember_choice(const std::vector<int>& key, int c) {
  if (g_tune.size() >= kMaxTuned) g_tune.clear();
  g_tune[key] = c;
}

bool same_work(const PermParams& a, const PermParams& b) {
  if (a.rank != b.rank || a.V != b.V || a.LA != b.LA || a.nA != b.nA || a.LB != b.LB || a.nB != b.nB ||
      a.lap != b.lap || a.ntiles != b.ntiles || a.bulk_rows != b.bulk_rows)
    return false;
  for (int i = 0; i < a.rank; ++i)
    if (a.tile[i] != b.tile[i]) return false;
  return true;
}

template <typename E, typename Store>
int run_copy_measured(int rank, const int* dims, const int* cptrn, const E* in, const Store& st, cudaStream_t s) {
  int64_t vol = 1;
  for (int i = 0; i < rank; ++i) vol *= dims[i];
  std::vector<int> key{(int)sizeof(E), rank};
  key.insert(key.end(), dims, dims + rank);
  key.insert(key.end(), cptrn, cptrn + rank);
  int pick = -1;
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) pick = it->second;
  }
  static const bool tune_on = [] { const char* e = getenv("TB_PERM_TUNE"); return !(e && e[0] == '0'); }();
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) { cudaGetLastError(); cap = cudaStreamCaptureStatusActive; }
  // TB_PERM_TMA=1 / 0: the TMA-staged kernel wherever it applies / never
  // (tuning and test switch; results are identical)
  static const int tma_env = [] { const char* e = getenv("TB_PERM_TMA"); return e ? (e[0] == '1' ? 1 : 0) : -1; }();
  const bool tune = pick < 0 && tune_on && tma_env < 0 && vol * (int64_t)sizeof(E) >= kTuneMinBytes &&
                    cap == cudaStreamCaptureStatusNone;
  if (!tune) {
    const int c = tma_env == 1 ? kTmaCand : (pick < 0 ? 0 : pick);
    const TileBounds b = kTileCandidates[(c == kBulkRowsCand || c == kTmaCand) ? 0 : c];
    PermParams P;
    int e = build_perm_plan_o2n((int)sizeof(E), rank, dims, cptrn, &P, b.vmin_kb, b.vmax_kb, b.min_run);
    if (e == 0) {
      if (c == kTmaCand && tma_env != 0) {
        TmaPermParams T;
        if (tma_perm_plan(P, in, &T)) return launch_perm_tma<E, Store>(T, st, s);
      }
      if (c == kBulkRowsCand && long_row_copy(P)) P.bulk_rows = 1;
      return launch_perm<E, Store>(P, in, st, s);
    }
    if (e != TB_ERR_NOT_IMPLEMENTED) return e;
    return run_scatter<E, Store>(rank, dims, cptrn, in, st, s);
  }
  static PermParams plans[kNumPlanCandidates];  // large; built under the lock below
  std::lock_guard<std::mutex> g(g_tune_mu);
  int n = 0, idx[kNumPlanCandidates];
  for (int c = 0; c < kNumTileCandidates; ++c) {
    int e = build_perm_plan_o2n((int)sizeof(E), rank, dims, cptrn, &plans[n], kTileCandidates[c].vmin_kb,
                                kTileCandidates[c].vmax_kb, kTileCandidates[c].min_run);
    if (e == TB_ERR_NOT_IMPLEMENTED && c == 0) {
      remember_choice(key, 0);
      return run_scatter<E, Store>(rank, dims, cptrn, in, st, s);
    }
    if (e) { if (c == 0) return e; continue; }
    bool dup = false;
    for (int k = 0; k < n; ++k) dup = dup || same_work(plans[k], plans[n]);
    if (!dup) idx[n++] = c;
  }
  if (long_row_copy(plans[0])) {  // plans[0] is the default plan (c == 0 always builds first)
    plans[n] = plans[0];
    plans[n].bulk_rows = 1;
    idx[n++] = kBulkRowsCand;
  }
  static TmaPermParams tma;  // large (a tensor map); built under the lock
  const bool with_tma = tma_perm_plan(plans[0], in, &tma);
  if (n == 1 && !with_tma) { remember_choice(key, 0); return launch_perm<E, Store>(plans[0], in, st, s); }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) { set_error("cudaEventCreate failed"); return TB_ERR_CUDA; }
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); set_error("cudaEventCreate failed"); return TB_ERR_CUDA; }
  float best_ms = 0.f, ms0 = 0.f;
  int best = 0, err = 0;
  if (with_tma) idx[n++] = kTmaCand;
  auto run = [&](int k) {
    return idx[k] == kTmaCand ? launch_perm_tma<E, Store>(tma, st, s) : launch_perm<E, Store>(plans[k], in, st, s);
  };
  for (int k = 0; k < n && !err; ++k) {
    if ((err = run(k))) break;  // untimed: first launch of a variant
    cudaEventRecord(e0, s);
    if ((err = run(k))) break;
    cudaEventRecord(e1, s);
    float ms = 0.f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      set_error("timing a permutation plan failed");
      err = TB_ERR_CUDA;
      break;
    }
    if (k == 0) { ms0 = best_ms = ms; best = 0; }
    else if (ms < best_ms) { best_ms = ms; best = k; }
    static const bool trace = [] { const char* e = getenv("TB_PERM_TRACE"); return e && e[0] == '1'; }();
    if (trace) fprintf(stderr, "perm candidate %d: %.4f ms\n", idx[k], ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err) return err;
  if (best != 0 && best_ms > 0.98f * ms0) best = 0;
  remember_choice(key, idx[best]);
  return 0;
}

// Runs a permutation with the tiled engine, or the scatter kernel when the
// plan builder declines the layout.
// Runs a permutation with the tiled engine, or the scatter kernel when the
// plan builder declines the layout.  Used where output must be written once
// (the fused add), so nothing is timed: the plan is the one the measured
// choice keeps for copies of the same shape and element size when there is
// one, else the default plan -- or, for a general plan (several dimensions in
// a load or store block) whose default tile is too large for the list
// kernel's registers, the smaller tile of the {8, 16} KB candidate.
template <typename E, typename Store>
int run_permutation(int rank, const int* dims, const int* cptrn, const E* in, const Store& st,
                    cudaStream_t s, bool force_scatter = false) {
  if (!force_scatter) {
    std::vector<int> key{(int)sizeof(E), rank};
    key.insert(key.end(), dims, dims + rank);
    key.insert(key.end(), cptrn, cptrn + rank);
    int pick = -1;
    {
      std::lock_guard<std::mutex> g(g_tune_mu);
      auto it = g_tune.find(key);
      if (it != g_tune.end()) pick = it->second;
    }
    const TileBounds b = kTileCandidates[(pick < 0 || pick == kBulkRowsCand || pick == kTmaCand) ? 0 : pick];
    PermParams P;
    int e = build_perm_plan_o2n((int)sizeof(E), rank, dims, cptrn, &P, b.vmin_kb, b.vmax_kb, b.min_run);
    for (int c : {kListCand, kListCandShort}) {
      if (e != 0 || pick >= 0 || P.lin2d || glist_vector_bytes(P, in)) break;
      PermParams Q;
      const TileBounds q = kTileCandidates[c];
      if (build_perm_plan_o2n((int)sizeof(E), rank, dims, cptrn, &Q, q.vmin_kb, q.vmax_kb, q.min_run) == 0 &&
          glist_vector_bytes(Q, in))
        P = Q;
    }
    if (e == 0) return launch_perm<E, Store>(P, in, st, s);
    if (e != TB_ERR_NOT_IMPLEMENTED) return e;
  }
  return run_scatter<E, Store>(rank, dims, cptrn, in, st, s);
}

int tensor_copy_impl(int dtk, int rank, const int* dims, const int* cptrn, const void* in,
                     void* out, int conj_bits, cudaStream_t s, bool scatter) {
  const int es = elem_bytes(dtk);
  if (!es || !in || !out) { set_error("tb_tensor_copy: bad data kind or null pointer"); return TB_ERR_INVALID_ARGS; }
  int64_t vol;
  if (int e = check_dims(rank, dims, &vol)) { set_error("tb_tensor_copy: bad extents"); return e; }
  int ident[kMaxRank];
  if (!cptrn) { for (int i = 0; i < rank; ++i) ident[i] = i + 1; cptrn = ident; }
  bool conj = ((conj_bits & 1) ^ ((conj_bits >> 1) & 1)) && is_complex(dtk);
  if (scatter) {
    switch (es) {
      case 4: return run_scatter<uint32_t>(rank, dims, cptrn, (const uint32_t*)in, StoreCopy<uint32_t>{(uint32_t*)out}, s);
      case 8:
        if (conj) return run_scatter<uint64_t>(rank, dims, cptrn, (const uint64_t*)in, StoreConjC4{(uint64_t*)out}, s);
        return run_scatter<uint64_t>(rank, dims, cptrn, (const uint64_t*)in, StoreCopy<uint64_t>{(uint64_t*)out}, s);
      case 16:
        if (conj) return run_scatter<u128>(rank, dims, cptrn, (const u128*)in, StoreConjC8{(u128*)out}, s);
        return run_scatter<u128>(rank, dims, cptrn, (const u128*)in, StoreCopy<u128>{(u128*)out}, s);
    }
    return TB_ERR_INVALID_ARGS;
  }
  switch (es) {
    case 4: return run_copy_measured<uint32_t>(rank, dims, cptrn, (const uint32_t*)in,
                                               StoreCopy<uint32_t>{(uint32_t*)out}, s);
    case 8:
      if (conj) return run_copy_measured<uint64_t>(rank, dims, cptrn, (const uint64_t*)in,
                                                   StoreConjC4{(uint64_t*)out}, s);
      return run_copy_measured<uint64_t>(rank, dims, cptrn, (const uint64_t*)in,
                                         StoreCopy<uint64_t>{(uint64_t*)out}, s);
    case 16:
      if (conj) return run_copy_measured<u128>(rank, dims, cptrn, (const u128*)in,
                                               StoreConjC8{(u128*)out}, s);
      return run_copy_measured<u128>(rank, dims, cptrn, (const u128*)in, StoreCopy<u128>{(u128*)out}, s);
  }
  return TB_ERR_INVALID_ARGS;
}

int tensor_add_impl(int dtk, int rank, const int* ldims, const int* cptrn, void* d, const void* l,
                    double sr, double si, int conj_bits, cudaStream_t s) {
  if (!elem_bytes(dtk) || !d || !l) { set_error("tb_tensor_add: bad data kind or null pointer"); return TB_ERR_INVALID_ARGS; }
  int64_t vol;
  if (int e = check_dims(rank, ldims, &vol)) { set_error("tb_tensor_add: bad extents"); return e; }
  int ident[kMaxRank];
  if (!cptrn) { for (int i = 0; i < rank; ++i) ident[i] = i + 1; cptrn = ident; }
  bool lconj = ((conj_bits & 1) ^ ((conj_bits >> 1) & 1)) != 0;
  switch (dtk) {
    case kR4: {
      const float a = (float)cmplx8_to_real8(sr, si);
      return run_permutation<float>(rank, ldims, cptrn, (const float*)l, AddScalar<float>{(float*)d, a}, s);
    }
    case kR8: {
      const double a = cmplx8_to_real8(sr, si);
      return run_permutation<double>(rank, ldims, cptrn, (const double*)l, AddScalar<double>{(double*)d, a}, s);
    }
    case kC4:
      return run_permutation<float2>(rank, ldims, cptrn, (const float2*)l,
                                     AddC4{(float2*)d, (float)sr, (float)si, lconj}, s);
    case kC8:
      return run_permutation<double2>(rank, ldims, cptrn, (const double2*)l,
                                      AddC8{(double2*)d, sr, si, lconj}, s);
  }
  return TB_ERR_INVALID_ARGS;
}

}  // namespace tb

extern "C" int tb_tensor_copy(int data_kind, int rank, const int* in_dims, const int* cptrn,
                              const void* in, void* out, int conj_bits, void* stream) {
  return tb::tensor_copy_impl(data_kind, rank, in_dims, cptrn, in, out, conj_bits,
                              (cudaStream_t)stream, false);
}

extern "C" int tb_tensor_copy_scatter(int data_kind, int rank, const int* in_dims, const int* cptrn,
                                      const void* in, void* out, int conj_bits, void* stream) {
  return tb::tensor_copy_impl(data_kind, rank, in_dims, cptrn, in, out, conj_bits,
                              (cudaStream_t)stream, true);
}

extern "C" int tb_tensor_add(int data_kind, int rank, const int* l_dims, const int* cptrn, void* d,
                             const void* l, double scale_real, double scale_imag, int conj_bits,
                             void* stream) {
  return tb::tensor_add_impl(data_kind, rank, l_dims, cptrn, d, l, scale_real, scale_imag, conj_bits,
                             (cudaStream_t)stream);
}
