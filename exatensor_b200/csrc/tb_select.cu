// tb_select.cpp -- contraction descriptors and the learned plan selector.
//
// The descriptor summarises what decides the speed of a contraction plan: the
// matricized sizes M, N, K (log2), work and footprint, ranks, the smallest
// extents of the row, column and contracted groups, whether L, R and D are
// already in the TTGT matrix orders (no permutation pass needed), and the data
// type.  The selector is a 3-layer MLP (trained by tb_mlp.cu's kernels on
// autotuner timings) evaluated here on the host for each TB_METHOD_AUTO call:
// a few tens of thousands of multiply-adds, far cheaper than a GPU round trip.
#include <dlfcn.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <cstring>
#include <string>
#include <mutex>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "tb_common.cuh"
#include "tb_contract.h"
#include "tb_pattern.h"

namespace tb {
namespace {

float lg2(double v) { return (float)std::log2(v < 1.0 ? 1.0 : v); }

// True when the tensor with these dims is already laid out as the TTGT matrix
// whose fastest index groups are `first` then `second` (each in group order;
// s1 of `first` and of `second` give the tensor's strides).
bool in_matrix_order(const std::vector<MGroup>& first, const std::vector<MGroup>& second, bool first_s2,
                     bool second_s2) {
  int64_t expect = 1;
  for (auto& g : first) {
    if ((first_s2 ? g.s2 : g.s1) != expect) return false;
    expect *= g.ext;
  }
  for (auto& g : second) {
    if ((second_s2 ? g.s2 : g.s1) != expect) return false;
    expect *= g.ext;
  }
  return true;
}

struct Selector {
  std::mutex mu;
  bool on = false;
  int nh = 0;
  std::vector<float> p, mean, scale;
  float margin = 0.f;
  int autotune = 0;
  std::unordered_map<uint64_t, int> cache;
  std::unordered_set<uint64_t> seen;  // close calls met once, not yet timed
};
Selector& sel() {
  static Selector S;
  return S;
}

// Host inference of the network, layer by layer with the weight rows read in
// order (W_l is [in][out]): out += x_i * W[i][:] over the inputs, plain
// multiply-adds that the compiler vectorises.
void mlp_host(const Selector& S, const float* x, float* y) {
  constexpr int F = TB_DESC_FEATURES, O = TB_SELECT_PLANS, kMaxH = 4096;
  const int H = S.nh;
  const float* W1 = S.p.data();
  const float* b1 = W1 + (size_t)F * H;
  const float* W2 = b1 + H;
  const float* b2 = W2 + (size_t)H * H;
  const float* W3 = b2 + H;
  const float* b3 = W3 + (size_t)H * O;
  alignas(64) float h1[kMaxH], h2[kMaxH];
  float xn[F], out[O];
  for (int i = 0; i < F; ++i) xn[i] = (x[i] - S.mean[i]) / S.scale[i];
  auto layer = [](const float* in, int n_in, const float* W, const float* b, int n_out, float* o, bool relu) {
    for (int k = 0; k < n_out; ++k) o[k] = b[k];
    for (int i = 0; i < n_in; ++i) {
      const float xi = in[i];
      const float* w = W + (size_t)i * n_out;
      for (int k = 0; k < n_out; ++k) o[k] += xi * w[k];
    }
    if (relu)
      for (int k = 0; k < n_out; ++k) o[k] = o[k] > 0.f ? o[k] : 0.f;
  };
  layer(xn, F, W1, b1, H, h1, true);
  layer(h1, H, W2, b2, H, h2, true);
  layer(h2, H, W3, b3, O, out, false);
  for (int k = 0; k < O; ++k) y[k] = out[k];
}

}  // namespace

int descriptor_of(const Matricization& Z0, int dtk, float* f) {
  Matricization Z = Z0;
  const double M = (double)Z.M, N = (double)Z.N, K = (double)Z.K;
  const double es = elem_bytes(dtk);
  const bool cplx = is_complex(dtk);
  auto minext = [](const std::vector<MGroup>& g) {
    int64_t m = 0;
    for (auto& x : g) m = m == 0 ? x.ext : std::min<int64_t>(m, x.ext);
    return (double)(m ? m : 1);
  };
  // L as [M][K] with K fastest (contracted groups first), R as [N][K], D as [M][N]
  std::vector<MGroup> kl = Z.k, kr = Z.k;
  for (auto& g : kr) g.s1 = g.s2;  // R strides of the contracted groups
  f[0] = lg2(M);
  f[1] = lg2(N);
  f[2] = lg2(K);
  f[3] = lg2((cplx ? 8.0 : 2.0) * M * N * K);
  f[4] = lg2((M * K + N * K + M * N) * es);
  f[5] = (float)Z.drank;
  f[6] = (float)Z.lrank;
  f[7] = (float)Z.rrank;
  f[8] = (float)Z.k.size();
  f[9] = lg2(minext(Z.k));
  f[10] = lg2(minext(Z.m));
  f[11] = lg2(minext(Z.n));
  f[12] = in_matrix_order(kl, Z.m, false, false) ? 1.f : 0.f;
  f[13] = in_matrix_order(kr, Z.n, false, false) ? 1.f : 0.f;
  f[14] = in_matrix_order(Z.m, Z.n, true, true) ? 1.f : 0.f;
  f[15] = is_double(dtk) ? 1.f : 0.f;
  return 0;
}

// Shapes remembered by the measured fallback (seen once, or decided); past
// this many the sets are cleared, so memory stays bounded in long runs.
constexpr size_t kMaxRemembered = (size_t)1 << 16;

// Plans the descriptor allows: INT8 slices (plan kCandSlices) are FP64-only.
bool plan_applies(const float* f, int i) { return i != kCandSlices || f[15] != 0.f; }

int best_plan(const float* f, const float* y) {
  int best = 0;
  for (int i = 1; i < TB_SELECT_PLANS; ++i)
    if (plan_applies(f, i) && y[i] < y[best]) best = i;
  return best;
}

int selector_pick(const float* f, int* idx, unsigned* tune_mask, uint64_t* key) {
  Selector& S = sel();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.on) return -1;
  float y[TB_SELECT_PLANS];
  mlp_host(S, f, y);
  const int best = best_plan(f, y);
  *idx = best;
  // key: the descriptor quantised to 1/64 (log2 units)
  uint64_t h = 1469598103934665603ull;
  for (int i = 0; i < TB_DESC_FEATURES; ++i) {
    h ^= (uint64_t)(int64_t)std::lround(f[i] * 64.f);
    h *= 1099511628211ull;
  }
  *key = h;
  // Timing candidates costs a few contractions: only worth it for large ones,
  // and only for the plans predicted within the margin of the best -- or, for
  // very large ones (beyond the corpus's 4 GiB footprints the network
  // extrapolates, and a wrong pick costs most), for every plan.
  constexpr float kTuneMinLog2Flops = 34.0f;     // about 1.7e10 FLOP
  constexpr float kTuneAllMinLog2Flops = 38.0f;  // about 2.7e11 FLOP
  unsigned mask = 0;
  if (S.autotune && f[3] >= kTuneMinLog2Flops)
    for (int i = 0; i < TB_SELECT_PLANS; ++i)
      if (plan_applies(f, i) && (y[i] - y[best] < S.margin || f[3] >= kTuneAllMinLog2Flops)) mask |= 1u << i;
  if (mask == (1u << best)) mask = 0;  // nothing close: the prediction stands
  if (mask) {
    auto it = S.cache.find(h);
    if (it != S.cache.end()) {
      *idx = it->second;
      mask = 0;
    } else {
      if (S.seen.size() >= kMaxRemembered) S.seen.clear();
      if (S.seen.insert(h).second) {
        // first time this shape is seen: take the prediction; time the
        // candidates only if the same shape comes back (one-off shapes never pay)
        mask = 0;
      }
    }
  }
  *tune_mask = mask;
  return 0;
}

void selector_remember(uint64_t key, int idx) {
  Selector& S = sel();
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.cache.size() >= kMaxRemembered) S.cache.clear();  // bounded memory: decisions are re-measured
  S.cache[key] = idx;
}

}  // namespace tb

using namespace tb;

extern "C" int tb_contract_descriptor(const int* cptrn, int data_kind, int drank, const int* d_dims, int lrank,
                                      const int* l_dims, int rrank, const int* r_dims, float* features) {
  if (!cptrn || !features || !elem_bytes(data_kind)) { set_error("tb_contract_descriptor: bad arguments"); return TB_ERR_INVALID_ARGS; }
  Matricization Z;
  if (int e = matricize(cptrn, drank, d_dims, lrank, l_dims, rrank, r_dims, &Z)) {
    set_error("tb_contract_descriptor: pattern does not match the shapes (code %d)", e);
    return e;
  }
  return descriptor_of(Z, data_kind, features);
}

extern "C" int tb_selector_install(int n_hidden, const float* params, const float* mean, const float* scale,
                                   float margin, int autotune) {
  Selector& S = sel();
  std::lock_guard<std::mutex> lk(S.mu);
  S.cache.clear();
  S.seen.clear();
  if (!params) { S.on = false; return 0; }
  if (n_hidden < 1 || n_hidden > 4096 || !mean || !scale) {
    set_error("tb_selector_install: bad arguments (hidden units 1..4096)");
    return TB_ERR_INVALID_ARGS;
  }
  const int F = TB_DESC_FEATURES, O = TB_SELECT_PLANS;
  const size_t n = (size_t)F * n_hidden + n_hidden + (size_t)n_hidden * n_hidden + n_hidden + (size_t)n_hidden * O + O;
  S.p.assign(params, params + n);
  S.mean.assign(mean, mean + F);
  S.scale.assign(scale, scale + F);
  for (auto& v : S.scale)
    if (!(v > 0.f)) v = 1.f;
  S.nh = n_hidden;
  S.margin = margin;
  S.autotune = autotune;
  S.on = true;
  return 0;
}

extern "C" int tb_selector_choose(const float* features, float* predicted) {
  Selector& S = sel();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.on || !features) return -1;
  float y[TB_SELECT_PLANS];
  mlp_host(S, features, y);
  if (predicted) std::memcpy(predicted, y, sizeof(y));
  return best_plan(features, y);
}

extern "C" int tb_selector_time(const float* features, int iters, double* us_per_call) {
  if (!features || iters < 1 || !us_per_call) return TB_ERR_INVALID_ARGS;
  Selector& S = sel();
  if (!S.on) return -1;
  volatile int sink = 0;
  const auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < iters; ++i) {
    std::lock_guard<std::mutex> lk(S.mu);
    float y[TB_SELECT_PLANS];
    mlp_host(S, features, y);
    sink = sink + best_plan(features, y);
  }
  const auto t1 = std::chrono::steady_clock::now();
  *us_per_call = std::chrono::duration<double, std::micro>(t1 - t0).count() / iters;
  return 0;
}

// Weights file: "TBSEL001", int32 features, hidden, outputs, float32 margin,
// int32 autotune, float32 mean[features], scale[features], then the network's
// parameters (W1 b1 W2 b2 W3 b3).
extern "C" int tb_selector_load(const char* path) {
  if (!path) return TB_ERR_INVALID_ARGS;
  FILE* f = std::fopen(path, "rb");
  if (!f) { set_error("tb_selector_load: cannot open %s", path); return TB_ERR_INVALID_ARGS; }
  char magic[8];
  int32_t nf = 0, nh = 0, no = 0, at = 0;
  float margin = 0.f;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "TBSEL001", 8) == 0 &&
            std::fread(&nf, 4, 1, f) == 1 && std::fread(&nh, 4, 1, f) == 1 && std::fread(&no, 4, 1, f) == 1 &&
            std::fread(&margin, 4, 1, f) == 1 && std::fread(&at, 4, 1, f) == 1 && nf == TB_DESC_FEATURES &&
            no == TB_SELECT_PLANS && nh > 0 && nh <= 4096;
  std::vector<float> mean(nf > 0 ? nf : 0), scale(nf > 0 ? nf : 0), p;
  if (ok) {
    const size_t n = (size_t)nf * nh + nh + (size_t)nh * nh + nh + (size_t)nh * no + no;
    p.resize(n);
    ok = std::fread(mean.data(), 4, nf, f) == (size_t)nf && std::fread(scale.data(), 4, nf, f) == (size_t)nf &&
         std::fread(p.data(), 4, n, f) == n;
  }
  std::fclose(f);
  if (!ok) { set_error("tb_selector_load: %s is not a selector weights file", path); return TB_ERR_INVALID_ARGS; }
  return tb_selector_install(nh, p.data(), mean.data(), scale.data(), margin, at);
}

namespace tb {
// Installs the weights shipped next to the library (selector_weights.bin)
// unless a selector is already installed; TB_SELECTOR=0 disables this and
// TB_SELECTOR=<path> names another file.  Called by tb_device_init.
void selector_autoload() {
  static std::once_flag once;
  std::call_once(once, [] {
    const char* env = std::getenv("TB_SELECTOR");
    if (env && std::strcmp(env, "0") == 0) return;
    {
      Selector& S = sel();
      std::lock_guard<std::mutex> lk(S.mu);
      if (S.on) return;
    }
    std::string path;
    if (env && *env) {
      path = env;
    } else {
      Dl_info info;
      if (!dladdr((void*)&tb_selector_load, &info) || !info.dli_fname) return;
      path = info.dli_fname;
      const size_t slash = path.rfind('/');
      path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/selector_weights.bin";
    }
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return;
    std::fclose(f);
    if (tb_selector_load(path.c_str())) set_error("");  // a bad file leaves the size rule in place
  });
}
}  // namespace tb
