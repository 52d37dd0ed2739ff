// tb_contract.cu -- tensor contraction driver: D = beta*D + alpha*op(L)*op(R).
//
// Two executions of the same contraction:
//  * TB_METHOD_TTGT ("plain", the reference's scheme in
//    TALSH/tensor_algebra_gpu_nvidia.cu:5847-7188): permute L and R into
//    K-major matrices, GEMM in the tensor's own data type, then permute the
//    result into D with the alpha/beta update.  Layouts that are already
//    matrix-shaped skip their permutation.
//  * TB_METHOD_FUSED (tb_tc.cu): the operand gathers fuse the input
//    permutations with the conversion to tensor-core formats and the epilogue
//    writes D through the output permutation with alpha/beta applied.
// A full contraction into a scalar (D rank 0) uses a deterministic two-pass
// dot-product kernel (the reference's gpu_array_dot_product__, :531).
#include "tb_common.cuh"
#include "tb_contract.h"
#include "tb_gemm.h"
#include "tb_pattern.h"
#include "tb_permute.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

namespace tb {

namespace {

thread_local tb_contract_stats_t g_stats;

double real_alpha(double re, double im) {
  if (re != 0.0) return std::hypot(re, im) * (re > 0 ? 1.0 : -1.0);
  return im;
}

// Store functors for the final C -> D permutation of the TTGT path.  Those
// that read D expose load / put (kRMW), so that the permutation kernels issue
// a batch of D loads before the dependent writes.
template <typename R>
struct StoreAxpy {  // d = d + v*a
  R* out; R a;
  static constexpr bool kRMW = true;
  using Old = R;
  __device__ __forceinline__ R load(int64_t o) const { return out[o]; }
  __device__ __forceinline__ void put(int64_t o, const R& v, const R& old) const { out[o] = old + v * a; }
  __device__ __forceinline__ void operator()(int64_t o, const R& v) const { put(o, v, out[o]); }
};
template <typename R>
struct StoreScaled {  // d = v*a
  R* out; R a;
  __device__ __forceinline__ void operator()(int64_t o, const R& v) const { out[o] = v * a; }
};
template <typename C2, typename R>
struct StoreAxpyC {  // d = beta*d + alpha*v (complex)
  C2* out; R ar, ai, br, bi;
  static constexpr bool kRMW = true;
  using Old = C2;
  __device__ __forceinline__ C2 load(int64_t o) const {
    if (br != R(0) || bi != R(0)) return out[o];
    C2 z; z.x = R(0); z.y = R(0);
    return z;
  }
  __device__ __forceinline__ void put(int64_t o, const C2& v, const C2& d) const {
    C2 r;
    r.x = ar * v.x - ai * v.y;
    r.y = ar * v.y + ai * v.x;
    if (br != R(0) || bi != R(0)) {
      r.x += br * d.x - bi * d.y;
      r.y += br * d.y + bi * d.x;
    }
    out[o] = r;
  }
  __device__ __forceinline__ void operator()(int64_t o, const C2& v) const { put(o, v, load(o)); }
};

// ---- full contraction (dot product) ----------------------------------------
struct DotParams {
  int nk;
  int64_t K;
  int64_t ext[kMaxRank];
  FastDiv div[kMaxRank];
  int64_t ls[kMaxRank], rs[kMaxRank];
};
constexpr int kDotBlocks = 592, kDotThreads = 256;

template <typename E, bool CPLX>
__global__ void __launch_bounds__(kDotThreads) dot_pass1(const __grid_constant__ DotParams P, const E* __restrict__ L,
                                                         const E* __restrict__ R, int lconj, int rconj,
                                                         double2* __restrict__ partial) {
  __shared__ double2 red[kDotThreads];
  double sr = 0.0, si = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kDotThreads + threadIdx.x; i < P.K; i += (int64_t)gridDim.x * kDotThreads) {
    uint64_t r = (uint64_t)i;
    int64_t lo = 0, ro = 0;
    for (int d = 0; d < P.nk; ++d) {
      const uint64_t q = P.div[d].div(r);
      const int64_t x = (int64_t)(r - q * (uint64_t)P.ext[d]);
      r = q;
      lo += x * P.ls[d];
      ro += x * P.rs[d];
    }
    if constexpr (CPLX) {
      const double ar = (double)L[lo].x, ai = lconj ? -(double)L[lo].y : (double)L[lo].y;
      const double br = (double)R[ro].x, bi = rconj ? -(double)R[ro].y : (double)R[ro].y;
      sr += ar * br - ai * bi;
      si += ar * bi + ai * br;
    } else {
      sr += (double)L[lo] * (double)R[ro];
    }
  }
  red[threadIdx.x] = make_double2(sr, si);
  __syncthreads();
  for (int w = kDotThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      red[threadIdx.x].x += red[threadIdx.x + w].x;
      red[threadIdx.x].y += red[threadIdx.x + w].y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

template <typename E, bool CPLX>
__global__ void dot_pass2(const double2* __restrict__ partial, int n, E* __restrict__ D, double ar, double ai,
                          double br, double bi) {
  __shared__ double2 red[kDotThreads];
  double sr = 0.0, si = 0.0;
  for (int i = threadIdx.x; i < n; i += kDotThreads) { sr += partial[i].x; si += partial[i].y; }
  red[threadIdx.x] = make_double2(sr, si);
  __syncthreads();
  for (int w = kDotThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      red[threadIdx.x].x += red[threadIdx.x + w].x;
      red[threadIdx.x].y += red[threadIdx.x + w].y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double xr = red[0].x, xi = red[0].y;
    if constexpr (CPLX) {
      double orr = ar * xr - ai * xi, oi = ar * xi + ai * xr;
      if (br != 0.0 || bi != 0.0) {
        const double dr = (double)D[0].x, di = (double)D[0].y;
        orr += br * dr - bi * di;
        oi += br * di + bi * dr;
      }
      D[0].x = orr; D[0].y = oi;
    } else {
      double o = ar * xr;
      if (br != 0.0) o += br * (double)D[0];
      D[0] = (E)o;
    }
  }
}

template <typename E, bool CPLX>
int run_dot(const Matricization& Z, void* d, const void* l, const void* r, double ar, double ai, double br,
            double bi, int lconj, int rconj, cudaStream_t s) {
  DotParams P;
  std::memset(&P, 0, sizeof(P));
  P.nk = (int)Z.k.size();
  P.K = Z.K;
  for (int i = 0; i < P.nk; ++i) {
    P.ext[i] = Z.k[i].ext; P.div[i].init((uint64_t)Z.k[i].ext);
    P.ls[i] = Z.k[i].s1; P.rs[i] = Z.k[i].s2;
  }
  double2* partial = nullptr;
  if (int e = scratch_alloc((void**)&partial, kDotBlocks * sizeof(double2), s)) return e;
  dot_pass1<E, CPLX><<<kDotBlocks, kDotThreads, 0, s>>>(P, (const E*)l, (const E*)r, lconj, rconj, partial);
  dot_pass2<E, CPLX><<<1, kDotThreads, 0, s>>>(partial, kDotBlocks, (E*)d, ar, ai, br, bi);
  count_launch();
  count_launch();
  cudaError_t e = cudaGetLastError();
  scratch_free(partial, s);
  if (e != cudaSuccess) { set_error("dot kernels: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
  return 0;
}

// ---- TTGT ---------------------------------------------------------------------
// Permutes a tensor (dims/strides given per source dim) into the layout
// described by per-dim destination strides.
template <typename E, typename Store>
int permute_general(int rank, const int64_t* dims, const int64_t* sin, const int64_t* sout, const E* in,
                    const Store& st, cudaStream_t s) {
  PermParams P;
  int e = build_perm_plan((int)sizeof(E), rank, dims, sin, sout, &P);
  if (e) { set_error("permutation plan declined (code %d)", e); return e; }
  return launch_perm<E, Store>(P, in, st, s);
}

// Source-dim strides of L (or R) in its K-major matrix: contracted dims first
// in Z.k order, then the uncontracted dims in group order, row stride K.
void matrix_strides(const Matricization& Z, bool left, int rank, const int* dims, int64_t* d, int64_t* sin,
                    int64_t* sout) {
  int64_t s = 1;
  for (int i = 0; i < rank; ++i) { d[i] = dims[i]; sin[i] = s; s *= dims[i]; }
  int64_t ks = 1;
  for (auto& g : Z.k) { sout[left ? g.dpos : g.src] = ks; ks *= g.ext; }
  int64_t us = Z.K;
  for (auto& g : (left ? Z.m : Z.n)) { sout[g.src] = us; us *= g.ext; }
}

bool is_identity(int rank, const int64_t* sin, const int64_t* sout) {
  for (int i = 0; i < rank; ++i) if (sin[i] != sout[i]) return false;
  return true;
}

template <typename E>
int ttgt(const Matricization& Z, int dtk, const int* ddims, void* d, const int* ldims, const void* l,
         const int* rdims, const void* r, double ar, double ai, bool accumulate, int lconj, int rconj,
         cudaStream_t s) {
  const int es = (int)sizeof(E);
  int64_t dd[kMaxRank], si[kMaxRank], so[kMaxRank];
  void* Lt = nullptr; void* Rt = nullptr; void* Ct = nullptr;
  const void* A = l; const void* B = r;
  int err = 0;
  // L -> [M][K]
  matrix_strides(Z, true, Z.lrank, ldims, dd, si, so);
  if (!is_identity(Z.lrank, si, so)) {
    if ((err = scratch_alloc(&Lt, (size_t)Z.M * Z.K * es, s))) goto done;
    if ((err = permute_general<E>(Z.lrank, dd, si, so, (const E*)l, StoreCopy<E>{(E*)Lt}, s))) goto done;
    A = Lt;
  }
  // R -> [N][K]
  matrix_strides(Z, false, Z.rrank, rdims, dd, si, so);
  if (!is_identity(Z.rrank, si, so)) {
    if ((err = scratch_alloc(&Rt, (size_t)Z.N * Z.K * es, s))) goto done;
    if ((err = permute_general<E>(Z.rrank, dd, si, so, (const E*)r, StoreCopy<E>{(E*)Rt}, s))) goto done;
    B = Rt;
  }
  {
    // C = [M][N] with m fastest (group order): is D already in that layout?
    const int nm = (int)Z.m.size(), nn = (int)Z.n.size();
    int64_t cs = 1;
    bool dtriv = true;
    for (int i = 0; i < nm; ++i) { dd[i] = Z.m[i].ext; si[i] = cs; so[i] = Z.m[i].s2; cs *= Z.m[i].ext; }
    for (int i = 0; i < nn; ++i) { dd[nm + i] = Z.n[i].ext; si[nm + i] = cs; so[nm + i] = Z.n[i].s2; cs *= Z.n[i].ext; }
    dtriv = is_identity(nm + nn, si, so);
    const bool cplx = is_complex(dtk);
    const double realpha = cplx ? ar : real_alpha(ar, ai);
    if (dtriv) {
      const int ts = timed_begin(s);
      err = gemm_plain_tn(dtk, Z.M, Z.N, Z.K, A, Z.K, B, Z.K, d, Z.M, realpha, cplx ? ai : 0.0,
                          accumulate ? 1.0 : 0.0, 0.0, lconj, rconj, s);
      timed_end(ts, s);
      goto done;
    }
    if ((err = scratch_alloc(&Ct, (size_t)Z.M * Z.N * es, s))) goto done;
    {
      const int ts = timed_begin(s);
      err = gemm_plain_tn(dtk, Z.M, Z.N, Z.K, A, Z.K, B, Z.K, Ct, Z.M, 1.0, 0.0, 0.0, 0.0, lconj, rconj, s);
      timed_end(ts, s);
      if (err) goto done;
    }
    const int rk = nm + nn;
    switch (dtk) {
      case kR4: {
        const float a = (float)realpha;
        err = accumulate ? permute_general<float>(rk, dd, si, so, (const float*)Ct, StoreAxpy<float>{(float*)d, a}, s)
                         : permute_general<float>(rk, dd, si, so, (const float*)Ct, StoreScaled<float>{(float*)d, a}, s);
        break;
      }
      case kR8: {
        err = accumulate ? permute_general<double>(rk, dd, si, so, (const double*)Ct, StoreAxpy<double>{(double*)d, realpha}, s)
                         : permute_general<double>(rk, dd, si, so, (const double*)Ct, StoreScaled<double>{(double*)d, realpha}, s);
        break;
      }
      case kC4:
        err = permute_general<float2>(rk, dd, si, so, (const float2*)Ct,
                                      StoreAxpyC<float2, float>{(float2*)d, (float)ar, (float)ai,
                                                                accumulate ? 1.f : 0.f, 0.f}, s);
        break;
      case kC8:
        err = permute_general<double2>(rk, dd, si, so, (const double2*)Ct,
                                       StoreAxpyC<double2, double>{(double2*)d, ar, ai, accumulate ? 1.0 : 0.0, 0.0}, s);
        break;
    }
  }
done:
  scratch_free(Lt, s);
  scratch_free(Rt, s);
  scratch_free(Ct, s);
  return err;
}

}  // namespace

// Runs a non-scalar contraction with plan->method (TTGT or FUSED).  With
// fallback, a fused request outside the tensor-core path's scope runs as TTGT.
int run_method(const Matricization& Z, int dtk, const int* ddims, void* d, const int* ldims, const void* l,
               const int* rdims, const void* r, double ar, double ai, int accumulative, int lconj, int rconj,
               const tb_plan_t* plan, cudaStream_t s, bool fallback = true) {
  if (plan->method == TB_METHOD_FUSED) {
    const int e = contract_fused(Z, dtk, ddims, d, ldims, l, rdims, r, ar, ai, accumulative != 0, lconj, rconj, plan, s,
                                 &g_stats);
    if (e != TB_ERR_NOT_IMPLEMENTED) { if (!e) g_stats.method = TB_METHOD_FUSED; return e; }
    if (!fallback) return e;  // explicitly requested: no silent substitution
  }
  g_stats.method = TB_METHOD_TTGT;
  g_stats.gemm_launches = 1;
  switch (dtk) {
    case kR4: return ttgt<float>(Z, dtk, ddims, d, ldims, l, rdims, r, ar, ai, accumulative != 0, 0, 0, s);
    case kR8: return ttgt<double>(Z, dtk, ddims, d, ldims, l, rdims, r, ar, ai, accumulative != 0, 0, 0, s);
    case kC4: return ttgt<float2>(Z, dtk, ddims, d, ldims, l, rdims, r, ar, ai, accumulative != 0, lconj, rconj, s);
    case kC8: return ttgt<double2>(Z, dtk, ddims, d, ldims, l, rdims, r, ar, ai, accumulative != 0, lconj, rconj, s);
  }
  return TB_ERR_INVALID_ARGS;
}

int contract_impl(const int* cptrn, int dtk, int drank, const int* ddims, void* d, int lrank, const int* ldims,
                  const void* l, int rrank, const int* rdims, const void* r, double ar, double ai, int conj_bits,
                  int accumulative, const tb_plan_t* plan, cudaStream_t s) {
  std::memset(&g_stats, 0, sizeof(g_stats));
  if (!elem_bytes(dtk)) { set_error("tb_tensor_contract: invalid data kind %d", dtk); return TB_ERR_INVALID_ARGS; }
  if (!cptrn || !d || !l || !r) { set_error("tb_tensor_contract: null argument"); return TB_ERR_INVALID_ARGS; }
  Matricization Z;
  int e = matricize(cptrn, drank, ddims, lrank, ldims, rrank, rdims, &Z);
  if (e) { set_error("tb_tensor_contract: pattern does not match the shapes (code %d)", e); return e; }
  int lconj = 0, rconj = 0;
  if (is_complex(dtk)) {
    lconj = (conj_bits >> 1) & 1; rconj = (conj_bits >> 2) & 1;
    if (conj_bits & 1) { lconj ^= 1; rconj ^= 1; }
  }
  const bool cplx = is_complex(dtk);
  g_stats.m = Z.M; g_stats.n = Z.N; g_stats.k = Z.K;
  g_stats.flops = (cplx ? 8.0 : 2.0) * (double)Z.M * (double)Z.N * (double)Z.K;
  if (drank == 0) {
    const double br = accumulative ? 1.0 : 0.0;
    const double ra = cplx ? ar : real_alpha(ar, ai), ia = cplx ? ai : 0.0;
    g_stats.method = TB_METHOD_TTGT;
    switch (dtk) {
      case kR4: return run_dot<float, false>(Z, d, l, r, ra, ia, br, 0.0, 0, 0, s);
      case kR8: return run_dot<double, false>(Z, d, l, r, ra, ia, br, 0.0, 0, 0, s);
      case kC4: return run_dot<float2, true>(Z, d, l, r, ra, ia, br, 0.0, lconj, rconj, s);
      case kC8: return run_dot<double2, true>(Z, d, l, r, ra, ia, br, 0.0, lconj, rconj, s);
    }
  }
  int method = plan ? plan->method : TB_METHOD_AUTO;
  tb_plan_t learned;
  if (method == TB_METHOD_AUTO) {
    // learned selector when installed, else the size rule
    float f[TB_DESC_FEATURES];
    int idx = -1;
    unsigned tune = 0;
    uint64_t key = 0;
    descriptor_of(Z, dtk, f);
    auto candidate = [&](int c) {
      tb_plan_t cp = plan ? *plan : tb_plan_t{};
      cp.method = c == 0 ? TB_METHOD_TTGT : TB_METHOD_FUSED;
      cp.tile_n = c == 1 ? 128 : (c >= 2 ? 256 : 0);
      cp.tile_m = c == kCandPair ? 256 : 0;
      if (c == kCandSlices) { cp.slices = 6; cp.moduli = -1; }
      return cp;
    };
    if (selector_pick(f, &idx, &tune, &key) == 0) {
      if (tune) {
        // no timing (it waits on the host) while the stream is captured into a graph
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
          cudaGetLastError();
          tune = 0;
        }
      }
      if (tune) {
        // time each candidate in the mask with alpha = 0, beta = 1 (D unchanged):
        // one untimed run each (first-use costs), then two timed rounds that
        // visit the candidates in turn, keeping each one's faster time, so that
        // clock drift under the power cap does not favour the one timed first
        static const bool trace = [] { const char* e = getenv("TB_SELECT_TRACE"); return e && e[0] == '1'; }();
        constexpr int kRounds = 2;
        float t[kNumCandidates];
        bool ok[kNumCandidates];
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        for (int c = 0; c < kNumCandidates; ++c) {
          t[c] = 1e30f;
          ok[c] = false;
          if (!(tune & (1u << c))) continue;
          tb_plan_t cp = candidate(c);
          ok[c] = run_method(Z, dtk, ddims, d, ldims, l, rdims, r, 0.0, 0.0, 1, lconj, rconj, &cp, s) == 0;
          cudaGetLastError();
        }
        for (int round = 0; round < kRounds; ++round)
          for (int c = 0; c < kNumCandidates; ++c) {
            if (!ok[c]) continue;
            tb_plan_t cp = candidate(c);
            cudaEventRecord(e0, s);
            const int ce = run_method(Z, dtk, ddims, d, ldims, l, rdims, r, 0.0, 0.0, 1, lconj, rconj, &cp, s);
            cudaEventRecord(e1, s);
            float ms = 0.f;
            if (!ce && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
              t[c] = std::min(t[c], ms);
            else
              ok[c] = false;
            cudaGetLastError();
          }
        float best = 1e30f;
        for (int c = 0; c < kNumCandidates; ++c)
          if (ok[c] && t[c] < best) { best = t[c]; idx = c; }
        if (trace) {
          std::fprintf(stderr, "tb_select: M=%lld N=%lld K=%lld", (long long)Z.M, (long long)Z.N, (long long)Z.K);
          for (int c = 0; c < kNumCandidates; ++c)
            if (tune & (1u << c)) std::fprintf(stderr, " cand%d=%.3fms", c, ok[c] ? t[c] : -1.f);
          std::fprintf(stderr, " -> %d\n", idx);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        selector_remember(key, idx);
        std::memset(&g_stats, 0, sizeof(g_stats));
        g_stats.m = Z.M; g_stats.n = Z.N; g_stats.k = Z.K;
        g_stats.flops = (cplx ? 8.0 : 2.0) * (double)Z.M * (double)Z.N * (double)Z.K;
      }
      learned = candidate(idx);
      return run_method(Z, dtk, ddims, d, ldims, l, rdims, r, ar, ai, accumulative, lconj, rconj, &learned, s,
                        /*fallback=*/true);
    }
    method = select_method(dtk, Z, plan);
  }
  if (method == TB_METHOD_AUTO) method = TB_METHOD_TTGT;
  learned = plan ? *plan : tb_plan_t{};
  const bool requested = plan && plan->method == TB_METHOD_FUSED;
  learned.method = method;
  return run_method(Z, dtk, ddims, d, ldims, l, rdims, r, ar, ai, accumulative, lconj, rconj, &learned, s,
                    /*fallback=*/!requested);
}

}  // namespace tb

extern "C" int tb_tensor_contract(const int* cptrn, int data_kind, int drank, const int* d_dims, void* d,
                                  int lrank, const int* l_dims, const void* l, int rrank, const int* r_dims,
                                  const void* r, double alpha_real, double alpha_imag, int conj_bits,
                                  int accumulative, const tb_plan_t* plan, void* stream) {
  return tb::contract_impl(cptrn, data_kind, drank, d_dims, d, lrank, l_dims, l, rrank, r_dims, r, alpha_real,
                           alpha_imag, conj_bits, accumulative, plan, (cudaStream_t)stream);
}

extern "C" int tb_tensor_contract_str(const char* pattern, int data_kind, int drank, const int* d_dims, void* d,
                                      int lrank, const int* l_dims, const void* l, int rrank, const int* r_dims,
                                      const void* r, double alpha_real, double alpha_imag, int accumulative,
                                      const tb_plan_t* plan, void* stream) {
  tb::ParsedPattern P;
  if (int e = tb::parse_pattern(pattern, &P)) {
    tb::set_error("pattern parse error %d in \"%s\"", e, pattern ? pattern : "(null)");
    return TB_ERR_PATTERN;
  }
  if (P.rrank < 0 || P.drank != drank || P.lrank != lrank || P.rrank != rrank) {
    tb::set_error("pattern ranks (%d,%d,%d) do not match the tensors (%d,%d,%d)", P.drank, P.lrank, P.rrank, drank,
                  lrank, rrank);
    return TB_ERR_INVALID_ARGS;
  }
  if (P.hyper) { tb::set_error("hyper-contractions are not executed on the GPU path"); return TB_ERR_NOT_IMPLEMENTED; }
  return tb::contract_impl(P.cptrn, data_kind, drank, d_dims, d, lrank, l_dims, l, rrank, r_dims, r, alpha_real,
                           alpha_imag, P.conj_bits, accumulative, plan, (cudaStream_t)stream);
}

extern "C" int tb_last_contract_stats(tb_contract_stats_t* stats) {
  if (!stats) return TB_ERR_INVALID_ARGS;
  *stats = tb::g_stats;
  return 0;
}

// ---- no-allocation variant of the plain (TTGT) contraction ---------------------
// Same kernels as the TTGT path above, but every temporary buffer is carved
// from one static device array instead of the stream-ordered pool, so a call
// makes no allocation.  Nothing in the array has to start at zero: every byte
// a kernel reads there is written earlier in the same call (the GEMM does not
// read its output when beta is 0), so no clear is queued.  The array keeps the
// previous call's data; calls on one stream are ordered by the stream, calls
// that overlap on the GPU race.
static __device__ __align__(256) unsigned char tb_noalloc_arena[TB_NOALLOC_ARENA_BYTES];

namespace tb {
namespace {

unsigned char* g_arena_addr[64] = {nullptr};
std::mutex g_arena_mu;

// Device address of the array on the current device, looked up once per
// device (with that device current); the host-side name is not a device
// address and is never passed to a kernel.
int noalloc_arena(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    set_error("tb_tensor_contract_noalloc: no usable current device (%s)", cudaGetErrorString(e));
    return TB_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_arena_mu);
  if (!g_arena_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, tb_noalloc_arena);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      set_error("tb_tensor_contract_noalloc: cannot look up the scratch array on device %d (%s)", dev,
                cudaGetErrorString(e));
      return TB_ERR_CUDA;
    }
    g_arena_addr[dev] = (unsigned char*)p;
  }
  *out = g_arena_addr[dev];
  return 0;
}

uint64_t round256(unsigned __int128 b) { return (uint64_t)((b + 255) / 256 * 256); }

template <typename E, bool CPLX>
int dot_noalloc(const Matricization& Z, void* d, const void* l, const void* r, double ar, double ai, double br,
                int lconj, int rconj, unsigned char* arena, cudaStream_t s) {
  DotParams P;
  std::memset(&P, 0, sizeof(P));
  P.nk = (int)Z.k.size();
  P.K = Z.K;
  for (int i = 0; i < P.nk; ++i) {
    P.ext[i] = Z.k[i].ext; P.div[i].init((uint64_t)Z.k[i].ext);
    P.ls[i] = Z.k[i].s1; P.rs[i] = Z.k[i].s2;
  }
  double2* partial = (double2*)arena;  // every block writes its own entry
  dot_pass1<E, CPLX><<<kDotBlocks, kDotThreads, 0, s>>>(P, (const E*)l, (const E*)r, lconj, rconj, partial);
  dot_pass2<E, CPLX><<<1, kDotThreads, 0, s>>>(partial, kDotBlocks, (E*)d, ar, ai, br, 0.0);
  count_launch();
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_error("dot kernels: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
  return 0;
}

template <typename E>
int ttgt_noalloc(const Matricization& Z, int dtk, const int* ldims, const void* l, const int* rdims, const void* r,
                 void* d, double ar, double ai, bool accumulate, int lconj, int rconj, unsigned char* arena,
                 cudaStream_t s) {
  const size_t es = sizeof(E);
  int64_t dd[kMaxRank], si[kMaxRank], so[kMaxRank];
  E* Lt = (E*)arena;
  E* Rt = (E*)(arena + round256((unsigned __int128)Z.M * Z.K * es));
  E* Ct = (E*)((unsigned char*)Rt + round256((unsigned __int128)Z.N * Z.K * es));
  const void* A = l;
  const void* B = r;
  int err = 0;
  matrix_strides(Z, true, Z.lrank, ldims, dd, si, so);
  if (!is_identity(Z.lrank, si, so)) {
    if ((err = permute_general<E>(Z.lrank, dd, si, so, (const E*)l, StoreCopy<E>{Lt}, s))) return err;
    A = Lt;
  }
  matrix_strides(Z, false, Z.rrank, rdims, dd, si, so);
  if (!is_identity(Z.rrank, si, so)) {
    if ((err = permute_general<E>(Z.rrank, dd, si, so, (const E*)r, StoreCopy<E>{Rt}, s))) return err;
    B = Rt;
  }
  const int nm = (int)Z.m.size(), nn = (int)Z.n.size();
  int64_t cs = 1;
  for (int i = 0; i < nm; ++i) { dd[i] = Z.m[i].ext; si[i] = cs; so[i] = Z.m[i].s2; cs *= Z.m[i].ext; }
  for (int i = 0; i < nn; ++i) { dd[nm + i] = Z.n[i].ext; si[nm + i] = cs; so[nm + i] = Z.n[i].s2; cs *= Z.n[i].ext; }
  const bool cplx = is_complex(dtk);
  const double realpha = cplx ? ar : real_alpha(ar, ai);
  if (is_identity(nm + nn, si, so)) {  // D is already the product matrix
    return gemm_plain_tn(dtk, Z.M, Z.N, Z.K, A, Z.K, B, Z.K, d, Z.M, realpha, cplx ? ai : 0.0,
                         accumulate ? 1.0 : 0.0, 0.0, lconj, rconj, s);
  }
  if ((err = gemm_plain_tn(dtk, Z.M, Z.N, Z.K, A, Z.K, B, Z.K, Ct, Z.M, 1.0, 0.0, 0.0, 0.0, lconj, rconj, s)))
    return err;
  const int rk = nm + nn;
  switch (dtk) {
    case kR4: {
      const float a = (float)realpha;
      return accumulate ? permute_general<float>(rk, dd, si, so, (const float*)Ct, StoreAxpy<float>{(float*)d, a}, s)
                        : permute_general<float>(rk, dd, si, so, (const float*)Ct, StoreScaled<float>{(float*)d, a}, s);
    }
    case kR8:
      return accumulate
                 ? permute_general<double>(rk, dd, si, so, (const double*)Ct, StoreAxpy<double>{(double*)d, realpha}, s)
                 : permute_general<double>(rk, dd, si, so, (const double*)Ct,
                                           StoreScaled<double>{(double*)d, realpha}, s);
    case kC4:
      return permute_general<float2>(rk, dd, si, so, (const float2*)Ct,
                                     StoreAxpyC<float2, float>{(float2*)d, (float)ar, (float)ai,
                                                               accumulate ? 1.f : 0.f, 0.f}, s);
    case kC8:
      return permute_general<double2>(rk, dd, si, so, (const double2*)Ct,
                                      StoreAxpyC<double2, double>{(double2*)d, ar, ai, accumulate ? 1.0 : 0.0, 0.0},
                                      s);
  }
  return TB_ERR_INVALID_ARGS;
}

}  // namespace

int contract_noalloc_impl(const int* cptrn, int dtk, int drank, const int* ddims, void* d, int lrank,
                          const int* ldims, const void* l, int rrank, const int* rdims, const void* r, double ar,
                          double ai, int conj_bits, int accumulative, cudaStream_t s) {
  std::memset(&g_stats, 0, sizeof(g_stats));
  if (!elem_bytes(dtk)) {
    set_error("tb_tensor_contract_noalloc: invalid data kind %d", dtk);
    return TB_ERR_INVALID_ARGS;
  }
  if (!cptrn || !d || !l || !r) { set_error("tb_tensor_contract_noalloc: null argument"); return TB_ERR_INVALID_ARGS; }
  Matricization Z;
  int e = matricize(cptrn, drank, ddims, lrank, ldims, rrank, rdims, &Z);
  if (e) { set_error("tb_tensor_contract_noalloc: pattern does not match the shapes (code %d)", e); return e; }
  // Scratch bound: permuted L and R plus the product matrix (or the dot
  // partials), each rounded up to 256 bytes; checked before anything is queued.
  const unsigned __int128 es = (unsigned)elem_bytes(dtk);
  const unsigned __int128 M = (uint64_t)Z.M, N = (uint64_t)Z.N, K = (uint64_t)Z.K;
  const unsigned __int128 need = drank == 0 ? (unsigned __int128)round256(kDotBlocks * sizeof(double2))
                                            : (unsigned __int128)round256(M * K * es) + round256(N * K * es) +
                                                  round256(M * N * es);
  if (need > (unsigned __int128)TB_NOALLOC_ARENA_BYTES) {
    set_error("tb_tensor_contract_noalloc: this contraction needs %.0f bytes of scratch (permuted L and R and the "
              "product matrix), more than the %llu-byte static scratch array; use tb_tensor_contract",
              (double)need, (unsigned long long)TB_NOALLOC_ARENA_BYTES);
    return TB_ERR_LIMIT;
  }
  if (!device_error_word_if_created()) {
    set_error("tb_tensor_contract_noalloc: call tb_device_init on this device first");
    return TB_ERR_INVALID_ARGS;
  }
  unsigned char* arena = nullptr;
  if ((e = noalloc_arena(&arena))) return e;
  int lconj = 0, rconj = 0;
  if (is_complex(dtk)) {
    lconj = (conj_bits >> 1) & 1; rconj = (conj_bits >> 2) & 1;
    if (conj_bits & 1) { lconj ^= 1; rconj ^= 1; }
  }
  const bool cplx = is_complex(dtk), acc = accumulative != 0;
  g_stats.m = Z.M; g_stats.n = Z.N; g_stats.k = Z.K;
  g_stats.flops = (cplx ? 8.0 : 2.0) * (double)Z.M * (double)Z.N * (double)Z.K;
  g_stats.method = TB_METHOD_TTGT;
  if (drank == 0) {
    const double br = acc ? 1.0 : 0.0;
    const double ra = cplx ? ar : real_alpha(ar, ai), ia = cplx ? ai : 0.0;
    switch (dtk) {
      case kR4: return dot_noalloc<float, false>(Z, d, l, r, ra, ia, br, 0, 0, arena, s);
      case kR8: return dot_noalloc<double, false>(Z, d, l, r, ra, ia, br, 0, 0, arena, s);
      case kC4: return dot_noalloc<float2, true>(Z, d, l, r, ra, ia, br, lconj, rconj, arena, s);
      case kC8: return dot_noalloc<double2, true>(Z, d, l, r, ra, ia, br, lconj, rconj, arena, s);
    }
  }
  g_stats.gemm_launches = 1;
  switch (dtk) {
    case kR4: return ttgt_noalloc<float>(Z, dtk, ldims, l, rdims, r, d, ar, ai, acc, 0, 0, arena, s);
    case kR8: return ttgt_noalloc<double>(Z, dtk, ldims, l, rdims, r, d, ar, ai, acc, 0, 0, arena, s);
    case kC4: return ttgt_noalloc<float2>(Z, dtk, ldims, l, rdims, r, d, ar, ai, acc, lconj, rconj, arena, s);
    case kC8: return ttgt_noalloc<double2>(Z, dtk, ldims, l, rdims, r, d, ar, ai, acc, lconj, rconj, arena, s);
  }
  return TB_ERR_INVALID_ARGS;
}

}  // namespace tb

extern "C" int tb_tensor_contract_noalloc(const int* cptrn, int data_kind, int drank, const int* d_dims, void* d,
                                          int lrank, const int* l_dims, const void* l, int rrank,
                                          const int* r_dims, const void* r, double alpha_real, double alpha_imag,
                                          int conj_bits, int accumulative, void* stream) {
  return tb::contract_noalloc_impl(cptrn, data_kind, drank, d_dims, d, lrank, l_dims, l, rrank, r_dims, r,
                                   alpha_real, alpha_imag, conj_bits, accumulative, (cudaStream_t)stream);
}
