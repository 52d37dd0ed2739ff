// tb_runtime.cu -- device selection, error reporting, scratch memory, and the
// elementwise kernels (init, scale, norms, seeded fill).
#include "tb_common.cuh"
#include "tb_contract.h"

#include <cmath>
#include <cstdarg>
#include <atomic>
#include <mutex>
#include <vector>

namespace tb {

namespace {
thread_local char g_err[512] = "";
int g_sms[64] = {0};
unsigned int* g_err_word[64] = {nullptr};
std::mutex g_mu;
}  // namespace

int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) { cudaGetLastError(); return 0; }
  return d < 0 || d >= 64 ? 0 : d;
}

thread_local bool g_timing = false;
thread_local std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_timed;

int timed_begin(cudaStream_t s) {
  if (!g_timing) return -1;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s);
  g_timed.push_back({a, b});
  return (int)g_timed.size() - 1;
}

void timed_end(int slot, cudaStream_t s) {
  if (slot >= 0 && slot < (int)g_timed.size()) cudaEventRecord(g_timed[slot].second, s);
}

std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int num_sms() {
  const int d = current_device();
  if (!g_sms[d]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
    g_sms[d] = n > 0 ? n : 148;
  }
  return g_sms[d];
}

unsigned int* device_error_word() {
  const int d = current_device();
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_err_word[d]) {
    void* p = nullptr;
    if (cudaMalloc(&p, 256) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, 256);
    g_err_word[d] = (unsigned int*)p;
  }
  return g_err_word[d];
}

unsigned int* device_error_word_if_created() {
  const int d = current_device();
  std::lock_guard<std::mutex> lk(g_mu);
  return g_err_word[d];
}

int scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  if (bytes == 0) return 0;
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("scratch allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return TB_ERR_NO_MEMORY;
  }
  return 0;
}

void scratch_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

// ---------------------------------------------------------------------------
// Elementwise kernels.  Scale and init reproduce tensor_block_scale /
// tensor_block_init (TALSH/tensor_algebra_cpu.F90:1821, :955): one rounding
// per product, complex products by the textbook formula.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void fill_kernel(T* __restrict__ d, T v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = v;
}

__global__ void scale_r4(float* __restrict__ d, float a, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = __fmul_rn(d[i], a);
}
__global__ void scale_r8(double* __restrict__ d, double a, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = __dmul_rn(d[i], a);
}
__global__ void scale_c4(float2* __restrict__ d, float ar, float ai, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float2 v = d[i];
    d[i] = make_float2(__fsub_rn(__fmul_rn(v.x, ar), __fmul_rn(v.y, ai)),
                       __fadd_rn(__fmul_rn(v.x, ai), __fmul_rn(v.y, ar)));
  }
}
__global__ void scale_c8(double2* __restrict__ d, double ar, double ai, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double2 v = d[i];
    d[i] = make_double2(__dsub_rn(__dmul_rn(v.x, ar), __dmul_rn(v.y, ai)),
                        __dadd_rn(__dmul_rn(v.x, ai), __dmul_rn(v.y, ar)));
  }
}

// Deterministic norms: pass 1 writes one FP64 partial per block (fixed
// grid, fixed per-thread order, fixed tree), pass 2 sums the partials in
// index order.  The result does not depend on timing.
constexpr int kNormBlocks = 1024, kNormThreads = 256;

template <int DTK>
__device__ __forceinline__ double norm_term(const void* d, int64_t i, int which) {
  double re, im = 0.0;
  if (DTK == kR4) re = ((const float*)d)[i];
  else if (DTK == kR8) re = ((const double*)d)[i];
  else if (DTK == kC4) { float2 v = ((const float2*)d)[i]; re = v.x; im = v.y; }
  else { double2 v = ((const double2*)d)[i]; re = v.x; im = v.y; }
  if (which == 1) return (DTK == kR4 || DTK == kR8) ? fabs(re) : hypot(re, im);
  return re * re + im * im;
}

template <int DTK>
__global__ void __launch_bounds__(kNormThreads) norm_pass1(const void* __restrict__ d, int64_t n, int which,
                                                           double* __restrict__ partial) {
  __shared__ double red[kNormThreads];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kNormThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kNormThreads)
    s += norm_term<DTK>(d, i, which);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kNormThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void norm_pass2(const double* __restrict__ partial, int n, double* __restrict__ out) {
  __shared__ double red[kNormThreads];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += kNormThreads) s += partial[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kNormThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// splitmix64 stream: element i takes draw i (complex: draws 2i, 2i+1).
__device__ __forceinline__ double splitmix_u01(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

template <typename T, bool CPLX>
__global__ void fill_uniform_kernel(T* __restrict__ d, int64_t n, uint64_t seed, double lo, double hi) {
  const int64_t nn = CPLX ? 2 * n : n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (T)(lo + (hi - lo) * splitmix_u01(seed, (uint64_t)i));
}

int grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  int64_t cap = (int64_t)num_sms() * 8;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

double cmplx_to_real(double re, double im) {
  if (re != 0.0) return std::hypot(re, im) * (re > 0 ? 1.0 : -1.0);
  return im;
}

}  // namespace tb

using namespace tb;

extern "C" const char* tb_last_error(void) { return tb::g_err; }

extern "C" long long tb_launch_count(void) { return tb::g_launches.load(); }

extern "C" int tb_timing_enable(int on) {
  tb::g_timing = on != 0;
  return 0;
}

extern "C" int tb_timing_read(double* total_ms, int* count) {
  double t = 0.0;
  for (auto& pr : tb::g_timed) {
    cudaEventSynchronize(pr.second);
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) t += ms;
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  cudaGetLastError();
  if (count) *count = (int)tb::g_timed.size();
  if (total_ms) *total_ms = t;
  tb::g_timed.clear();
  return 0;
}

extern "C" int tb_data_kind_size(int data_kind) { return elem_bytes(data_kind); }

extern "C" int tb_device_init(int gpu) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    set_error("no CUDA device available");
    return TB_ERR_CUDA;
  }
  if (gpu < 0 || gpu >= n) { set_error("GPU %d out of range (%d present)", gpu, n); return TB_ERR_INVALID_ARGS; }
  TB_CUDA(cudaSetDevice(gpu));
  cudaDeviceProp prop;
  TB_CUDA(cudaGetDeviceProperties(&prop, gpu));
  if (prop.major != 10) {
    set_error("device %d is sm_%d%d; this library is built for sm_100a only", gpu, prop.major, prop.minor);
    return TB_ERR_NOT_IMPLEMENTED;
  }
  // The learned plan selector shipped next to the library (if any).
  selector_autoload();
  // Keep freed scratch in the pool between calls.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, gpu) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  if (!device_error_word()) { set_error("cannot allocate the device error word"); return TB_ERR_CUDA; }
  num_sms();
  return 0;
}

extern "C" int tb_device_check(void* stream) {
  unsigned int* w = device_error_word();
  if (!w) return TB_ERR_CUDA;
  unsigned int h = 0;
  TB_CUDA(cudaMemcpyAsync(&h, w, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  TB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  if (h) {
    TB_CUDA(cudaMemsetAsync(w, 0, sizeof(unsigned int), (cudaStream_t)stream));
    set_error("device-side error code %u recorded by a kernel", h);
    return TB_ERR_DEVICE;
  }
  return 0;
}

extern "C" int tb_tensor_init(int data_kind, size_t volume, void* d, double vr, double vi, void* stream) {
  if (!elem_bytes(data_kind) || (!d && volume)) { set_error("tb_tensor_init: bad arguments"); return TB_ERR_INVALID_ARGS; }
  if (!volume) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  const int g = grid_for((int64_t)volume);
  switch (data_kind) {
    case kR4: fill_kernel<float><<<g, 256, 0, s>>>((float*)d, (float)vr, volume); break;
    case kR8: fill_kernel<double><<<g, 256, 0, s>>>((double*)d, vr, volume); break;
    case kC4: fill_kernel<float2><<<g, 256, 0, s>>>((float2*)d, make_float2((float)vr, (float)vi), volume); break;
    case kC8: fill_kernel<double2><<<g, 256, 0, s>>>((double2*)d, make_double2(vr, vi), volume); break;
  }
  TB_CHECK_LAUNCH();
  return 0;
}

extern "C" int tb_tensor_scale(int data_kind, size_t volume, void* d, double sr, double si, void* stream) {
  if (!elem_bytes(data_kind) || (!d && volume)) { set_error("tb_tensor_scale: bad arguments"); return TB_ERR_INVALID_ARGS; }
  if (!volume) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  const int g = grid_for((int64_t)volume);
  switch (data_kind) {
    case kR4: scale_r4<<<g, 256, 0, s>>>((float*)d, (float)cmplx_to_real(sr, si), volume); break;
    case kR8: scale_r8<<<g, 256, 0, s>>>((double*)d, cmplx_to_real(sr, si), volume); break;
    case kC4: scale_c4<<<g, 256, 0, s>>>((float2*)d, (float)sr, (float)si, volume); break;
    case kC8: scale_c8<<<g, 256, 0, s>>>((double2*)d, sr, si, volume); break;
  }
  TB_CHECK_LAUNCH();
  return 0;
}

extern "C" int tb_tensor_norm(int data_kind, size_t volume, const void* d, int which, double* result,
                              void* stream) {
  if (!elem_bytes(data_kind) || !result || (which != 1 && which != 2) || (!d && volume)) {
    set_error("tb_tensor_norm: bad arguments");
    return TB_ERR_INVALID_ARGS;
  }
  cudaStream_t s = (cudaStream_t)stream;
  double* scratch = nullptr;
  if (int e = scratch_alloc((void**)&scratch, (kNormBlocks + 1) * sizeof(double), s)) return e;
  const int64_t n = (int64_t)volume;
  switch (data_kind) {
    case kR4: norm_pass1<kR4><<<kNormBlocks, kNormThreads, 0, s>>>(d, n, which, scratch); break;
    case kR8: norm_pass1<kR8><<<kNormBlocks, kNormThreads, 0, s>>>(d, n, which, scratch); break;
    case kC4: norm_pass1<kC4><<<kNormBlocks, kNormThreads, 0, s>>>(d, n, which, scratch); break;
    case kC8: norm_pass1<kC8><<<kNormBlocks, kNormThreads, 0, s>>>(d, n, which, scratch); break;
  }
  norm_pass2<<<1, kNormThreads, 0, s>>>(scratch, kNormBlocks, scratch + kNormBlocks);
  count_launch();
  count_launch();
  cudaError_t le = cudaGetLastError();
  double h = 0.0;
  cudaError_t ce = cudaMemcpyAsync(&h, scratch + kNormBlocks, sizeof(double), cudaMemcpyDeviceToHost, s);
  scratch_free(scratch, s);
  cudaError_t se = cudaStreamSynchronize(s);
  if (le != cudaSuccess || ce != cudaSuccess || se != cudaSuccess) {
    set_error("tb_tensor_norm: %s", cudaGetErrorString(le != cudaSuccess ? le : ce != cudaSuccess ? ce : se));
    return TB_ERR_CUDA;
  }
  *result = h;
  return 0;
}

extern "C" int tb_fill_uniform(int data_kind, size_t volume, void* d, uint64_t seed, double lo, double hi,
                               void* stream) {
  if (!elem_bytes(data_kind) || (!d && volume)) { set_error("tb_fill_uniform: bad arguments"); return TB_ERR_INVALID_ARGS; }
  if (!volume) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = (int64_t)volume;
  const int g = grid_for(is_complex(data_kind) ? 2 * n : n);
  switch (data_kind) {
    case kR4: fill_uniform_kernel<float, false><<<g, 256, 0, s>>>((float*)d, n, seed, lo, hi); break;
    case kR8: fill_uniform_kernel<double, false><<<g, 256, 0, s>>>((double*)d, n, seed, lo, hi); break;
    case kC4: fill_uniform_kernel<float, true><<<g, 256, 0, s>>>((float*)d, n, seed, lo, hi); break;
    case kC8: fill_uniform_kernel<double, true><<<g, 256, 0, s>>>((double*)d, n, seed, lo, hi); break;
  }
  TB_CHECK_LAUNCH();
  return 0;
}
