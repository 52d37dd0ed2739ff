// tb_peak.cu -- tensor-core throughput probes: the denominators of the
// contraction rooflines, measured on the GPU the library runs on.
//
//   TB_PEAK_I8    tcgen05.mma kind::i8   (M 128, N 256, K 32, INT32 in TMEM)
//   TB_PEAK_BF16  tcgen05.mma kind::f16  (M 128, N 256, K 16, BF16 in, FP32 in TMEM)
//   TB_PEAK_F64   mma.sync m8n8k4 f64    (DMMA, the plain FP64 path's instruction)
//
// The tcgen05 probes run one CTA per SM; one thread issues MMAs back to back
// on operands resident in shared memory (the SWIZZLE_128B K-major layout of
// the contraction GEMMs), into one TMEM accumulator, and waits (bounded) for
// their completion.  No global memory is read, so the result is the tensor
// pipe's issue rate at the clock the GPU runs at, which is what the GEMMs'
// achieved rates are compared with.  The DMMA probe runs independent
// accumulator chains per warp at full occupancy.  Operation counts:
// 2*M*N*K per MMA (multiply and add counted separately, TAL-SH's FLOP
// accounting).
#include "tb_common.cuh"
#include "tb_sm100.cuh"

namespace tb {
namespace {

constexpr int kPeakThreads = 128;
constexpr int kPeakN = 256;
// operand tiles (A 128 x 128 B, B 256 x 128 B) plus alignment slack; the
// request is large enough that one CTA occupies an SM
constexpr size_t kPeakSmem = 1024 + 128 * 128 + kPeakN * 128 + 64 * 1024;

template <bool I8>
__global__ void __launch_bounds__(kPeakThreads, 1) peak_tc_kernel(long long iters, unsigned int* err) {
  using namespace sm100;
  extern __shared__ __align__(1024) unsigned char pk_smem[];
  unsigned char* base = (unsigned char*)(((uintptr_t)pk_smem + 1023) & ~(uintptr_t)1023);
  unsigned char* smA = base;
  unsigned char* smB = base + 128 * 128;
  __shared__ uint64_t done_bar;
  __shared__ uint32_t tmem_base;
  // pseudo-random operands (the tensor pipe's power draw depends on the data):
  // INT8 any byte; BF16 values of magnitude in [1, 2) with random signs
  for (int i = threadIdx.x; i < (128 * 128 + kPeakN * 128) / 4; i += kPeakThreads) {
    uint32_t h = (uint32_t)i * 0x9E3779B9u + 0x7F4A7C15u;
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
    reinterpret_cast<uint32_t*>(base)[i] = I8 ? h : ((h & 0x807F807Fu) | 0x3F803F80u);
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (threadIdx.x == 0) {
    mbar_init(&done_bar, 1);
    fence_barrier_init();
  }
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    tmem_alloc(&tmem_base, kPeakN);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  if (threadIdx.x == 0) {
    constexpr uint32_t kIdesc = idesc(I8, kPeakN);
    const uint32_t sa = smem_u32(smA), sb = smem_u32(smB);
    for (long long it = 0; it < iters; ++it) {
      const int kk = (int)(it & 3);  // the four 32-byte K steps of a 128-byte swizzled row
      mma<I8>(tmem, sdesc_k128(sa + kk * 32), sdesc_k128(sb + kk * 32), kIdesc, it == 0 ? 0u : 1u);
    }
    mma_commit(&done_bar);
  }
  // the issuing thread blocks while the MMA queue is full, so once it has
  // issued everything only the queued MMAs remain: the bounded wait starts
  // after that point, not during the whole run
  __syncthreads();
  const bool ok = mbar_wait_warp(&done_bar, 0, err, 21u);
  (void)ok;
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kPeakN);
  }
}

// DMMA m8n8k4: four independent accumulator chains per warp.
__global__ void __launch_bounds__(256) peak_dmma_kernel(long long iters, double* sink) {
  double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * threadIdx.x;
  double c[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  for (long long it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                   : "+d"(c[q][0]), "+d"(c[q][1])
                   : "d"(a), "d"(b));
  }
  const double s = c[0][0] + c[0][1] + c[1][0] + c[1][1] + c[2][0] + c[2][1] + c[3][0] + c[3][1];
  if (s == 12345.678) sink[threadIdx.x] = s;  // keeps the chains alive
}

}  // namespace
}  // namespace tb

using namespace tb;

extern "C" int tb_peak_measure(int kind, long long iters, double* ops_per_s, double* ms, void* stream) {
  if (!ops_per_s || iters <= 0 || (kind != TB_PEAK_I8 && kind != TB_PEAK_BF16 && kind != TB_PEAK_F64))
    return TB_ERR_INVALID_ARGS;
  cudaStream_t s = (cudaStream_t)stream;
  const int sms = num_sms();
  double ops = 0.0;
  cudaEvent_t e0, e1;
  TB_CUDA(cudaEventCreate(&e0));
  TB_CUDA(cudaEventCreate(&e1));
  int rc = 0;
  // one untimed launch (clocks up, code loaded), then the timed one
  for (int rep = 0; rep < 2 && !rc; ++rep) {
    if (rep == 1) cudaEventRecord(e0, s);
    if (kind == TB_PEAK_F64) {
      const int blocks = sms * 8;
      peak_dmma_kernel<<<blocks, 256, 0, s>>>(iters, nullptr);
      ops = 2.0 * 8 * 8 * 4 * 4 * (double)iters * (blocks * 256 / 32);
    } else {
      static DeviceOnce attr_i8, attr_bf;
      cudaError_t e = kind == TB_PEAK_I8 ? smem_limit_once(attr_i8, peak_tc_kernel<true>, (int)kPeakSmem)
                                         : smem_limit_once(attr_bf, peak_tc_kernel<false>, (int)kPeakSmem);
      if (e != cudaSuccess) { set_error("peak probe smem attribute: %s", cudaGetErrorString(e)); rc = TB_ERR_CUDA; break; }
      if (kind == TB_PEAK_I8) peak_tc_kernel<true><<<sms, kPeakThreads, kPeakSmem, s>>>(iters, device_error_word());
      else peak_tc_kernel<false><<<sms, kPeakThreads, kPeakSmem, s>>>(iters, device_error_word());
      ops = 2.0 * 128 * kPeakN * (kind == TB_PEAK_I8 ? 32 : 16) * (double)iters * sms;
    }
    count_launch();
    if (cudaError_t e = cudaGetLastError()) { set_error("peak probe launch: %s", cudaGetErrorString(e)); rc = TB_ERR_CUDA; }
  }
  if (!rc) {
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) { cudaGetLastError(); rc = TB_ERR_CUDA; }
  }
  float t = 0.f;
  if (!rc && cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) { cudaGetLastError(); rc = TB_ERR_CUDA; }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (int d = tb_device_check(stream)) return d;
  *ops_per_s = t > 0.f ? ops / (t * 1e-3) : 0.0;
  if (ms) *ms = t;
  return 0;
}
