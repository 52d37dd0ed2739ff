// tb_common.cuh -- shared definitions for the B200 tensor-algebra kernels.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/talsh_b200.h"

namespace tb {

// TAL-SH data kinds (TALSH/tensor_algebra.h:67-72).
constexpr int kR4 = 4, kR8 = 8, kC4 = 14, kC8 = 18;
constexpr int kMaxRank = 56;  // MAX_TENSOR_RANK (TALSH/tensor_algebra.h:59)

inline int elem_bytes(int dtk) {
  switch (dtk) { case kR4: return 4; case kR8: return 8; case kC4: return 8; case kC8: return 16; }
  return 0;
}
inline bool is_complex(int dtk) { return dtk == kC4 || dtk == kC8; }
inline bool is_double(int dtk) { return dtk == kR8 || dtk == kC8; }

// Records the last error message (per thread) for tb_last_error().
void set_error(const char* fmt, ...);

#define TB_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      ::tb::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return TB_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

// Counts this library's kernel launches (tb_launch_count) and checks them.
void count_launch();
#define TB_CHECK_LAUNCH()                                                          \
  do {                                                                             \
    ::tb::count_launch();                                                          \
    cudaError_t e_ = cudaGetLastError();                                           \
    if (e_ != cudaSuccess) {                                                       \
      ::tb::set_error("%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return TB_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

// Optional CUDA-event timing of the dominant (GEMM) kernels, per thread:
// timed_begin records a start event on s when timing is on (returns -1 when
// off); timed_end records the matching stop event.
int timed_begin(cudaStream_t s);
void timed_end(int slot, cudaStream_t s);

// Number of SMs of the current device (cached).
int num_sms();

// The current CUDA device, 0..63 (0 when the query fails).
int current_device();

// Once-per-device flags.  Function attributes (the dynamic shared-memory
// limit) and occupancy results belong to one device's context, so each
// device sets or measures them on its first launch.  Devices are a bit mask;
// concurrent first launches may both set the attribute, which is harmless.
struct DeviceOnce {
  std::atomic<unsigned long long> bits{0};
  bool done(int dev) const { return (bits.load(std::memory_order_acquire) >> dev) & 1ull; }
  void mark(int dev) { bits.fetch_or(1ull << dev, std::memory_order_acq_rel); }
};

// Raises the dynamic shared-memory limit of `kern` to `bytes` on the current
// device the first time it is asked for that device.
template <typename K>
inline cudaError_t smem_limit_once(DeviceOnce& once, K kern, int bytes) {
  const int dev = current_device();
  if (once.done(dev)) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) once.mark(dev);
  return e;
}

// Stream-ordered scratch from the device's default memory pool.
int scratch_alloc(void** p, size_t bytes, cudaStream_t s);
void scratch_free(void* p, cudaStream_t s);

// Device-side error word: kernels record failures here instead of trapping.
// Codes: 1 = bounded wait expired, 2 = index out of range.
__device__ __forceinline__ void record_device_error(unsigned int* flag, unsigned int code) {
  if (flag) atomicCAS(flag, 0u, code);
}
unsigned int* device_error_word();  // per-device word, zero when healthy
unsigned int* device_error_word_if_created();  // the same word, or null; never allocates

}  // namespace tb

#include "tb_fastdiv.h"
