// tb_fastdiv.h -- host/device fast division by runtime constants.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define TB_HD __host__ __device__ __forceinline__
#else
#define TB_HD inline
#endif

namespace tb {

// Unsigned 64-bit division by a runtime constant (Granlund-Montgomery,
// "round-up" variant: m = floor(2^64 (2^l - d) / d) + 1, l = ceil(log2 d)).
struct FastDiv {
  uint64_t d = 1;
  uint64_t m = 0;  // 0 means d is a power of two
  int s = 0;
  FastDiv() = default;
  explicit FastDiv(uint64_t div) { init(div); }
  void init(uint64_t div) {
    d = div ? div : 1;
    s = 0;
    while ((1ull << s) < d) ++s;
    if ((d & (d - 1)) == 0) { m = 0; return; }
    unsigned __int128 num = ((unsigned __int128)1 << (64 + s));
    m = (uint64_t)(num / d - ((unsigned __int128)1 << 64) + 1);
  }
  TB_HD uint64_t div(uint64_t n) const {
    if (m == 0) return n >> s;
#ifdef __CUDA_ARCH__
    uint64_t t = __umul64hi(n, m);
#else
    uint64_t t = (uint64_t)(((unsigned __int128)n * m) >> 64);
#endif
    return (t + ((n - t) >> 1)) >> (s - 1);
  }
};

// 32-bit magic division for 0 <= n < 2^31: q = (n * magic) >> shift.
inline void magic32(uint32_t d, uint32_t* magic, int* shift) {
  if (d == 0) d = 1;
  int sh = 0;
  while ((1ull << sh) < d) ++sh;
  const uint64_t num = 1ull << (31 + sh);
  *magic = (uint32_t)((num + d - 1) / d);
  *shift = 31 + sh;
}
TB_HD uint32_t fdiv32(uint32_t n, uint32_t magic, int shift) {
  return (uint32_t)(((uint64_t)n * magic) >> shift);
}

}  // namespace tb
