// tb_tc_prep.cuh -- operand preparation for the tensor-core contractions:
// TMA tensor maps over operand planes, offset tables, row exponent maxima, and
// the gathers that convert operands (read through offset tables, so that the
// input permutation is fused) into INT8 slice planes or BF16 parts.  Each
// kernel exists in a dense form (one operand per launch) and a grouped form
// (a table of operand jobs per launch, for block-sparse contractions).
#pragma once
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>
#include <type_traits>
#include <vector>

#include "tb_common.cuh"
#include "tb_pattern.h"
#include "tb_tc_gemm.cuh"

namespace tb {
namespace {

// ---- TMA tensor maps (driver entry point, no libcuda link) --------------------
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// 3-D map over planes of [rows][kpad] K-major operands, 128-byte rows per box.
int make_operand_map(CUtensorMap* map, const void* base, bool i8, int64_t kpad, int64_t rows, int planes,
                     int box_rows) {
  auto enc = get_encode();
  if (!enc) { set_error("cuTensorMapEncodeTiled is unavailable"); return TB_ERR_CUDA; }
  const int es = i8 ? 1 : 2;
  cuuint64_t dims[3] = {(cuuint64_t)kpad, (cuuint64_t)rows, (cuuint64_t)planes};
  cuuint64_t strides[2] = {(cuuint64_t)(kpad * es), (cuuint64_t)(kpad * es * rows)};
  cuuint32_t box[3] = {(cuuint32_t)(128 / es), (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, i8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed (%d)", (int)r); return TB_ERR_CUDA; }
  return 0;
}

// ---- offset tables: out[i] = sum_g digit_g(i) * stride_g (first group fastest) --
struct OffsetParams {
  int ng;
  int64_t count;
  int64_t ext[kMaxRank];
  FastDiv div[kMaxRank];
  int64_t stride[kMaxRank];
};

__global__ void offsets_kernel(const __grid_constant__ OffsetParams P, int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P.count; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t r = (uint64_t)i;
    int64_t o = 0;
    for (int g = 0; g < P.ng; ++g) {
      const uint64_t q = P.div[g].div(r);
      o += (int64_t)(r - q * (uint64_t)P.ext[g]) * P.stride[g];
      r = q;
    }
    out[i] = o;
  }
}

int build_offsets(const std::vector<MGroup>& groups, bool use_s2, int64_t* out, cudaStream_t s) {
  OffsetParams P;
  std::memset(&P, 0, sizeof(P));
  P.ng = (int)groups.size();
  P.count = 1;
  for (int g = 0; g < P.ng; ++g) {
    P.ext[g] = groups[g].ext;
    P.div[g].init((uint64_t)groups[g].ext);
    P.stride[g] = use_s2 ? groups[g].s2 : groups[g].s1;
    P.count *= groups[g].ext;
  }
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((P.count + 255) / 256, num_sms() * 8));
  offsets_kernel<<<(unsigned)blocks, 256, 0, s>>>(P, out);
  TB_CHECK_LAUNCH();
  return 0;
}

// ---- operand conversion helpers --------------------------------------------------
__device__ __forceinline__ unsigned exp_field(double x) {
  return (unsigned)((__double_as_longlong(x) >> 52) & 0x7FF);
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// ---- operand gather: 64 x 64 tiles through source offset tables ----------------
// Element (m, k) of a matricized operand lives at src[lm[m] + lk[k]].  A tile
// is read with lanes along whichever index is contiguous in the source, staged
// in shared memory, and converted with lanes along k so that every thread
// writes 4 consecutive K positions of each output plane in one store.
// Tiles cover [0, rows_pad) x [0, kpad_src): padding is written as zeros.
constexpr int kGThreads = 256;
constexpr int kMaxSlicesDev = 7;
template <typename E> constexpr int gather_rows() { return sizeof(E) == 16 ? 32 : 64; }  // 32-34 KB tiles
constexpr int kGK = 64;

enum GatherMode { G_SLICE_R8, G_SLICE_C8A, G_SLICE_C8B, G_SPLIT_R4, G_SPLIT_C4A, G_SPLIT_C4B,
                  G_RESID_R8, G_RESID_C8A, G_RESID_C8B };

// Ozaki scheme II operands: each scaled value x in (-1/2, 1/2) becomes the
// integer X = floor(x 2^(p+1)) (|X| <= 2^p, exact in FP64), stored as its
// residues modulo the pairwise coprime moduli m_i <= 256 in the symmetric
// range (signed 8 bits), one plane per modulus.  The moduli are the first n
// entries of one fixed table, so the gathers see them as compile-time
// constants.
constexpr int kMaxModuli = 15;
TB_HD constexpr int residue_modulus(int i) {
  return i == 0 ? 256 : i == 1 ? 255 : i == 2 ? 253 : i == 3 ? 251 : i == 4 ? 247 : i == 5 ? 241 : i == 6 ? 239
       : i == 7 ? 233 : i == 8 ? 229 : i == 9 ? 227 : i == 10 ? 223 : i == 11 ? 211 : i == 12 ? 199 : i == 13 ? 197
       : 193;
}
// 2^e mod m
TB_HD constexpr int pow2_mod(int e, int m) {
  int r = 1 % m;
  for (int i = 0; i < e; ++i) r = (2 * r) % m;
  return r;
}
// c_ij = 2^(16 j) mod m_i in the symmetric range [-(m-1)/2, m/2]
TB_HD constexpr int residue_cdig(int i, int j) {
  const int m = residue_modulus(i), c = pow2_mod(16 * j, m);
  return c > (m - 1) / 2 ? c - m : c;
}

struct ResidueSpec {
  int n;                    // moduli: residue_modulus(0 .. n-1)
  int p;                    // operand bits: |X| <= 2^p
  double pscale;            // 2^(p+1)
  int ndig;                 // balanced 16-bit digits of X: 3 (p <= 46) or 4
};

struct GatherParams {
  const void* src;
  const int64_t* lm;   // source offset of row m (m < rows)
  const int64_t* lk;   // source offset of contracted index k (k < K)
  int64_t rows, K;     // valid extents
  int64_t kpad;        // real row length of the output planes (elements)
  int64_t pstride;     // elements per plane
  void* planes;
  unsigned* rowE;      // per row: largest exponent field (slice modes read it; the
                       // split modes set it to 2047 for rows with a NaN or an infinity)
  int slices;
  int lanes_on_k;      // 1: consecutive k are contiguous in the source
  double isign;        // -1 conjugates the imaginary part
  ResidueSpec rs;      // residue modes: the moduli
};

// Residues of integers |X| <= 2^p (p <= 63) held exactly as doubles.  X is
// split once into balanced 16-bit digits D_j (|D_j| <= 2^15; three digits
// when p <= 47), so that for every modulus the residue is
//   raw = sum_j D_j c_j   (c_j = 2^(16 j) mod m in the symmetric range, c_0 = 1),
// exact in FP32 (|raw| <= 4 * 2^15 * 128 = 2^24), then r = raw - m rint(raw / m)
// in [-m/2, m/2] -- exact, the quotient rounded by the 1.5 * 2^23 trick (right
// since raw / m is never within 1/(2m) of a half integer for odd m, and the
// product's error is far below that).  The low byte of r, read off the bit
// pattern of r + 1.5 * 2^23, is r in signed 8 bits (for m = 256, r = 128 gives
// -128, the same residue).  For m = 256 the residue is D_0's low byte.
struct Digits16 { float d[4]; };

// NDIG = 3: the top digit is x2 itself (|x2| <= 2^15 + 1 for p <= 47);
// NDIG = 4: x2 is split once more (|x3| <= 2^(p-48) + 1).
template <int NDIG>
__device__ __forceinline__ Digits16 digits16(double X) {
  Digits16 g;
  const double x1 = rint(X * (1.0 / 65536.0));
  g.d[0] = (float)fma(-x1, 65536.0, X);
  const double x2 = rint(x1 * (1.0 / 65536.0));
  g.d[1] = (float)fma(-x2, 65536.0, x1);
  if constexpr (NDIG > 3) {
    const double x3 = rint(x2 * (1.0 / 65536.0));
    g.d[2] = (float)fma(-x3, 65536.0, x2);
    g.d[3] = (float)x3;
  } else {
    g.d[2] = (float)x2;
    g.d[3] = 0.f;
  }
  return g;
}

// Three balanced 16-bit digits of X = rint(v), |v| <= 2^46, without
// conversions: Y = v + (1.5 * 2^52 + B), B = 2^15 (1 + 2^16 + 2^32), rounds v
// to the nearest integer (one rounding: Y lies in [2^52, 2^53)) and leaves
// X + B in Y's low 48 mantissa bits.  Its 16-bit fields u_j (0 <= u_j < 2^16)
// give X = sum_j (u_j - 2^15) 2^(16 j); a field placed under the bit pattern
// of 1.5 * 2^23 (one byte permute) is the float 1.5 * 2^23 + u_j, and one
// subtraction gives d_j = u_j - 2^15 exactly.
__device__ __forceinline__ Digits16 digits16_rint(double v) {
  constexpr double kMB = 6896139076927488.0;  // 1.5 * 2^52 + 2^15 + 2^31 + 2^47
  constexpr float kBias = 12582912.0f + 32768.0f;
  const double Y = v + kMB;
  const uint32_t lo = (uint32_t)__double2loint(Y), hi = (uint32_t)__double2hiint(Y);
  Digits16 g;
  g.d[0] = __uint_as_float(__byte_perm(lo, 0x4B400000u, 0x7610)) - kBias;
  g.d[1] = __uint_as_float(__byte_perm(lo, 0x4B400000u, 0x7632)) - kBias;
  g.d[2] = __uint_as_float(__byte_perm(hi, 0x4B400000u, 0x7610)) - kBias;
  g.d[3] = 0.f;
  return g;
}

// Digits of one operand value x of a row with scale exponent se: X = rint(x
// 2^(se + p + 1)) for NDIG = 3 (sc = 2^(se + p + 1) when that is a double,
// else 0), floor of the same for NDIG = 4.  Both are integers with |X| <= 2^p.
template <int NDIG>
__device__ __forceinline__ Digits16 operand_digits(double x, int se, double sc, double pscale) {
  if constexpr (NDIG == 3) {
    return digits16_rint(sc != 0.0 ? x * sc : scale2(x, se) * pscale);
  } else {
    return digits16<NDIG>(floor(scale2(x, se) * pscale));
  }
}

// r + 1.5 * 2^23 for modulus I of two values at once (packed FP32 pairs,
// each component rounded as fmaf / __fadd_rn): the low byte of each
// component's bit pattern is its residue
template <int NDIG, int I>
__device__ __forceinline__ float2 residue_shifted2(const float2 (&d)[4]) {
  constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
  constexpr int m = residue_modulus(I);
  const float2 magic = make_float2(kMagic, kMagic);
  if constexpr (m == 256) {
    return __fadd2_rn(d[0], magic);
  } else {
    constexpr float negm = -(float)m, inv = 1.0f / (float)m;
    constexpr float c1 = (float)residue_cdig(I, 1), c2 = (float)residue_cdig(I, 2), c3 = (float)residue_cdig(I, 3);
    float2 raw = __ffma2_rn(d[1], make_float2(c1, c1), d[0]);
    raw = __ffma2_rn(d[2], make_float2(c2, c2), raw);
    if constexpr (NDIG > 3) raw = __ffma2_rn(d[3], make_float2(c3, c3), raw);
    const float2 q = __fadd2_rn(__ffma2_rn(raw, make_float2(inv, inv), magic), make_float2(-kMagic, -kMagic));
    return __fadd2_rn(__ffma2_rn(q, make_float2(negm, negm), raw), magic);
  }
}

// low bytes of four words, packed little-endian
__device__ __forceinline__ uint32_t pack_low_bytes(float a, float b, float c, float d) {
  const uint32_t lo = __byte_perm(__float_as_uint(a), __float_as_uint(b), 0x0040);
  const uint32_t hi = __byte_perm(__float_as_uint(c), __float_as_uint(d), 0x0040);
  return __byte_perm(lo, hi, 0x5410);
}

// Residue I of four values, packed little-endian.
template <int NDIG, int I>
__device__ __forceinline__ uint32_t residue4(const Digits16 (&g)[4]) {
  float2 a[4], b[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    a[j] = make_float2(g[0].d[j], g[1].d[j]);
    b[j] = make_float2(g[2].d[j], g[3].d[j]);
  }
  const float2 ra = residue_shifted2<NDIG, I>(a), rb = residue_shifted2<NDIG, I>(b);
  return pack_low_bytes(ra.x, ra.y, rb.x, rb.y);
}

// f(integral_constant<int, I>) for I = I0 .. min(n, N) - 1 (n uniform)
template <int I, int N, class F>
__device__ __forceinline__ void for_moduli(int n, F&& f) {
  if constexpr (I < N) {
    if (I < n) {
      f(std::integral_constant<int, I>{});
      for_moduli<I + 1, N>(n, f);
    }
  }
}

// Slices of x in (-1/2, 1/2): balanced signed base-256 digits of the fixed-point
// value X = floor(x * 2^55) = sum_i d_i 2^(48-8i), d_i in [-128, 127] for
// i >= 1 and |d_0| <= 64.  With Y = X + 0x808080808080 the low bytes of Y are
// d_i + 128 and Y >> 48 = d_0, so each slice is one byte of Y (bit 7 flipped
// for i >= 1).  Digit i has weight 2^-(8i+7); the digits are centred on zero,
// so the parts dropped by keeping s slices or slice pairs do not accumulate a
// bias over K.  The scaling by 2^55 is exact and the conversion rounds toward
// minus infinity.
__device__ __forceinline__ long long fixed55(double x) {
  return __double2ll_rd(x * 36028797018963968.0) + 0x808080808080ll;  // 2^55; Y
}
// Slice i of four consecutive values, packed little-endian into one word.
__device__ __forceinline__ uint32_t slice4(long long y0, long long y1, long long y2, long long y3, int i) {
  const int sh = 48 - 8 * i;
  const uint32_t flip = i == 0 ? 0u : 0x80808080u;
  return ((uint32_t)((y0 >> sh) & 255) | ((uint32_t)((y1 >> sh) & 255) << 8) |
          ((uint32_t)((y2 >> sh) & 255) << 16) | ((uint32_t)((y3 >> sh) & 255) << 24)) ^
         flip;
}

// Operand element type of a gather mode.
template <int MODE>
struct GatherElem {
  static constexpr bool CPLX = MODE == G_SLICE_C8A || MODE == G_SLICE_C8B || MODE == G_SPLIT_C4A ||
                               MODE == G_SPLIT_C4B || MODE == G_RESID_C8A || MODE == G_RESID_C8B;
  static constexpr bool F32 = MODE == G_SPLIT_R4 || MODE == G_SPLIT_C4A || MODE == G_SPLIT_C4B;
  using R = typename std::conditional<F32, float, double>::type;
  using E = typename std::conditional<CPLX, typename std::conditional<F32, float2, double2>::type, R>::type;
};
// Dynamic shared memory of a gather CTA: two tile buffers, a ring of three
// tiles' K offsets, the row offsets and the row scale exponents.
// K tile of a gather mode (64 for all: 32-wide tiles with four CTAs per SM
// ran the real residue gather 1.7x slower)
template <int MODE>
constexpr int gather_tk() { return kGK; }
template <int MODE>
constexpr int gather_smem_bytes() {
  using E = typename GatherElem<MODE>::E;
  return 2 * gather_rows<E>() * (gather_tk<MODE>() + 1) * (int)sizeof(E) + 3 * gather_tk<MODE>() * 8 +
         gather_rows<E>() * 20;
}

// Asynchronous copy of one element into shared memory; zero-filled when
// !valid (src is then any valid address and is not read).
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* sdst, const void* gsrc, bool valid) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
  const int n = valid ? BYTES : 0;
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(gsrc), "n"(BYTES), "r"(n) : "memory");
}

template <int MODE, int NDIG = 3>
__device__ __forceinline__ void gather_body(const GatherParams& P, int64_t rowtile, int ky, int kstep) {
  constexpr bool CPLX = GatherElem<MODE>::CPLX;
  constexpr bool F32 = GatherElem<MODE>::F32;
  using R = typename GatherElem<MODE>::R;
  using E = typename GatherElem<MODE>::E;
  (void)sizeof(R);
  constexpr int TM = gather_rows<E>(), TK = gather_tk<MODE>();
  // Tiles move global -> shared with cp.async, double-buffered: tile i+1 is in
  // flight while tile i converts, without passing through registers.  Its
  // source addresses need the K offsets of tile i+1, which sit in shared
  // memory: they were read from global memory (into a register, by one thread
  // per k) during tile i-1's conversion and stored at its end.
  extern __shared__ __align__(16) unsigned char gather_smem[];
  E* tbuf = reinterpret_cast<E*>(gather_smem);                                        // [2][TM][TK+1]
  int64_t* lkbuf = reinterpret_cast<int64_t*>(gather_smem + 2 * TM * (TK + 1) * sizeof(E));  // [3][TK]
  int64_t* sm_lm = lkbuf + 3 * TK;                                                     // [TM]
  double* sm_sc = reinterpret_cast<double*>(sm_lm + TM);  // residue modes: 2^(se + p + 1), or 0
  int* sm_se = reinterpret_cast<int*>(sm_sc + TM);  // slice and residue modes: the row's scale exponent
  auto tile_at = [&](int b) { return reinterpret_cast<E (*)[TK + 1]>(tbuf + (size_t)b * TM * (TK + 1)); };
  // Within a row, k sits at column (k % 4) * TK/4 + k / 4: the conversion's
  // lanes read k = 4j + t for the TK/4 lanes j of a row, which then fall on
  // consecutive columns (no bank conflicts within a row) instead of every
  // fourth one.
  auto col = [](int k) { return (k & 3) * (TK / 4) + (k >> 2); };
  const int64_t m0 = rowtile * TM;
  const int tid = threadIdx.x;
  const E* src = (const E*)P.src;
  const int64_t ntiles = (P.kpad / (CPLX ? 2 : 1)) / TK;  // conversion also writes the padding
  if (ky >= ntiles) return;  // uniform: no tile for this CTA
  if (tid < TM) {
    sm_lm[tid] = (m0 + tid < P.rows) ? P.lm[m0 + tid] : -1;
    if constexpr (!F32) {
      const int se = 1021 - (int)(m0 + tid < P.rows ? P.rowE[m0 + tid] : 1021u);
      sm_se[tid] = se;
      sm_sc[tid] = se + P.rs.p + 1 <= 1023 ? pow2d(se + P.rs.p + 1) : 0.0;
    }
  }
  if (tid < TK) {
    for (int j = 0; j < 2; ++j) {
      const int64_t k = ((int64_t)ky + (int64_t)j * kstep) * TK + tid;
      lkbuf[j * TK + tid] = k < P.K ? P.lk[k] : 0;
    }
  }
  constexpr int IT = TM * TK / kGThreads;
  auto issue_tile = [&](int64_t k0, int b, const int64_t* lkt) {
    E (*t)[TK + 1] = tile_at(b);
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int idx = tid + it * kGThreads;
      const int mm = P.lanes_on_k ? idx / TK : idx % TM;
      const int kk = P.lanes_on_k ? idx % TK : idx / TM;
      const bool valid = sm_lm[mm] >= 0 && k0 + kk < P.K;
      cp_async_elem<(int)sizeof(E)>(&t[mm][col(kk)], valid ? src + sm_lm[mm] + lkt[kk] : src, valid);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  __syncthreads();  // sm_lm and the first two tiles' K offsets ready
  issue_tile((int64_t)ky * TK, 0, lkbuf);
  int i = 0;
  for (int64_t kt = ky; kt < ntiles; kt += kstep, ++i) {
    const int64_t k0 = kt * TK;
    __syncthreads();  // buffer (i+1) & 1 consumed; K offsets of tile i+1 visible
    if (kt + kstep < ntiles)
      issue_tile((kt + kstep) * TK, (i + 1) & 1, lkbuf + ((i + 1) % 3) * TK);
    else
      asm volatile("cp.async.commit_group;\n" ::: "memory");  // empty group: keeps the count
    int64_t lk2 = 0;  // K offset of tile i+2 (one per thread < TK), stored after the conversion
    {
      const int64_t k = (kt + 2 * (int64_t)kstep) * TK + tid;
      if (tid < TK && kt + 2 * (int64_t)kstep < ntiles && k < P.K) lk2 = P.lk[k];
    }
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this thread's copies of tile i
    __syncthreads();                                          // everyone's
    E (*tile)[TK + 1] = tile_at(i & 1);
    {
      // convert: thread -> (row mm, 4 consecutive k)
      for (int idx = tid; idx < TM * (TK / 4); idx += kGThreads) {
        const int mm = idx / (TK / 4), kq = (idx % (TK / 4)) * 4;
        const int64_t m = m0 + mm, k = k0 + kq;
        if constexpr (MODE == G_RESID_R8) {
          const int se = sm_se[mm];
          const double sc = sm_sc[mm];
          Digits16 g[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) g[t] = operand_digits<NDIG>(tile[mm][col(kq + t)], se, sc, P.rs.pscale);
          int8_t* base = (int8_t*)P.planes + m * P.kpad + k;
          for_moduli<0, kMaxModuli>(P.rs.n, [&](auto ic) {
            constexpr int I = decltype(ic)::value;
            *reinterpret_cast<uint32_t*>(base + I * P.pstride) = residue4<NDIG, I>(g);
          });
        } else if constexpr (MODE == G_RESID_C8A) {
          // A' row m: (re, im) interleaved along K
          const int se = sm_se[mm];
          const double sc = sm_sc[mm];
          Digits16 ga[4], gb[4];
#pragma unroll
          for (int t = 0; t < 2; ++t) {
            const E v0 = tile[mm][col(kq + t)], v1 = tile[mm][col(kq + 2 + t)];
            ga[2 * t] = operand_digits<NDIG>(v0.x, se, sc, P.rs.pscale);
            ga[2 * t + 1] = operand_digits<NDIG>(P.isign * v0.y, se, sc, P.rs.pscale);
            gb[2 * t] = operand_digits<NDIG>(v1.x, se, sc, P.rs.pscale);
            gb[2 * t + 1] = operand_digits<NDIG>(P.isign * v1.y, se, sc, P.rs.pscale);
          }
          int8_t* base = (int8_t*)P.planes + m * P.kpad + 2 * k;
          for_moduli<0, kMaxModuli>(P.rs.n, [&](auto ic) {
            constexpr int I = decltype(ic)::value;
            *reinterpret_cast<uint2*>(base + I * P.pstride) = make_uint2(residue4<NDIG, I>(ga), residue4<NDIG, I>(gb));
          });
        } else if constexpr (MODE == G_RESID_C8B) {
          // B' rows 2n = (re, -im), 2n+1 = (im, re) interleaved along K
          const int se = sm_se[mm];
          const double sc = sm_sc[mm];
          Digits16 R[4], I[4], NI[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const E v = tile[mm][col(kq + t)];
            R[t] = operand_digits<NDIG>(v.x, se, sc, P.rs.pscale);
            I[t] = operand_digits<NDIG>(P.isign * v.y, se, sc, P.rs.pscale);
            NI[t] = operand_digits<NDIG>(-P.isign * v.y, se, sc, P.rs.pscale);
          }
          const Digits16 r0a[4] = {R[0], NI[0], R[1], NI[1]}, r0b[4] = {R[2], NI[2], R[3], NI[3]};
          const Digits16 r1a[4] = {I[0], R[0], I[1], R[1]}, r1b[4] = {I[2], R[2], I[3], R[3]};
          int8_t* b0 = (int8_t*)P.planes + (2 * m) * P.kpad + 2 * k;
          int8_t* b1 = b0 + P.kpad;
          for_moduli<0, kMaxModuli>(P.rs.n, [&](auto ic) {
            constexpr int J = decltype(ic)::value;
            *reinterpret_cast<uint2*>(b0 + J * P.pstride) =
                make_uint2(residue4<NDIG, J>(r0a), residue4<NDIG, J>(r0b));
            *reinterpret_cast<uint2*>(b1 + J * P.pstride) =
                make_uint2(residue4<NDIG, J>(r1a), residue4<NDIG, J>(r1b));
          });
        } else if constexpr (MODE == G_SLICE_R8) {
          const int se = sm_se[mm];
          long long X[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) X[t] = fixed55(scale2(tile[mm][col(kq + t)], se));
          int8_t* base = (int8_t*)P.planes + m * P.kpad + k;
#pragma unroll
          for (int i = 0; i < kMaxSlicesDev; ++i)
            if (i < P.slices) *reinterpret_cast<uint32_t*>(base + i * P.pstride) = slice4(X[0], X[1], X[2], X[3], i);
        } else if constexpr (MODE == G_SLICE_C8A) {
          // A' row m: (re, im) interleaved along K
          const int se = sm_se[mm];
          long long R[4], I[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const E v = tile[mm][col(kq + t)];
            R[t] = fixed55(scale2(v.x, se));
            I[t] = fixed55(scale2(P.isign * v.y, se));
          }
          int8_t* base = (int8_t*)P.planes + m * P.kpad + 2 * k;
#pragma unroll
          for (int i = 0; i < kMaxSlicesDev; ++i)
            if (i < P.slices) {
              uint2 w = make_uint2(slice4(R[0], I[0], R[1], I[1], i), slice4(R[2], I[2], R[3], I[3], i));
              *reinterpret_cast<uint2*>(base + i * P.pstride) = w;
            }
        } else if constexpr (MODE == G_SLICE_C8B) {
          // B' rows 2n = (re, -im), 2n+1 = (im, re) interleaved along K
          const int se = sm_se[mm];
          long long R[4], I[4], NI[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const E v = tile[mm][col(kq + t)];
            const double im = scale2(P.isign * v.y, se);
            R[t] = fixed55(scale2(v.x, se));
            I[t] = fixed55(im);
            NI[t] = fixed55(-im);
          }
          int8_t* b0 = (int8_t*)P.planes + (2 * m) * P.kpad + 2 * k;
          int8_t* b1 = b0 + P.kpad;
#pragma unroll
          for (int i = 0; i < kMaxSlicesDev; ++i)
            if (i < P.slices) {
              *reinterpret_cast<uint2*>(b0 + i * P.pstride) =
                  make_uint2(slice4(R[0], NI[0], R[1], NI[1], i), slice4(R[2], NI[2], R[3], NI[3], i));
              *reinterpret_cast<uint2*>(b1 + i * P.pstride) =
                  make_uint2(slice4(I[0], R[0], I[1], R[1], i), slice4(I[2], R[2], I[3], R[3], i));
            }
        } else if constexpr (MODE == G_SPLIT_R4) {
          __nv_bfloat16 h[4], l[4];
          bool nf = false;
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            split_bf16(tile[mm][col(kq + t)], h[t], l[t]);
            nf |= !isfinite(tile[mm][col(kq + t)]);
          }
          if (nf && P.rowE && m < P.rows) atomicMax(&P.rowE[m], 2047u);  // row left to the non-finite fix-up
          __nv_bfloat16* base = (__nv_bfloat16*)P.planes + m * P.kpad + k;
          __nv_bfloat162 hh[2] = {{h[0], h[1]}, {h[2], h[3]}}, ll[2] = {{l[0], l[1]}, {l[2], l[3]}};
          *reinterpret_cast<uint2*>(base) = *reinterpret_cast<uint2*>(hh);
          *reinterpret_cast<uint2*>(base + P.pstride) = *reinterpret_cast<uint2*>(ll);
        } else {
          // complex FP32: A' rows (re, im); B' rows 2n (re, -im), 2n+1 (im, re)
          __nv_bfloat16 hr[4], lr[4], hi[4], li[4], nhi[4], nli[4];
          bool nf = false;
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const E v = tile[mm][col(kq + t)];
            const float im = (float)P.isign * v.y;
            split_bf16(v.x, hr[t], lr[t]);
            split_bf16(im, hi[t], li[t]);
            split_bf16(-im, nhi[t], nli[t]);
            nf |= !isfinite(v.x) || !isfinite(v.y);
          }
          if (nf && P.rowE && m < P.rows) atomicMax(&P.rowE[m], 2047u);  // row left to the non-finite fix-up
          if constexpr (MODE == G_SPLIT_C4A) {
            __nv_bfloat16* base = (__nv_bfloat16*)P.planes + m * P.kpad + 2 * k;
            __nv_bfloat162 H[4] = {{hr[0], hi[0]}, {hr[1], hi[1]}, {hr[2], hi[2]}, {hr[3], hi[3]}};
            __nv_bfloat162 L[4] = {{lr[0], li[0]}, {lr[1], li[1]}, {lr[2], li[2]}, {lr[3], li[3]}};
            *reinterpret_cast<uint4*>(base) = *reinterpret_cast<uint4*>(H);
            *reinterpret_cast<uint4*>(base + P.pstride) = *reinterpret_cast<uint4*>(L);
          } else {
            __nv_bfloat16* b0 = (__nv_bfloat16*)P.planes + (2 * m) * P.kpad + 2 * k;
            __nv_bfloat16* b1 = b0 + P.kpad;
            __nv_bfloat162 H0[4] = {{hr[0], nhi[0]}, {hr[1], nhi[1]}, {hr[2], nhi[2]}, {hr[3], nhi[3]}};
            __nv_bfloat162 L0[4] = {{lr[0], nli[0]}, {lr[1], nli[1]}, {lr[2], nli[2]}, {lr[3], nli[3]}};
            __nv_bfloat162 H1[4] = {{hi[0], hr[0]}, {hi[1], hr[1]}, {hi[2], hr[2]}, {hi[3], hr[3]}};
            __nv_bfloat162 L1[4] = {{li[0], lr[0]}, {li[1], lr[1]}, {li[2], lr[2]}, {li[3], lr[3]}};
            *reinterpret_cast<uint4*>(b0) = *reinterpret_cast<uint4*>(H0);
            *reinterpret_cast<uint4*>(b0 + P.pstride) = *reinterpret_cast<uint4*>(L0);
            *reinterpret_cast<uint4*>(b1) = *reinterpret_cast<uint4*>(H1);
            *reinterpret_cast<uint4*>(b1 + P.pstride) = *reinterpret_cast<uint4*>(L1);
          }
        }
      }
    }
    if (tid < TK) lkbuf[((i + 2) % 3) * TK + tid] = lk2;
  }
}

// (the complex B' residue mode holds three digit sets per value: two CTAs per
// SM leave it registers enough not to spill)
template <int MODE, int NDIG = 3>
__global__ void __launch_bounds__(kGThreads, MODE == G_RESID_C8B ? 2 : 3)
    gather_kernel(const __grid_constant__ GatherParams P) {
  gather_body<MODE, NDIG>(P, blockIdx.x, blockIdx.y, gridDim.y);
}

// Grouped form: CTA x works on row tile map[x].y of job map[x].x.
template <int MODE>
__global__ void __launch_bounds__(kGThreads, 3) gather_grouped_kernel(const GatherParams* __restrict__ jobs,
                                                                   const int2* __restrict__ map) {
  const int2 jm = map[blockIdx.x];
  const GatherParams P = jobs[jm.x];
  gather_body<MODE>(P, jm.y, blockIdx.y, gridDim.y);
}

// Sets the grouped gather's dynamic shared-memory limit on the current device
// (once per device; call it before any stream capture).
template <int MODE>
cudaError_t gather_grouped_prepare() {
  static DeviceOnce once;
  return smem_limit_once(once, gather_grouped_kernel<MODE>, gather_smem_bytes<MODE>());
}

// exponents: rowexp[r] = rowE[r / rep] - 1021 (rep = 2 for complex B' rows).
// With a list, the source rows flagged 2047 (a NaN or an infinity) are also
// appended to it (in no particular order; *count counts them).
__global__ void exps_kernel(const unsigned* __restrict__ rowE, int* __restrict__ out, int64_t n, int rep,
                            int* __restrict__ list = nullptr, int* __restrict__ count = nullptr) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned e = rowE[i / rep];
    out[i] = (int)e - 1021;
    if (list && e >= 2047u && i % rep == 0) list[atomicAdd(count, 1)] = (int)(i / rep);
  }
}

// ---- non-finite fix-up -----------------------------------------------------------
// D entries whose row of A or column of B holds a NaN or an infinity are left
// untouched by the GEMM epilogue (nf_skip) and computed here as plain dot
// products in FP64 (FP32 data too, rounded once at the end), so that
// non-finite values propagate the way an IEEE GEMM propagates them: a NaN
// term, an infinity times zero, or infinities of both signs give NaN; other
// infinities give an infinity of their sign.  Work: one warp per entry, the
// entries of the flagged rows (all columns) and then of the flagged columns
// (the rows that are not flagged).  With nothing flagged every CTA returns at
// once.
struct NfParams {
  const void* srcA;
  const void* srcB;
  const int64_t *lmA, *lkA, *lmB, *lkB;  // operand offsets (rows, contracted index)
  const int64_t *dm, *dn;                 // D offsets of rows of A and columns of B
  void* D;
  int64_t M, N, K;                        // rows of A, columns of B (complex: pairs), contracted extent
  const unsigned* rowE;                   // 2047: the row holds a non-finite value
  const int* badrows;                     // flagged rows of A, count nbad[0]
  const int* badcols;                     // flagged columns of B, count nbad[1]
  const int* nbad;
  double isignA, isignB;                  // -1: conjugate the operand
  double ar, ai, br, bi;                  // alpha, beta (beta 0: D is not read)
};

template <typename R, bool CPLX>
__global__ void __launch_bounds__(256) nonfinite_fixup_kernel(const __grid_constant__ NfParams P) {
  const int nbr = P.nbad[0], nbc = P.nbad[1];
  if (nbr == 0 && nbc == 0) return;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t total = (int64_t)nbr * P.N + (int64_t)nbc * P.M;
  for (int64_t e = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); e < total; e += warps) {
    int64_t m, n;
    if (e < (int64_t)nbr * P.N) {
      m = P.badrows[e / P.N];
      n = e % P.N;
    } else {
      const int64_t f = e - (int64_t)nbr * P.N;
      n = P.badcols[f / P.M];
      m = f % P.M;
      if (P.rowE[m] >= 2047u) continue;  // done with the flagged rows
    }
    const int64_t a0 = P.lmA[m], b0 = P.lmB[n];
    double sr = 0.0, si = 0.0;
    if constexpr (!CPLX) {
      const R* A = (const R*)P.srcA;
      const R* B = (const R*)P.srcB;
      for (int64_t k = lane; k < P.K; k += 32) sr += (double)A[a0 + P.lkA[k]] * (double)B[b0 + P.lkB[k]];
    } else {
      using C2 = typename std::conditional<sizeof(R) == 8, double2, float2>::type;
      const C2* A = (const C2*)P.srcA;
      const C2* B = (const C2*)P.srcB;
      for (int64_t k = lane; k < P.K; k += 32) {
        const C2 x = A[a0 + P.lkA[k]], y = B[b0 + P.lkB[k]];
        const double xr = x.x, xi = P.isignA * (double)x.y, yr = y.x, yi = P.isignB * (double)y.y;
        sr += xr * yr - xi * yi;
        si += xr * yi + xi * yr;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      if (CPLX) si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane != 0) continue;
    const int64_t off = P.dm[m] + P.dn[n];
    if constexpr (!CPLX) {
      R* D = (R*)P.D;
      const double v = P.ar * sr;
      D[off] = (R)(P.br == 0.0 ? v : P.br * (double)D[off] + v);
    } else {
      using C2 = typename std::conditional<sizeof(R) == 8, double2, float2>::type;
      C2* D = (C2*)P.D;
      double vr = P.ar * sr - P.ai * si, vi = P.ar * si + P.ai * sr;
      if (P.br != 0.0 || P.bi != 0.0) {
        const C2 d = D[off];
        vr += P.br * (double)d.x - P.bi * (double)d.y;
        vi += P.br * (double)d.y + P.bi * (double)d.x;
      }
      C2 w;
      w.x = (R)vr;
      w.y = (R)vi;
      D[off] = w;
    }
  }
}


// ---- Ozaki scheme II reconstruction (Chinese remainder theorem) ------------------
// With M = prod m_i, M_i = M / m_i and y_i = M_i^-1 mod m_i, the exact integer
// dot product is C = sum_i t_i M_i mod M, t_i = (r_i y_i) mod m_i, taken in the
// symmetric range (|C| < M / 2 by the choice of p).  Each t_i M_i < M, so the
// sum stays below n M < 2^123 in 128 bits.  C is converted to FP64 (about one
// rounding), scaled by 2^(e_m + f_n - 2(p+1)) exactly, and D = beta D +
// alpha C through the offset tables.  Rows and columns flagged as holding a
// NaN or an infinity are left to the fix-up kernel.  Persistent CTAs take
// whole columns, threads along the rows (D's fastest).
struct CrtParams {
  const uint8_t* res;          // residue planes [i][column][row], bytes
  int64_t res_ld, res_plane;
  int n;
  int mod[kMaxModuli], y[kMaxModuli];
  uint64_t mi_lo[kMaxModuli], mi_hi[kMaxModuli];
  uint64_t M_lo, M_hi;
  double Md;                   // M as a double
  int64_t rows, cols;          // rows of A; columns of B (complex: column pairs)
  const int64_t* dm;
  const int64_t* dn;
  void* D;
  const int* rowexp;
  const int* colexp;
  int shift;                   // 2 (p + 1)
  double ar, ai, br, bi;
};

__device__ __forceinline__ double u128_to_double(unsigned __int128 x) {
  return (double)(uint64_t)(x >> 64) * 18446744073709551616.0 + (double)(uint64_t)x;
}

// The table of crt_kernel: entry i * 256 + r = ((r y_i) mod m_i) M_i (r < m_i),
// built by each CTA in shared memory, so that a residue costs one lookup and a
// 128-bit addition.
constexpr int kCrtTableBytes = kMaxModuli * 256 * 16;
struct alignas(16) CrtEntry { uint64_t lo, hi; };

// Residues of the four D entries (col, m .. m + 3) from the n planes: one
// 32-bit load per plane (m a multiple of 4; the planes' row length and plane
// stride are multiples of 4 bytes, so the words are aligned and lie inside the
// padded plane even past the last row), byte t of word i holding residue i of
// row m + t.
__device__ __forceinline__ void crt_load4(const CrtParams& P, int64_t col, int64_t m, uint32_t (&w)[kMaxModuli]) {
  const uint8_t* rp = P.res + col * P.res_ld + m;
#pragma unroll
  for (int i = 0; i < kMaxModuli; ++i) w[i] = i < P.n ? *reinterpret_cast<const uint32_t*>(rp + i * P.res_plane) : 0u;
}
__device__ __forceinline__ void crt_byte(const uint32_t (&w)[kMaxModuli], int t, uint32_t (&r)[kMaxModuli]) {
#pragma unroll
  for (int i = 0; i < kMaxModuli; ++i) r[i] = __byte_perm(w[i], 0u, 0x4440 + t);
}

// The exact integer from its residues, in FP64 (about one rounding).
__device__ __forceinline__ double crt_combine(const CrtParams& P, const CrtEntry* tab, const uint32_t (&r)[kMaxModuli]) {
  uint64_t lo = 0, hi = 0;
#pragma unroll
  for (int i = 0; i < kMaxModuli; ++i) {
    if (i >= P.n) break;
    const CrtEntry t = tab[i * 256 + r[i]];
    lo += t.lo;
    hi += t.hi + (lo < t.lo ? 1u : 0u);
  }
  unsigned __int128 S = ((unsigned __int128)hi << 64) | lo;
  const unsigned __int128 M = ((unsigned __int128)P.M_hi << 64) | P.M_lo;
  // S < n M: subtract q M, q = floor(S / M) estimated in FP64 (within one), then
  // at most a few exact corrections
  uint64_t q = (uint64_t)(u128_to_double(S) / P.Md);
  if (q > 0) --q;
  S -= (unsigned __int128)q * M;
  for (int it = 0; it < 4 && S >= M; ++it) S -= M;
  const bool neg = S > (M >> 1);
  const double v = u128_to_double(neg ? M - S : S);
  return neg ? -v : v;
}

// Each CTA takes residue columns (one real D column, or one complex one: its
// two residue columns) and each thread, for every four consecutive rows it
// owns, loads one word per plane -- the residues of all four rows -- before
// combining them.  (One byte load per plane and row kept four times as many
// loads in flight for the same bytes; four columns per group took 113
// registers and ran 8% slower.)
template <bool CPLX>
__global__ void __launch_bounds__(256) crt_kernel(const __grid_constant__ CrtParams P) {
  extern __shared__ __align__(16) unsigned char crt_smem[];
  CrtEntry* tab = reinterpret_cast<CrtEntry*>(crt_smem);
  for (int e = threadIdx.x; e < P.n * 256; e += blockDim.x) {
    const int i = e >> 8, r = e & 255;
    CrtEntry t{0, 0};
    if (r < P.mod[i]) {
      const uint64_t c = (uint64_t)((r * P.y[i]) % P.mod[i]);
      const unsigned __int128 v = (unsigned __int128)c * (((unsigned __int128)P.mi_hi[i] << 64) | P.mi_lo[i]);
      t.lo = (uint64_t)v;
      t.hi = (uint64_t)(v >> 64);
    }
    tab[e] = t;
  }
  __syncthreads();
  constexpr int RC = CPLX ? 2 : 1;  // residue columns per D entry
  for (int64_t n = blockIdx.x; n < P.cols; n += gridDim.x) {
    const int ce = P.colexp[CPLX ? 2 * n : n];
    if (ce >= kNonFiniteExp) continue;  // flagged column: the fix-up's
    const int64_t dno = P.dn[n];
    for (int64_t m0 = 4 * (int64_t)threadIdx.x; m0 < P.rows; m0 += 4 * (int64_t)blockDim.x) {
      uint32_t w[RC][kMaxModuli];
#pragma unroll
      for (int j = 0; j < RC; ++j) crt_load4(P, n * RC + j, m0, w[j]);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int64_t m = m0 + t;
        if (m >= P.rows) break;
        const int re = P.rowexp[m];
        if (re >= kNonFiniteExp) continue;  // flagged row: the fix-up's
        const int e = re + ce - P.shift;
        const int64_t o = P.dm[m] + dno;
        uint32_t r[kMaxModuli];
        crt_byte(w[0], t, r);
        if constexpr (!CPLX) {
          double* D = (double*)P.D;
          const double v = P.ar * scale2(crt_combine(P, tab, r), e);
          D[o] = P.br == 0.0 ? v : fma(P.br, D[o], v);
        } else {
          const double xr = scale2(crt_combine(P, tab, r), e);
          crt_byte(w[RC - 1], t, r);
          const double xi = scale2(crt_combine(P, tab, r), e);
          double2* D = (double2*)P.D;
          double2 v;
          v.x = P.ar * xr - P.ai * xi;
          v.y = P.ar * xi + P.ai * xr;
          if (P.br != 0.0 || P.bi != 0.0) {
            const double2 d = D[o];
            v.x += P.br * d.x - P.bi * d.y;
            v.y += P.br * d.y + P.bi * d.x;
          }
          D[o] = v;
        }
      }
    }
  }
}

// Row maxima of the FP64 exponent fields (the slice scales), streamed without
// shared-memory staging: each thread keeps the running maximum of the rows it
// touches in registers over all K tiles of its CTA, and the CTA merges them once
// at the end.  Thread -> (row, k) mapping as in gather_kernel.
template <bool CPLX>
__device__ __forceinline__ void rowmax_body(const GatherParams& P, int64_t rowtile, int ky, int kstep) {
  using E = typename std::conditional<CPLX, double2, double>::type;
  constexpr int TM = gather_rows<E>(), TK = kGK, IT = TM * TK / kGThreads;
  __shared__ unsigned sm_max[TM];
  const int tid = threadIdx.x;
  if (tid < TM) sm_max[tid] = 0;
  const int64_t m0 = rowtile * TM;
  const E* src = (const E*)P.src;
  const int64_t nkt = (P.K + TK - 1) / TK;
  if (!P.lanes_on_k) {
    // rows contiguous in the source: each thread keeps one row (tid % TM) and
    // walks k = tid / TM + j * (threads / TM) -- one offset, one maximum
    constexpr int KS = kGThreads / TM;
    const int mm = tid % TM;
    const int64_t lm = m0 + mm < P.rows ? P.lm[m0 + mm] : -1;
    unsigned e = 0;
    if (lm >= 0) {
      for (int64_t kt = ky; kt < nkt; kt += kstep) {
        const int64_t k0 = kt * TK + tid / TM;
#pragma unroll
        for (int it = 0; it < TK / KS; ++it) {
          const int64_t k = k0 + it * KS;
          if (k < P.K) {
            const E v = src[lm + P.lk[k]];
            if constexpr (CPLX) e = max(e, max(exp_field(v.x), exp_field(v.y)));
            else e = max(e, exp_field(v));
          }
        }
      }
    }
    __syncthreads();
    if (e) atomicMax(&sm_max[mm], e);
    __syncthreads();
    if (tid < TM && sm_max[tid] && m0 + tid < P.rows) atomicMax(&P.rowE[m0 + tid], sm_max[tid]);
    return;
  }
  int64_t lmv[IT];
  unsigned emax[IT];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = tid + it * kGThreads;
    const int mm = idx / TK;
    lmv[it] = m0 + mm < P.rows ? P.lm[m0 + mm] : -1;
    emax[it] = 0;
  }
  for (int64_t kt = ky; kt < nkt; kt += kstep) {
    const int64_t k0 = kt * TK;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int idx = tid + it * kGThreads;
      const int kk = idx % TK;
      if (lmv[it] >= 0 && k0 + kk < P.K) {
        const E v = src[lmv[it] + P.lk[k0 + kk]];
        if constexpr (CPLX) emax[it] = max(emax[it], max(exp_field(v.x), exp_field(v.y)));
        else emax[it] = max(emax[it], exp_field(v));
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = tid + it * kGThreads;
    const int mm = idx / TK;
    if (emax[it]) atomicMax(&sm_max[mm], emax[it]);
  }
  __syncthreads();
  if (tid < TM && sm_max[tid] && m0 + tid < P.rows) atomicMax(&P.rowE[m0 + tid], sm_max[tid]);
}

template <bool CPLX>
__global__ void __launch_bounds__(kGThreads) rowmax_kernel(const __grid_constant__ GatherParams P) {
  rowmax_body<CPLX>(P, blockIdx.x, blockIdx.y, gridDim.y);
}

template <bool CPLX>
__global__ void __launch_bounds__(kGThreads) rowmax_grouped_kernel(const GatherParams* __restrict__ jobs,
                                                                   const int2* __restrict__ map) {
  const int2 jm = map[blockIdx.x];
  const GatherParams P = jobs[jm.x];
  rowmax_body<CPLX>(P, jm.y, blockIdx.y, gridDim.y);
}

template <bool CPLX>
int run_rowmax(const GatherParams& P, int64_t grid_rows, int64_t grid_k, cudaStream_t s) {
  if (grid_rows <= 0 || grid_k <= 0) return 0;
  if (grid_rows > INT32_MAX) { set_error("gather grid too large"); return TB_ERR_LIMIT; }
  int64_t gy = std::max<int64_t>(1, std::min<int64_t>(grid_k, (int64_t)num_sms() * 16 / std::max<int64_t>(1, grid_rows)));
  gy = std::min<int64_t>(gy, 65535);
  rowmax_kernel<CPLX><<<dim3((unsigned)grid_rows, (unsigned)gy), kGThreads, 0, s>>>(P);
  TB_CHECK_LAUNCH();
  return 0;
}

template <int MODE>
int run_gather(const GatherParams& P, int64_t grid_rows, int64_t grid_k, cudaStream_t s) {
  if (grid_rows <= 0 || grid_k <= 0) return 0;
  if (grid_rows > INT32_MAX) { set_error("gather grid too large"); return TB_ERR_LIMIT; }
  // enough CTAs to fill the GPU several times over; each walks a strided set of K tiles
  int64_t gy = std::max<int64_t>(1, std::min<int64_t>(grid_k, (int64_t)num_sms() * 16 / std::max<int64_t>(1, grid_rows)));
  gy = std::min<int64_t>(gy, 65535);
  constexpr int smem = gather_smem_bytes<MODE>();
  auto launch = [&](auto kern, DeviceOnce& once) -> int {
    const cudaError_t e = smem_limit_once(once, kern, smem);
    if (e != cudaSuccess) { set_error("gather smem attribute: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
    kern<<<dim3((unsigned)grid_rows, (unsigned)gy), kGThreads, smem, s>>>(P);
    return 0;
  };
  static DeviceOnce once3, once4;
  int err = 0;
  if constexpr (MODE == G_RESID_R8 || MODE == G_RESID_C8A || MODE == G_RESID_C8B) {
    err = P.rs.ndig > 3 ? launch(gather_kernel<MODE, 4>, once4) : launch(gather_kernel<MODE, 3>, once3);
  } else {
    err = launch(gather_kernel<MODE>, once3);
  }
  if (err) return err;
  TB_CHECK_LAUNCH();
  return 0;
}


}  // namespace
}  // namespace tb
