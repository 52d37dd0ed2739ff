// tb_tc.cu -- the tensor-core contraction path (TB_METHOD_FUSED).
//
// FP64 (R8, C8): Ozaki-style splitting into INT8 slices.  Each row m of the
// matricized left operand is scaled by 2^-e_m (e_m from the row's largest
// exponent) into (-1, 1) and written as s signed 7-bit digits
// a = 2^e_m * sum_i A_i 2^(-7i) (truncation, exact in FP64); the right
// operand likewise per column.  The tcgen05 GEMM (tb_tc_gemm.cuh) multiplies
// slice pairs (i, j) with i + j <= s + 1 exactly in INT32, grouping pairs with
// the same i + j into one TMEM accumulator as long as no INT32 overflow is
// possible, and the epilogue adds 2^(e_m + f_n - 7(i+j)) * acc in FP64 into D.
// FP32 (R4, C4): each value splits into BF16 high and low parts; the three
// products hi*hi + hi*lo + lo*hi accumulate in FP32 in TMEM.
// Complex data runs as a real GEMM of twice the size: A' = [Ar Ai] interleaved
// along K, B' rows (2n, 2n+1) = ([Br, -Bi], [Bi, Br]), so that columns (2n,
// 2n+1) of the product hold the real and imaginary parts of C(m, n).
//
// The operand preparation reads the tensors in their own layouts through the
// permutation engine (the input permutations are fused into the conversion),
// and the epilogue writes D through per-row and per-column offset tables (the
// output permutation) with alpha and beta applied.
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "tb_common.cuh"
#include "tb_contract.h"
#include "tb_permute.cuh"
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

// ---- operand preparation functors (applied by the permutation engine) ----------
// Output offsets o address a virtual [row][kpad] matrix (complex: complex units).
__device__ __forceinline__ unsigned exp_field(double x) {
  return (unsigned)((__double_as_longlong(x) >> 52) & 0x7FF);
}
__device__ __forceinline__ void row_max_exp(unsigned* rowE, uint64_t m, unsigned E) {
  if (E > *(volatile unsigned*)&rowE[m]) atomicMax(&rowE[m], E);
}

struct RowExpR8 {
  unsigned* rowE; FastDiv kdiv;
  __device__ __forceinline__ void operator()(int64_t o, const double& v) const {
    row_max_exp(rowE, kdiv.div((uint64_t)o), exp_field(v));
  }
};
struct RowExpC8 {
  unsigned* rowE; FastDiv kdiv;
  __device__ __forceinline__ void operator()(int64_t o, const double2& v) const {
    row_max_exp(rowE, kdiv.div((uint64_t)o), max(exp_field(v.x), exp_field(v.y)));
  }
};

// s signed 7-bit digits of x in (-1, 1): x = sum_i d_i 2^(-7 i) + remainder.
template <int S>
__device__ __forceinline__ void digits(double x, int8_t (&d)[S]) {
#pragma unroll
  for (int i = 0; i < S; ++i) {
    x *= 128.0;
    const double t = trunc(x);
    d[i] = (int8_t)(int)t;
    x -= t;
  }
}

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

struct SplitR4 {
  __nv_bfloat16* planes; int64_t pstride;
  __device__ __forceinline__ void operator()(int64_t o, const float& v) const {
    __nv_bfloat16 h, l;
    split_bf16(v, h, l);
    planes[o] = h;
    planes[pstride + o] = l;
  }
};
struct SplitC4A {
  __nv_bfloat16* planes; int64_t pstride; float isign;
  __device__ __forceinline__ void operator()(int64_t o, const float2& v) const {
    __nv_bfloat16 hr, lr, hi, li;
    split_bf16(v.x, hr, lr);
    split_bf16(isign * v.y, hi, li);
    __nv_bfloat162 a; a.x = hr; a.y = hi;
    __nv_bfloat162 b; b.x = lr; b.y = li;
    *reinterpret_cast<__nv_bfloat162*>(planes + 2 * o) = a;
    *reinterpret_cast<__nv_bfloat162*>(planes + pstride + 2 * o) = b;
  }
};
struct SplitC4B {
  __nv_bfloat16* planes; int64_t pstride; int64_t kcpad; FastDiv kdiv; float isign;
  __device__ __forceinline__ void operator()(int64_t o, const float2& v) const {
    const uint64_t n = kdiv.div((uint64_t)o);
    const int64_t k = o - (int64_t)n * kcpad;
    const int64_t r0 = (int64_t)(2 * n) * (2 * kcpad) + 2 * k, r1 = r0 + 2 * kcpad;
    const float br = v.x, bi = isign * v.y;
    __nv_bfloat16 hr, lr, hi, li, nhi, nli;
    split_bf16(br, hr, lr);
    split_bf16(bi, hi, li);
    split_bf16(-bi, nhi, nli);
    __nv_bfloat162 w;
    w.x = hr; w.y = nhi; *reinterpret_cast<__nv_bfloat162*>(planes + r0) = w;
    w.x = hi; w.y = hr;  *reinterpret_cast<__nv_bfloat162*>(planes + r1) = w;
    w.x = lr; w.y = nli; *reinterpret_cast<__nv_bfloat162*>(planes + pstride + r0) = w;
    w.x = li; w.y = lr;  *reinterpret_cast<__nv_bfloat162*>(planes + pstride + r1) = w;
  }
};

// exponents: rowexp[r] = rowE[r / rep] - 1022 (rep = 2 for complex B' rows)
__global__ void exps_kernel(const unsigned* __restrict__ rowE, int* __restrict__ out, int64_t n, int rep) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int)rowE[i / rep] - 1022;
}

// ---- driver ----------------------------------------------------------------------
constexpr int kDefaultSlices = 7;
constexpr int kMaxSlices = 8;

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// One operand of the GEMM: a source tensor, its row groups and its contracted
// dims (positions and extents in Z.k order).
struct Operand {
  const void* ptr;
  int rank;
  const int* dims;
  std::vector<MGroup> rows;   // uncontracted groups: s1 = stride in this tensor, s2 = stride in D
  std::vector<int> kpos;      // position of each contracted dim (Z.k order) in this tensor
  bool conj;
};

// Permutation-engine strides that map the tensor onto a virtual [row][rowlen]
// matrix (K fastest, contracted dims in Z.k order, rows in group order).
void gather_plan_dims(const Operand& op, const Matricization& Z, int64_t rowlen, int64_t* D, int64_t* SI,
                      int64_t* SO) {
  int64_t s = 1;
  for (int i = 0; i < op.rank; ++i) { D[i] = op.dims[i]; SI[i] = s; s *= op.dims[i]; }
  int64_t ks = 1;
  for (size_t q = 0; q < Z.k.size(); ++q) { SO[op.kpos[q]] = ks; ks *= Z.k[q].ext; }
  int64_t rs = rowlen;
  for (auto& g : op.rows) { SO[g.src] = rs; rs *= g.ext; }
}

template <typename E, typename F>
int gather(const Operand& op, const Matricization& Z, int64_t rowlen, const F& f, cudaStream_t s) {
  int64_t D[kMaxRank], SI[kMaxRank], SO[kMaxRank];
  gather_plan_dims(op, Z, rowlen, D, SI, SO);
  PermParams P;
  if (int e = build_perm_plan((int)sizeof(E), op.rank, D, SI, SO, &P)) {
    set_error("operand gather plan declined (%d)", e);
    return e == TB_ERR_NOT_IMPLEMENTED ? TB_ERR_NOT_IMPLEMENTED : e;
  }
  return launch_perm<E, F>(P, (const E*)op.ptr, f, s);
}

// Real and complex slice functors with a runtime slice count (<= kMaxSlices).
struct SliceR8R {
  int8_t* planes; int64_t pstride; const unsigned* rowE; FastDiv kdiv; int s;
  __device__ __forceinline__ void operator()(int64_t o, const double& v) const {
    const uint64_t m = kdiv.div((uint64_t)o);
    int8_t d[kMaxSlices];
    digits<kMaxSlices>(v * pow2d(1022 - (int)rowE[m]), d);
#pragma unroll
    for (int i = 0; i < kMaxSlices; ++i) if (i < s) planes[i * pstride + o] = d[i];
  }
};
struct SliceC8AR {
  int8_t* planes; int64_t pstride; const unsigned* rowE; FastDiv kdiv; double isign; int s;
  __device__ __forceinline__ void operator()(int64_t o, const double2& v) const {
    const uint64_t m = kdiv.div((uint64_t)o);
    const double sc = pow2d(1022 - (int)rowE[m]);
    int8_t dr[kMaxSlices], di[kMaxSlices];
    digits<kMaxSlices>(v.x * sc, dr);
    digits<kMaxSlices>(isign * v.y * sc, di);
#pragma unroll
    for (int i = 0; i < kMaxSlices; ++i)
      if (i < s) {
        char2 w; w.x = dr[i]; w.y = di[i];
        *reinterpret_cast<char2*>(planes + i * pstride + 2 * o) = w;
      }
  }
};
struct SliceC8BR {
  int8_t* planes; int64_t pstride; int64_t kcpad; const unsigned* rowE; FastDiv kdiv; double isign; int s;
  __device__ __forceinline__ void operator()(int64_t o, const double2& v) const {
    const uint64_t n = kdiv.div((uint64_t)o);
    const int64_t k = o - (int64_t)n * kcpad;
    const double sc = pow2d(1022 - (int)rowE[n]);
    int8_t dr[kMaxSlices], di[kMaxSlices];
    digits<kMaxSlices>(v.x * sc, dr);
    digits<kMaxSlices>(isign * v.y * sc, di);
    const int64_t r0 = (int64_t)(2 * n) * (2 * kcpad) + 2 * k, r1 = r0 + 2 * kcpad;
#pragma unroll
    for (int i = 0; i < kMaxSlices; ++i)
      if (i < s) {
        char2 a; a.x = dr[i]; a.y = (int8_t)(-di[i]);
        char2 b; b.x = di[i]; b.y = dr[i];
        *reinterpret_cast<char2*>(planes + i * pstride + r0) = a;
        *reinterpret_cast<char2*>(planes + i * pstride + r1) = b;
      }
  }
};

template <int BN, bool I8, int EPI>
int launch_tc(const TcGemmParams& P, cudaStream_t s) {
  constexpr size_t smem = tc_smem_bytes<BN>();
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(tc_gemm_kernel<BN, I8, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) { set_error("tcgen05 GEMM smem attribute: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
    attr = true;
  }
  const int tiles = P.mtiles * P.ntiles;
  const int grid = std::max(1, std::min(tiles, num_sms()));
  tc_gemm_kernel<BN, I8, EPI><<<grid, kTcThreads, smem, s>>>(P);
  TB_CHECK_LAUNCH();
  return 0;
}

template <int BN>
int launch_tc_epi(const TcGemmParams& P, int epi, cudaStream_t s) {
  switch (epi) {
    case EPI_OZAKI_R: return launch_tc<BN, true, EPI_OZAKI_R>(P, s);
    case EPI_OZAKI_C: return launch_tc<BN, true, EPI_OZAKI_C>(P, s);
    case EPI_BF16_R: return launch_tc<BN, false, EPI_BF16_R>(P, s);
    default: return launch_tc<BN, false, EPI_BF16_C>(P, s);
  }
}

}  // namespace

int select_method(int dtk, const Matricization& Z, const tb_plan_t* plan) {
  (void)dtk;
  if (plan && plan->method != TB_METHOD_AUTO) return plan->method;
  // tensor cores pay off once the GEMM is large enough to fill the GPU
  const double flops = 2.0 * (double)Z.M * (double)Z.N * (double)Z.K;
  if (Z.M >= 64 && Z.N >= 32 && Z.K >= 64 && flops >= 4e9) return TB_METHOD_FUSED;
  return TB_METHOD_TTGT;
}

int contract_fused(const Matricization& Z0, int dtk, const int* ddims, void* d, const int* ldims, const void* l,
                   const int* rdims, const void* r, double ar, double ai, bool accumulate, int lconj, int rconj,
                   const tb_plan_t* plan, cudaStream_t s, tb_contract_stats_t* stats) {
  (void)ddims;
  if (Z0.K < 1 || Z0.M < 1 || Z0.N < 1 || Z0.k.empty()) return TB_ERR_NOT_IMPLEMENTED;
  Matricization Z = Z0;
  // rows in D-stride order so that consecutive epilogue lanes write consecutive D
  auto by_d = [](const MGroup& x, const MGroup& y) { return x.s2 < y.s2; };
  std::stable_sort(Z.m.begin(), Z.m.end(), by_d);
  std::stable_sort(Z.n.begin(), Z.n.end(), by_d);
  // the operand holding D's fastest dimension plays the row (M) role
  const bool swap = !Z.n.empty() && (Z.m.empty() || Z.n[0].s2 < Z.m[0].s2);
  Operand Lop{l, Z.lrank, ldims, Z.m, {}, lconj != 0}, Rop{r, Z.rrank, rdims, Z.n, {}, rconj != 0};
  for (auto& g : Z.k) { Lop.kpos.push_back(g.dpos); Rop.kpos.push_back(g.src); }
  const Operand& A = swap ? Rop : Lop;
  const Operand& B = swap ? Lop : Rop;
  const bool cplx = is_complex(dtk), i8 = is_double(dtk);
  int64_t M = 1, Nc = 1;
  for (auto& g : A.rows) M *= g.ext;
  for (auto& g : B.rows) Nc *= g.ext;
  const int64_t K = Z.K;
  const int64_t Kr = cplx ? 2 * K : K, Nr = cplx ? 2 * Nc : Nc;
  const int64_t Kpad = round_up(Kr, 128);
  const int BN = (plan && plan->tile_n == 128) ? 128 : (plan && plan->tile_n == 256) ? 256 : (Nr >= 192 ? 256 : 128);
  const int64_t Mpad = round_up(M, 128), Npad = round_up(Nr, BN);
  if (Mpad / 128 * (Npad / BN) > INT32_MAX || M > INT32_MAX || Nr > INT32_MAX) return TB_ERR_LIMIT;
  // products and passes
  std::vector<std::vector<std::pair<int, int>>> passes;
  std::vector<int> shifts;
  int S = 0, npa = 2, npb = 2;
  if (i8) {
    S = (plan && plan->slices > 0) ? plan->slices : kDefaultSlices;
    if (S < 2 || S > kMaxSlices) { set_error("slice count %d outside 2..%d", S, kMaxSlices); return TB_ERR_INVALID_ARGS; }
    const int64_t per = (int64_t)127 * 127 * Kr;
    const int64_t cap = (int64_t)INT32_MAX / per;
    if (cap < 1) return TB_ERR_NOT_IMPLEMENTED;  // K too long for exact INT32 accumulation
    for (int dsum = 2; dsum <= S + 1; ++dsum) {
      std::vector<std::pair<int, int>> diag;
      for (int i = 1; i < dsum; ++i)
        if (i <= S && dsum - i <= S) diag.push_back({i - 1, dsum - i - 1});
      for (size_t b = 0; b < diag.size(); b += cap) {
        passes.emplace_back(diag.begin() + b, diag.begin() + std::min(diag.size(), (size_t)(b + cap)));
        shifts.push_back(7 * dsum);
      }
    }
    npa = npb = S;
  } else {
    const int terms = (plan && plan->bf16_terms == 4) ? 4 : 3;
    std::vector<std::pair<int, int>> p3 = {{0, 0}, {0, 1}, {1, 0}};
    if (terms == 4) p3.push_back({1, 1});
    passes.push_back(p3);
    shifts.push_back(0);
  }
  int nprod = 0;
  for (auto& p : passes) nprod += (int)p.size();
  if (nprod > kMaxProducts || (int)passes.size() > kMaxProducts) return TB_ERR_NOT_IMPLEMENTED;
  // scratch: operand planes, offset tables, exponents
  const int oes = i8 ? 1 : 2;
  const size_t bytesA = (size_t)npa * Mpad * Kpad * oes, bytesB = (size_t)npb * Npad * Kpad * oes;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t offA = 0, offB = al(bytesA), offDm = offB + al(bytesB), offDn = offDm + al(M * 8),
               offRE = offDn + al(Nc * 8), offCE = offRE + al(M * 4), offRX = offCE + al(Nc * 4),
               offCX = offRX + al(M * 4), total = offCX + al(Nr * 4);
  unsigned char* ws = nullptr;
  if (int e = scratch_alloc((void**)&ws, total, s)) return e;
  int err = 0;
  int8_t* Ap = (int8_t*)(ws + offA);
  int8_t* Bp = (int8_t*)(ws + offB);
  int64_t* dm = (int64_t*)(ws + offDm);
  int64_t* dn = (int64_t*)(ws + offDn);
  unsigned* rowE = (unsigned*)(ws + offRE);
  unsigned* colE = (unsigned*)(ws + offCE);
  int* rowx = (int*)(ws + offRX);
  int* colx = (int*)(ws + offCX);
  const bool padded = Mpad != M || Npad != Nr || Kpad != Kr;
  const int64_t rowlen = cplx ? Kpad / 2 : Kpad;  // gather row length in source elements
  do {
    if (padded && (cudaMemsetAsync(ws, 0, offDm, s) != cudaSuccess)) { err = TB_ERR_CUDA; break; }
    if ((err = build_offsets(A.rows, true, dm, s))) break;
    if ((err = build_offsets(B.rows, true, dn, s))) break;
    if (i8) {
      if (cudaMemsetAsync(rowE, 0, offRX - offRE, s) != cudaSuccess) { err = TB_ERR_CUDA; break; }
      const FastDiv kd((uint64_t)rowlen);
      if (!cplx) {
        if ((err = gather<double>(A, Z, rowlen, RowExpR8{rowE, kd}, s))) break;
        if ((err = gather<double>(B, Z, rowlen, RowExpR8{colE, kd}, s))) break;
      } else {
        if ((err = gather<double2>(A, Z, rowlen, RowExpC8{rowE, kd}, s))) break;
        if ((err = gather<double2>(B, Z, rowlen, RowExpC8{colE, kd}, s))) break;
      }
      exps_kernel<<<std::max<int64_t>(1, std::min<int64_t>((M + 255) / 256, 4096)), 256, 0, s>>>(rowE, rowx, M, 1);
      exps_kernel<<<std::max<int64_t>(1, std::min<int64_t>((Nr + 255) / 256, 4096)), 256, 0, s>>>(colE, colx, Nr,
                                                                                                  cplx ? 2 : 1);
      count_launch();
      count_launch();
      const int64_t psA = Mpad * Kpad, psB = Npad * Kpad;
      if (!cplx) {
        if ((err = gather<double>(A, Z, rowlen, SliceR8R{Ap, psA, rowE, kd, S}, s))) break;
        if ((err = gather<double>(B, Z, rowlen, SliceR8R{Bp, psB, colE, kd, S}, s))) break;
      } else {
        if ((err = gather<double2>(A, Z, rowlen, SliceC8AR{Ap, psA, rowE, kd, A.conj ? -1.0 : 1.0, S}, s))) break;
        if ((err = gather<double2>(B, Z, rowlen, SliceC8BR{Bp, psB, rowlen, colE, kd, B.conj ? -1.0 : 1.0, S}, s)))
          break;
      }
    } else {
      __nv_bfloat16* Ah = (__nv_bfloat16*)Ap;
      __nv_bfloat16* Bh = (__nv_bfloat16*)Bp;
      const int64_t psA = Mpad * Kpad, psB = Npad * Kpad;
      if (!cplx) {
        if ((err = gather<float>(A, Z, rowlen, SplitR4{Ah, psA}, s))) break;
        if ((err = gather<float>(B, Z, rowlen, SplitR4{Bh, psB}, s))) break;
      } else {
        const FastDiv kd((uint64_t)rowlen);
        if ((err = gather<float2>(A, Z, rowlen, SplitC4A{Ah, psA, A.conj ? -1.f : 1.f}, s))) break;
        if ((err = gather<float2>(B, Z, rowlen, SplitC4B{Bh, psB, rowlen, kd, B.conj ? -1.f : 1.f}, s))) break;
      }
    }
    // GEMM parameters
    static TcGemmParams P;  // large: kept off the stack
    std::memset(&P, 0, sizeof(P));
    if ((err = make_operand_map(&P.tmA, Ap, i8, Kpad, Mpad, npa, 128))) break;
    if ((err = make_operand_map(&P.tmB, Bp, i8, Kpad, Npad, npb, BN))) break;
    P.M = (int)M; P.N = (int)Nr;
    P.mtiles = (int)(Mpad / 128); P.ntiles = (int)(Npad / BN);
    P.kblocks = (int)(Kpad * oes / 128);
    P.npass = (int)passes.size();
    int q = 0;
    for (size_t p = 0; p < passes.size(); ++p) {
      P.pass_first[p] = q;
      P.pass_shift[p] = shifts[p];
      for (auto& pr : passes[p]) { P.prod_a[q] = pr.first; P.prod_b[q] = pr.second; ++q; }
    }
    P.pass_first[passes.size()] = q;
    P.D = d; P.dm = dm; P.dn = dn; P.rowexp = rowx; P.colexp = colx;
    const double realpha = cplx ? ar : (ar != 0.0 ? std::hypot(ar, ai) * (ar > 0 ? 1.0 : -1.0) : ai);
    P.ar = realpha; P.ai = cplx ? ai : 0.0;
    P.br = accumulate ? 1.0 : 0.0; P.bi = 0.0;
    P.err = device_error_word();
    const int epi = i8 ? (cplx ? EPI_OZAKI_C : EPI_OZAKI_R) : (cplx ? EPI_BF16_C : EPI_BF16_R);
    const int ts = timed_begin(s);
    err = BN == 256 ? launch_tc_epi<256>(P, epi, s) : launch_tc_epi<128>(P, epi, s);
    timed_end(ts, s);
    if (stats) {
      stats->slices = S;
      stats->passes = (int)passes.size();
      stats->gemm_launches = 1;
      stats->m = M; stats->n = Nr; stats->k = Kr;
    }
  } while (false);
  scratch_free(ws, s);
  return err;
}

}  // namespace tb
