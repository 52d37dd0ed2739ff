// tb_tc.cu -- the tensor-core contraction path (TB_METHOD_FUSED).
//
// FP64 (R8, C8): Ozaki-style splitting into 8-bit slices.  Each row m of the
// matricized left operand is scaled by 2^-e_m (e_m from the row's largest
// exponent) into (-1/2, 1/2) and cut into s balanced signed 8-bit digits of
// weight 2^-(8i+7), i = 0..s-1 (exact in FP64; see fixed55); the right
// operand likewise per column.  The tcgen05 GEMM (tb_tc_gemm.cuh) multiplies
// slice pairs (i, j) with i + j <= s - 1 exactly in INT32 (kind::i8),
// grouping pairs of equal i + j, split along K where needed, into one TMEM
// accumulator while no INT32 overflow is possible, and the epilogue adds
// 2^(e_m + f_n - 8(i+j) - 14) * acc in FP64 into D.
// FP32 (R4, C4): each value splits into BF16 high and low parts; the three
// products hi*hi + hi*lo + lo*hi accumulate in FP32 in TMEM.
// Complex data runs as a real GEMM of twice the size: A' = [Ar Ai] interleaved
// along K, B' rows (2n, 2n+1) = ([Br, -Bi], [Bi, Br]), so that columns (2n,
// 2n+1) of the product hold the real and imaginary parts of C(m, n).
//
// The operand preparation reads the tensors in their own layouts through
// per-row and per-index offset tables (the input permutations are fused into
// the conversion to slices or BF16 parts),
// and the epilogue writes D through per-row and per-column offset tables (the
// output permutation) with alpha and beta applied.
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "tb_common.cuh"
#include "tb_contract.h"
#include "tb_permute.cuh"
#include "tb_tc_gemm.cuh"
#include "tb_tc_prep.cuh"

namespace tb {

namespace {

// ---- driver ----------------------------------------------------------------------
constexpr int kDefaultSlices = 6;
constexpr int kMaxSlices = 7;  // 7 slices hold all 55 bits of the fixed-point value
constexpr int kBf16PassKBlocks = 32;  // split-BF16: K blocks (64 values each) per accumulator pass

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// One operand of the GEMM: a source tensor, its row groups and its contracted
// dims (Z.k order), each with strides in this tensor (s1) and in D (s2).
struct Operand {
  const void* ptr;
  std::vector<MGroup> rows;   // uncontracted groups: s1 = stride in this tensor, s2 = stride in D
  std::vector<MGroup> ks;     // contracted groups: s1 = stride in this tensor
  bool conj;
};

template <int BN, bool I8, int EPI>
int launch_tc(const TcGemmParams& P, cudaStream_t s) {
  constexpr size_t smem = tc_smem_bytes<BN>();
  static DeviceOnce attr;
  const cudaError_t e = smem_limit_once(attr, tc_gemm_kernel<BN, I8, EPI>, (int)smem);
  if (e != cudaSuccess) { set_error("tcgen05 GEMM smem attribute: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
  const int grid = std::max(1, std::min(gemm_units<EPI>(P), num_sms()));
  tc_gemm_kernel<BN, I8, EPI><<<grid, kTcThreads, smem, s>>>(P);
  TB_CHECK_LAUNCH();
  return 0;
}

// CTA-pair kernel: grid = 2 x (pairs that can be resident at once, capped by the tiles).
template <int BN, bool I8, int EPI>
int launch_tc2(const TcGemmParams& P, cudaStream_t s) {
  constexpr size_t smem = tc2_smem_bytes<BN>();
  // per device: the shared-memory limit and the pairs resident at once
  static std::atomic<int> max_pairs_of[64];
  const int dev = current_device();
  int max_pairs = max_pairs_of[dev].load(std::memory_order_relaxed);
  if (!max_pairs) {
    cudaError_t e = cudaFuncSetAttribute(tc_gemm2_kernel<BN, I8, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) { set_error("tcgen05 pair GEMM smem attribute: %s", cudaGetErrorString(e)); return TB_ERR_CUDA; }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * (unsigned)num_sms(), 1, 1);
    cfg.blockDim = dim3(kTcThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = 2; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int n = 0;
    e = cudaOccupancyMaxActiveClusters(&n, tc_gemm2_kernel<BN, I8, EPI>, &cfg);
    if (e != cudaSuccess || n < 1) {
      cudaGetLastError();
      n = num_sms() / 2;
    }
    max_pairs = n;
    max_pairs_of[dev].store(n, std::memory_order_relaxed);
  }
  const int pairs = std::max(1, std::min(gemm_units<EPI>(P), max_pairs));
  tc_gemm2_kernel<BN, I8, EPI><<<2 * pairs, kTcThreads, smem, s>>>(P);
  TB_CHECK_LAUNCH();
  return 0;
}

template <int BN>
int launch_tc_epi(const TcGemmParams& P, int epi, bool pair, cudaStream_t s) {
  if (pair) {
    switch (epi) {
      case EPI_RESID: return launch_tc2<BN, true, EPI_RESID>(P, s);
      case EPI_OZAKI_R: return launch_tc2<BN, true, EPI_OZAKI_R>(P, s);
      case EPI_OZAKI_C: return launch_tc2<BN, true, EPI_OZAKI_C>(P, s);
      case EPI_BF16_R: return launch_tc2<BN, false, EPI_BF16_R>(P, s);
      default: return launch_tc2<BN, false, EPI_BF16_C>(P, s);
    }
  }
  switch (epi) {
    case EPI_RESID: return launch_tc<BN, true, EPI_RESID>(P, s);
    case EPI_OZAKI_R: return launch_tc<BN, true, EPI_OZAKI_R>(P, s);
    case EPI_OZAKI_C: return launch_tc<BN, true, EPI_OZAKI_C>(P, s);
    case EPI_BF16_R: return launch_tc<BN, false, EPI_BF16_R>(P, s);
    default: return launch_tc<BN, false, EPI_BF16_C>(P, s);
  }
}

// ---- Ozaki scheme II: modular residues -----------------------------------------
// Pairwise coprime moduli <= 256, largest first (their residues in the
// symmetric range are signed 8-bit).  With n of them, M = prod m_i and the
// operands scaled to integers |X| <= 2^p, an exact INT32 GEMM per modulus and
// the Chinese remainder theorem give the exact integer product as long as
// M > 2 Kr 2^(2p) (Kr: the real contraction length).
constexpr int kModuliTable[kMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193};
constexpr bool moduli_table_matches() {
  for (int i = 0; i < kMaxModuli; ++i)
    if (kModuliTable[i] != residue_modulus(i)) return false;
  return true;
}
static_assert(moduli_table_matches(), "the gathers' compile-time moduli must be the plan's table");
constexpr int kMinModuli = 8;
constexpr int kMaxPassBlocks = 1023;  // K blocks of one exact INT32 pass (128^3 each, below 2^31)
constexpr int kResidueBitsTarget = 46;  // operand bits kept by the default choice (INT8 slices keep 47)

using u128 = unsigned __int128;

u128 moduli_product(int n) {
  u128 M = 1;
  for (int i = 0; i < n; ++i) M *= (u128)kModuliTable[i];
  return M;
}

// The largest p with M > 2 Kr 2^(2p) for n moduli (checked in exact integer arithmetic).
int residue_bits(int n, int64_t Kr) {
  const u128 M = moduli_product(n);
  int p = 0;
  while (p < 60 && (M >> (2 * (p + 1))) > (u128)(2 * Kr)) ++p;
  return p;
}

struct ResiduePlan {
  ResidueSpec rs;
  int p;
  CrtParams crt;  // constants only; pointers and sizes are filled by the caller
};

// Moduli count and constants for a contraction of real length Kr: `want` > 0
// asks for that many moduli, else the fewest with p >= kResidueBitsTarget.
// Returns false when no allowed count reaches kResidueBitsTarget bits.
bool plan_residues(int64_t Kr, int want, ResiduePlan* out) {
  int n = want;
  if (n <= 0) {
    for (n = kMinModuli; n <= kMaxModuli && residue_bits(n, Kr) < kResidueBitsTarget; ++n) {}
    if (n > kMaxModuli) return false;
  }
  if (n < kMinModuli || n > kMaxModuli) return false;
  // at most 52 bits: X = x 2^(p+1) rounded to an integer must be exact in
  // FP64; the automatic choice keeps the 46-bit target (three 16-bit digits
  // per operand in the gathers), an explicit moduli count all its bits
  const int p = std::min(residue_bits(n, Kr), want > 0 ? 52 : kResidueBitsTarget);
  if (p < 20) return false;
  ResiduePlan& R = *out;
  std::memset(&R, 0, sizeof(R));
  R.p = p;
  R.rs.n = n;
  R.rs.pscale = std::ldexp(1.0, p + 1);
  const u128 M = moduli_product(n);
  R.crt.n = n;
  R.crt.M_lo = (uint64_t)M;
  R.crt.M_hi = (uint64_t)(M >> 64);
  R.crt.Md = (double)(uint64_t)(M >> 64) * 18446744073709551616.0 + (double)(uint64_t)M;
  R.crt.shift = 2 * (p + 1);
  R.rs.p = p;
  R.rs.ndig = p <= 46 ? 3 : 4;
  for (int i = 0; i < n; ++i) {
    const int m = kModuliTable[i];
    const u128 Mi = M / (u128)m;
    const int mi_mod = (int)(Mi % (u128)m);
    int y = 0;
    for (int c = 1; c < m; ++c)
      if ((mi_mod * c) % m == 1) { y = c; break; }
    R.crt.mod[i] = m;
    R.crt.y[i] = y;
    R.crt.mi_lo[i] = (uint64_t)Mi;
    R.crt.mi_hi[i] = (uint64_t)(Mi >> 64);
  }
  return true;
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
  Operand Lop{l, Z.m, {}, lconj != 0}, Rop{r, Z.n, {}, rconj != 0};
  for (auto g : Z.k) {
    Lop.ks.push_back(g);                       // s1 = L stride
    MGroup h = g; h.s1 = g.s2; Rop.ks.push_back(h);  // R stride
  }
  (void)ldims; (void)rdims;
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
  // M tile: one SM per 128-row tile unless the plan asks for SM pairs (256
  // rows); the pair kernel halves the B traffic per SM but measured no faster
  // on the CCSD-like shapes, whose GEMMs run at the power cap.
  const bool pair = plan && plan->tile_m == 256;
  const int TM = pair ? 256 : 128;
  const int64_t Mpad = round_up(M, TM), Npad = round_up(Nr, BN);
  if (Mpad / 128 * (Npad / BN) > INT32_MAX || M > INT32_MAX || Nr > INT32_MAX) return TB_ERR_LIMIT;
  // products and passes: an entry multiplies plane a of A by plane b of B over
  // a K-block range; the entries of a pass share one exact INT32 accumulator.
  struct Entry { int a, b, kb0, kb1; };
  std::vector<std::vector<Entry>> passes;
  std::vector<int> shifts;
  const int kblocks = (int)(Kpad * (i8 ? 1 : 2) / 128);  // 128-byte K blocks
  int S = 0, npa = 2, npb = 2;
  // R8/C8: modular residues (one exact INT8 GEMM per modulus, fewer than the
  // slice pairs) unless the plan asks for INT8 slices or the contraction
  // needs more moduli; K ranges longer than one exact INT32 pass (1023 K
  // blocks) are cut into equal chunks whose residues the epilogue adds mod m.
  ResiduePlan RP;
  const int res_nch = (kblocks + kMaxPassBlocks - 1) / kMaxPassBlocks;
  const bool resid = i8 && !(plan && (plan->slices > 0 || plan->moduli < 0)) &&
                     plan_residues(Kr, plan ? plan->moduli : 0, &RP) && RP.rs.n * res_nch <= kMaxProducts;
  if (i8 && plan && plan->moduli > 0 && !resid) {
    set_error("modular residues: %d moduli do not fit this contraction (K = %lld)", plan->moduli, (long long)Kr);
    return TB_ERR_INVALID_ARGS;
  }
  if (resid) {
    const int chunk = (kblocks + res_nch - 1) / res_nch;
    for (int i = 0; i < RP.rs.n; ++i)
      for (int kb = 0; kb < kblocks; kb += chunk) {
        passes.push_back({{i, i, kb, std::min(kblocks, kb + chunk)}});
        shifts.push_back(RP.crt.mod[i]);  // the epilogue's modulus
      }
    npa = npb = RP.rs.n;
  } else if (i8) {
    S = (plan && plan->slices > 0) ? plan->slices : kDefaultSlices;
    if (S < 2 || S > kMaxSlices) { set_error("slice count %d outside 2..%d", S, kMaxSlices); return TB_ERR_INVALID_ARGS; }
    // |slice| <= 128, so one K block (128 products) adds at most 128^3.
    const int64_t cap = INT32_MAX;
    // The products of one i + j share a pass while the sum stays exact
    // (at most cap / 128^3 = 1023 K blocks per pass).  A group that needs
    // several passes gets passes of equal size, so that each pass's MMAs are
    // long enough to hide the previous pass's epilogue (1152 blocks: 576 +
    // 576, not 1023 + 129).
    const int64_t per_block = (int64_t)128 * 128 * 128;
    const int64_t max_blocks = cap / per_block;
    for (int dsum = 2; dsum <= S + 1; ++dsum) {   // 1-based slice indices with i + j = dsum
      int64_t total = 0;
      for (int i = 1; i < dsum; ++i)
        if (i <= S && dsum - i <= S) total += kblocks;
      if (total == 0) continue;
      const int64_t npass = (total + max_blocks - 1) / max_blocks;
      const int64_t room_max = (total + npass - 1) / npass;  // <= max_blocks
      std::vector<Entry> cur;
      int64_t load = 0;
      for (int i = 1; i < dsum; ++i) {
        const int j = dsum - i;
        if (i > S || j > S) continue;
        for (int kb = 0; kb < kblocks;) {
          if (load >= room_max) { passes.push_back(cur); shifts.push_back(8 * dsum - 2); cur.clear(); load = 0; }
          const int n = (int)std::min<int64_t>(room_max - load, kblocks - kb);
          cur.push_back({i - 1, j - 1, kb, kb + n});
          load += n;
          kb += n;
        }
      }
      if (!cur.empty()) { passes.push_back(cur); shifts.push_back(8 * dsum - 2); }
    }
    npa = npb = S;
  } else {
    // The FP32 accumulation of the tensor cores loses accuracy about linearly
    // with K (R4 CCSD-like, K = 36864: 1.8e-4 relative in one pass), so the K
    // range is cut into passes of kBf16PassKBlocks blocks (longer where the
    // entry limit requires) that the epilogue adds into D, one rounding each.
    static const int pass_kb = [] {
      const char* e = getenv("TB_BF16_PASS_KB");  // tuning knob
      const int v = e ? atoi(e) : 0;
      return v > 0 ? v : kBf16PassKBlocks;
    }();
    const int terms = (plan && plan->bf16_terms == 4) ? 4 : 3;
    const int max_passes = kMaxProducts / terms;  // the parameter block holds kMaxProducts entries
    const int step = std::max(pass_kb, (kblocks + max_passes - 1) / max_passes);
    for (int kb = 0; kb < kblocks; kb += step) {
      const int k1 = std::min(kblocks, kb + step);
      std::vector<Entry> p3 = {{0, 0, kb, k1}, {0, 1, kb, k1}, {1, 0, kb, k1}};
      if (terms == 4) p3.push_back({1, 1, kb, k1});
      passes.push_back(p3);
      shifts.push_back(0);
    }
  }
  int nprod = 0, nplane_products = 0;
  for (auto& p : passes) {
    nprod += (int)p.size();
    for (auto& e : p) nplane_products += (e.kb0 == 0);  // count each plane pair once
  }
  if (nprod > kMaxProducts || (int)passes.size() > kMaxProducts) {
    set_error("tensor-core plan needs %d GEMM entries in %d passes (limit %d)", nprod, (int)passes.size(),
              kMaxProducts);
    return TB_ERR_NOT_IMPLEMENTED;
  }
  // scratch: operand planes, offset tables, exponents
  const int oes = i8 ? 1 : 2;
  const size_t bytesA = (size_t)npa * Mpad * Kpad * oes, bytesB = (size_t)npb * Npad * Kpad * oes;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t offA = 0, offB = al(bytesA), offDm = offB + al(bytesB), offDn = offDm + al(M * 8),
               offLA = offDn + al(Nc * 8), offLB = offLA + al(M * 8), offKA = offLB + al(Nc * 8),
               offKB = offKA + al(K * 8), offRE = offKB + al(K * 8), offCE = offRE + al(M * 4),
               offRX = offCE + al(Nc * 4), offCX = offRX + al(M * 4), offBR = offCX + al(Nr * 4),
               offBC = offBR + al(M * 4), offNB = offBC + al(Nc * 4), offRES = offNB + 256,
               total = offRES + (resid ? al((size_t)RP.rs.n * Npad * Mpad) : 0);
  unsigned char* ws = nullptr;
  if (int e = scratch_alloc((void**)&ws, total, s)) return e;
  int err = 0;
  int8_t* Ap = (int8_t*)(ws + offA);
  int8_t* Bp = (int8_t*)(ws + offB);
  int64_t* dm = (int64_t*)(ws + offDm);
  int64_t* dn = (int64_t*)(ws + offDn);
  int64_t* lmA = (int64_t*)(ws + offLA);
  int64_t* lmB = (int64_t*)(ws + offLB);
  int64_t* lkA = (int64_t*)(ws + offKA);
  int64_t* lkB = (int64_t*)(ws + offKB);
  unsigned* rowE = (unsigned*)(ws + offRE);
  unsigned* colE = (unsigned*)(ws + offCE);
  int* rowx = (int*)(ws + offRX);
  int* colx = (int*)(ws + offCX);
  int* badrows = (int*)(ws + offBR);  // rows of A / columns of B holding a NaN or an infinity
  int* badcols = (int*)(ws + offBC);
  int* nbad = (int*)(ws + offNB);
  const int64_t ksrc_pad = cplx ? Kpad / 2 : Kpad;  // padded K in source elements
  do {
    if ((err = build_offsets(A.rows, true, dm, s))) break;
    if ((err = build_offsets(B.rows, true, dn, s))) break;
    if ((err = build_offsets(A.rows, false, lmA, s))) break;
    if ((err = build_offsets(B.rows, false, lmB, s))) break;
    if ((err = build_offsets(A.ks, false, lkA, s))) break;
    if ((err = build_offsets(B.ks, false, lkB, s))) break;
    GatherParams GA{}, GB{};
    GA.src = A.ptr; GA.lm = lmA; GA.lk = lkA; GA.rows = M; GA.K = K; GA.kpad = Kpad; GA.pstride = Mpad * Kpad;
    GA.planes = Ap; GA.rowE = rowE; GA.slices = S; GA.isign = A.conj ? -1.0 : 1.0;
    GA.lanes_on_k = (A.ks[0].s1 == 1 || A.rows.empty() || A.rows[0].s1 != 1) ? 1 : 0;
    if (resid) GA.rs = RP.rs;
    GB.src = B.ptr; GB.lm = lmB; GB.lk = lkB; GB.rows = Nc; GB.K = K; GB.kpad = Kpad; GB.pstride = Npad * Kpad;
    GB.planes = Bp; GB.rowE = colE; GB.slices = S; GB.isign = B.conj ? -1.0 : 1.0;
    GB.lanes_on_k = (B.ks[0].s1 == 1 || B.rows.empty() || B.rows[0].s1 != 1) ? 1 : 0;
    if (resid) GB.rs = RP.rs;
    const int tmr = i8 && cplx ? 32 : 64;               // gather tile rows (16-byte elements: 32)
    const int64_t gA = Mpad / tmr, gB = (cplx ? Npad / 2 : Npad) / tmr, gk = ksrc_pad / kGK;
    // row / column exponents and the lists of rows and columns flagged as
    // holding a NaN or an infinity (exponent field 2047): the epilogue leaves
    // their D entries to nonfinite_fixup_kernel
    if (cudaMemsetAsync(rowE, 0, offRX - offRE, s) != cudaSuccess) { err = TB_ERR_CUDA; break; }
    // nbad[0..1]: flagged row / column counts; nbad[2]: the GEMM's work-unit counter
    if (cudaMemsetAsync(nbad, 0, 4 * sizeof(int), s) != cudaSuccess) { err = TB_ERR_CUDA; break; }
    auto run_exps = [&]() -> int {
      exps_kernel<<<std::max<int64_t>(1, std::min<int64_t>((M + 255) / 256, 4096)), 256, 0, s>>>(rowE, rowx, M, 1,
                                                                                                 badrows, nbad);
      TB_CHECK_LAUNCH();
      exps_kernel<<<std::max<int64_t>(1, std::min<int64_t>((Nr + 255) / 256, 4096)), 256, 0, s>>>(
          colE, colx, Nr, cplx ? 2 : 1, badcols, nbad + 1);
      TB_CHECK_LAUNCH();
      return 0;
    };
    if (i8) {
      const int64_t eA = (M + tmr - 1) / tmr, eB = (Nc + tmr - 1) / tmr, ek = (K + kGK - 1) / kGK;
      if (!cplx) {
        if ((err = run_rowmax<false>(GA, eA, ek, s))) break;
        if ((err = run_rowmax<false>(GB, eB, ek, s))) break;
      } else {
        if ((err = run_rowmax<true>(GA, eA, ek, s))) break;
        if ((err = run_rowmax<true>(GB, eB, ek, s))) break;
      }
      if ((err = run_exps())) break;
      if (resid && !cplx) {
        if ((err = run_gather<G_RESID_R8>(GA, gA, gk, s))) break;
        if ((err = run_gather<G_RESID_R8>(GB, gB, gk, s))) break;
      } else if (resid) {
        if ((err = run_gather<G_RESID_C8A>(GA, gA, gk, s))) break;
        if ((err = run_gather<G_RESID_C8B>(GB, gB, gk, s))) break;
      } else if (!cplx) {
        if ((err = run_gather<G_SLICE_R8>(GA, gA, gk, s))) break;
        if ((err = run_gather<G_SLICE_R8>(GB, gB, gk, s))) break;
      } else {
        if ((err = run_gather<G_SLICE_C8A>(GA, gA, gk, s))) break;
        if ((err = run_gather<G_SLICE_C8B>(GB, gB, gk, s))) break;
      }
    } else {
      if (!cplx) {
        if ((err = run_gather<G_SPLIT_R4>(GA, gA, gk, s))) break;
        if ((err = run_gather<G_SPLIT_R4>(GB, gB, gk, s))) break;
      } else {
        if ((err = run_gather<G_SPLIT_C4A>(GA, gA, gk, s))) break;
        if ((err = run_gather<G_SPLIT_C4B>(GB, gB, gk, s))) break;
      }
      if ((err = run_exps())) break;  // the split gathers flag non-finite rows
    }
    // GEMM parameters
    // per call (about 2 KB), so that host threads contracting on different
    // streams never share a parameter block
    TcGemmParams P;
    std::memset(&P, 0, sizeof(P));
    if ((err = make_operand_map(&P.tmA, Ap, i8, Kpad, Mpad, npa, 128))) break;
    if ((err = make_operand_map(&P.tmB, Bp, i8, Kpad, Npad, npb, pair ? BN / 2 : BN))) break;
    P.M = (int)M; P.N = (int)Nr;
    P.mtiles = (int)(Mpad / TM); P.ntiles = (int)(Npad / BN);
    P.kblocks = (int)(Kpad * oes / 128);
    P.npass = (int)passes.size();
    P.res_nch = resid ? res_nch : 1;
    int q = 0;
    for (size_t p = 0; p < passes.size(); ++p) {
      P.pass_first[p] = q;
      P.pass_shift[p] = shifts[p];
      P.pass_magic[p] = resid ? (int)(4294967296ull / (unsigned long long)shifts[p]) : 0;
      for (auto& e : passes[p]) {
        P.prod_a[q] = e.a; P.prod_b[q] = e.b; P.prod_kb0[q] = e.kb0; P.prod_kb1[q] = e.kb1;
        ++q;
      }
    }
    P.pass_first[passes.size()] = q;
    P.D = d; P.dm = dm; P.dn = dn; P.rowexp = rowx; P.colexp = colx;
    const double realpha = cplx ? ar : (ar != 0.0 ? std::hypot(ar, ai) * (ar > 0 ? 1.0 : -1.0) : ai);
    P.ar = realpha; P.ai = cplx ? ai : 0.0;
    P.br = accumulate ? 1.0 : 0.0; P.bi = 0.0;
    P.err = device_error_word();
    P.nf_skip = resid ? 0 : 1;  // residues: crt_kernel leaves the flagged entries to the fix-up
    if (resid) {
      P.res = (uint8_t*)(ws + offRES);
      P.res_ld = Mpad;
      P.res_plane = Npad * Mpad;
    }
    // Work units: dynamic (a counter) unless TB_TC_SCHED=0.  L2 policy: with
    // residues every unit reads one modulus's planes, and all m-tiles re-read
    // that modulus's B plane -- when it fits in about three quarters of L2, B
    // is kept (evict-last) and A streamed (evict-first).  TB_TC_L2HINT=0 / 1
    // turns the policy off / on regardless.
    static const int sched_env = [] { const char* e = getenv("TB_TC_SCHED"); return e ? atoi(e) : 1; }();
    static const int hint_env = [] { const char* e = getenv("TB_TC_L2HINT"); return e ? atoi(e) : -1; }();
    P.sched = sched_env ? (unsigned*)(nbad + 2) : nullptr;
    const size_t bplane = (size_t)Npad * Kpad * oes;
    P.l2hint = hint_env >= 0 ? (hint_env ? 1 : 0) : (resid && bplane <= (size_t)96 << 20 ? 1 : 0);
    const int epi = resid ? EPI_RESID : i8 ? (cplx ? EPI_OZAKI_C : EPI_OZAKI_R) : (cplx ? EPI_BF16_C : EPI_BF16_R);
    const int ts = timed_begin(s);
    err = BN == 256 ? launch_tc_epi<256>(P, epi, pair, s) : launch_tc_epi<128>(P, epi, pair, s);
    timed_end(ts, s);
    if (err) break;
    if (resid) {
      // Chinese remainder reconstruction of the exact products into D
      CrtParams C = RP.crt;
      C.res = (const uint8_t*)(ws + offRES);
      C.res_ld = Mpad;
      C.res_plane = Npad * Mpad;
      C.rows = M;
      C.cols = Nc;
      C.dm = dm; C.dn = dn; C.D = d;
      C.rowexp = rowx; C.colexp = colx;
      C.ar = realpha; C.ai = cplx ? ai : 0.0; C.br = P.br; C.bi = 0.0;
      static DeviceOnce crt_attr_r, crt_attr_c;
      const cudaError_t ea = cplx ? smem_limit_once(crt_attr_c, crt_kernel<true>, kCrtTableBytes)
                                  : smem_limit_once(crt_attr_r, crt_kernel<false>, kCrtTableBytes);
      if (ea != cudaSuccess) { set_error("residue reconstruction smem attribute: %s", cudaGetErrorString(ea)); err = TB_ERR_CUDA; break; }
      const int64_t groups = Nc;  // column groups of crt_kernel (one D column each)
      const unsigned cg = (unsigned)std::max<int64_t>(1, std::min<int64_t>(groups, 3 * num_sms()));
      if (cplx) crt_kernel<true><<<cg, 256, kCrtTableBytes, s>>>(C);
      else crt_kernel<false><<<cg, 256, kCrtTableBytes, s>>>(C);
      count_launch();
      if (cudaError_t e = cudaGetLastError()) {
        set_error("residue reconstruction launch: %s", cudaGetErrorString(e));
        err = TB_ERR_CUDA;
        break;
      }
    }
    // entries of rows / columns with a NaN or an infinity (returns at once without)
    NfParams F;
    F.srcA = A.ptr; F.srcB = B.ptr;
    F.lmA = lmA; F.lkA = lkA; F.lmB = lmB; F.lkB = lkB;
    F.dm = dm; F.dn = dn; F.D = d;
    F.M = M; F.N = Nc; F.K = K;
    F.rowE = rowE; F.badrows = badrows; F.badcols = badcols; F.nbad = nbad;
    F.isignA = A.conj ? -1.0 : 1.0; F.isignB = B.conj ? -1.0 : 1.0;
    F.ar = realpha; F.ai = cplx ? ai : 0.0; F.br = P.br; F.bi = 0.0;
    const unsigned fgrid = (unsigned)(2 * num_sms());
    if (dtk == kR8) nonfinite_fixup_kernel<double, false><<<fgrid, 256, 0, s>>>(F);
    else if (dtk == kC8) nonfinite_fixup_kernel<double, true><<<fgrid, 256, 0, s>>>(F);
    else if (dtk == kR4) nonfinite_fixup_kernel<float, false><<<fgrid, 256, 0, s>>>(F);
    else nonfinite_fixup_kernel<float, true><<<fgrid, 256, 0, s>>>(F);
    count_launch();
    if (cudaError_t e = cudaGetLastError()) {
      set_error("non-finite fix-up launch: %s", cudaGetErrorString(e));
      err = TB_ERR_CUDA;
      break;
    }
    if (stats) {
      stats->slices = S;
      stats->passes = (int)passes.size();
      stats->products = nplane_products;
      stats->tile_n = BN;
      stats->tile_m = TM;
      stats->gemm_launches = 1;
      stats->m = M; stats->n = Nr; stats->k = Kr;
      stats->moduli = resid ? RP.rs.n : 0;
      stats->residue_bits = resid ? RP.p : 0;
    }
  } while (false);
  scratch_free(ws, s);
  return err;
}

}  // namespace tb
