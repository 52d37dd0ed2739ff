// ============================================================================
// talsh_oracle.cpp -- CPU restatement of TAL-SH's CP-TAL tensor-algebra path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
// baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// and reference legs may load it.  The product (exatensor_b200) never links or
// calls it.
//
// Parity pinning: the reference is Fortran (TALSH/tensor_algebra_cpu.F90) and
// cannot be compiled in this image (no Fortran compiler), so this restatement
// is pinned against the reference's own known-answer tests (closed-form values
// in TALSH/test.cpp and TALSH/main.F90, the explicit-loop check in
// TALSH/test.cpp:985-995, the digital pattern of TALSH/test.cpp:1094) and the
// 48-pattern corpus TALSH/tensor_contractions.txt; see tests/golden/.
//
// Arithmetic conventions mirrored from the reference build (gfortran -O3
// without -march, TALSH/Makefile FFLAGS_GNU_OPT): no fused multiply-add, so
// this file is compiled with -ffp-contract=off; complex products use the
// textbook formula (re = ar*br - ai*bi, im = ar*bi + ai*br).
//
// Layout: "dlf" (Fortran order, dimension 1 fastest), complex interleaved.
// Data kinds: R4=4, R8=8, C4=14, C8=18 (TALSH/tensor_algebra.h:67-72).
// ============================================================================
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <cmath>
#include <string>
#include <memory>
#include <vector>
#include <algorithm>
#include <dlfcn.h>
#include <omp.h>

namespace {

constexpr int R4 = 4, R8 = 8, C4 = 14, C8 = 18;
constexpr int MAXR = 56;

inline bool alnum_c(char c) {
  return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9');
}
inline bool alnum_us(char c) { return alnum_c(c) || c == '_'; }

template <typename T> struct cplx { T re, im; };

template <typename T> inline cplx<T> cmul(cplx<T> a, cplx<T> b) {
  cplx<T> r; r.re = a.re * b.re - a.im * b.im; r.im = a.re * b.im + a.im * b.re; return r;
}
template <typename T> inline cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> inline cplx<T> cconj(cplx<T> a) { return {a.re, -a.im}; }

int elem_size(int dtk) {
  switch (dtk) { case R4: return 4; case R8: return 8; case C4: return 8; case C8: return 16; }
  return 0;
}

// cmplx8_to_real8 (tensor_algebra_cpu.F90:430-445): modulus with the sign of
// the real part, or the imaginary part when the real part is zero.
double cmplx8_to_real8(double re, double im) {
  if (re != 0.0) return std::hypot(re, im) * (re > 0 ? 1.0 : -1.0);
  return im;
}

// Index-label check of get_contr_pattern_dig (tensor_algebra_cpu.F90:5503-5528):
// alphanumeric, optionally terminated by '+' (contravariant), non-empty.
bool label_ok(const std::string& lb, int& contra) {
  contra = 0;
  int n = (int)lb.size();
  if (n == 0) return false;
  for (int j = 0; j < n; ++j) {
    if (!alnum_c(lb[j])) {
      if (j < n - 1 || j == 0 || lb[j] != '+') return false;
      contra = 1;
    }
  }
  return true;
}

struct Occ { int arg; int pos; std::string label; bool active; };

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// get_contr_pattern_dig (tensor_algebra_cpu.F90:5307-5531): symbolic pattern
// -> digital pattern cptrn[lrank+rrank] (value >0: destination position,
// value <0: minus the partner position in the other input).  Conjugation bits:
// bit0 D, bit1 L, bit2 R, set by a '+' right after the tensor name.
// Returns the reference's error code (0 = success).
// ---------------------------------------------------------------------------
int orc_parse_pattern(const char* cptrn_str, int* cptrn, int* drank, int* lrank,
                      int* rrank, int* conj_bits) {
  std::string s(cptrn_str ? cptrn_str : "");
  while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();  // len_trim
  const int l = (int)s.size();
  *drank = -1; *lrank = -1; *rrank = -1;
  int conj = 0;
  if (conj_bits) *conj_bits = 0;
  if (l == 0) return 16;
  auto ch = [&](int p1) { return s[p1 - 1]; };  // 1-based access, as in the Fortran
  std::vector<Occ> occ;
  int adims[3] = {0, 0, 0};
  int n = -1, ks = 0, i = 1;
  while (i <= l) {
    bool found = false;
    while (i <= l) { if (ch(i) == '(') { found = true; break; } ++i; }
    if (!found) break;
    if (i > 2) {
      if (ch(i - 1) == '+' && alnum_us(ch(i - 2))) conj += (1 << (n + 1));
    }
    ks = i; ++i; ++n;
    int k = 1;
    if (n > 2) return 1;
    while (i <= l) {
      char c = ch(i);
      if (c == ',' || c == '|') {
        int a = std::abs(ks);
        std::string lb = s.substr(a, i - 1 - a);
        int cv;
        if (!label_ok(lb, cv)) return 2;
        occ.push_back({n, k, lb.substr(0, lb.size() - cv), true});
        ks = -i; ++k;
      } else if (c == ')') {
        int a = std::abs(ks);
        int j = i - 1 - a;
        if (j <= 0) {
          if (ks < 0) return 3;
        } else {
          std::string lb = s.substr(a, j);
          int cv;
          if (!label_ok(lb, cv)) return 4;
          occ.push_back({n, k, lb.substr(0, lb.size() - cv), true});
          ++k;
        }
        ks = 0; ++i; break;
      }
      ++i;
    }
    if (ks != 0) return 5;
    adims[n] = k - 1;
  }
  if (ks != 0) return 6;
  const int nocc = (int)occ.size();
  auto next_active = [&](int from, const std::string& lb) {
    for (int v = from + 1; v < nocc; ++v) if (occ[v].active && occ[v].label == lb) return v;
    return -1;
  };
  if (n == 2) {
    *drank = adims[0]; *lrank = adims[1]; *rrank = adims[2];
    for (int u = 0; u < nocc; ++u) {
      if (!occ[u].active) continue;
      if (u == nocc - 1) return 7;  // an active label in the last slot has no partner
      const int k1 = occ[u].arg, k2 = occ[u].pos;
      for (int kf = 1; kf <= 2; ++kf) {
        int v = next_active(u, occ[u].label);
        if (v >= 0) {
          const int k3 = occ[v].arg, k4 = occ[v].pos;
          if (k1 == 0 && k3 == 1) {
            if (kf != 1) return 8;
            cptrn[k4 - 1] = k2;
          } else if (k1 == 0 && k3 == 2) {
            cptrn[*lrank + k4 - 1] = k2;
          } else if (k1 == 1 && k3 == 2) {
            if (kf != 1) return 9;
            cptrn[k2 - 1] = -k4; cptrn[*lrank + k4 - 1] = -k2;
          } else {
            return 10;
          }
          occ[v].active = false;
        } else {
          if (kf == 1) return 11;
        }
      }
      occ[u].active = false;
    }
  } else if (n == 1) {
    *drank = adims[0]; *lrank = adims[1];
    for (int u = 0; u < nocc; ++u) {
      if (!occ[u].active) continue;
      if (u == nocc - 1) return 12;
      const int k1 = occ[u].arg, k2 = occ[u].pos;
      int v = next_active(u, occ[u].label);
      if (v >= 0) {
        const int k3 = occ[v].arg, k4 = occ[v].pos;
        if (k1 == 0 && k3 == 1) cptrn[k4 - 1] = k2; else return 13;
        occ[v].active = false;
      } else {
        return 14;
      }
      occ[u].active = false;
    }
  } else {
    return 15;
  }
  if (conj_bits) *conj_bits = conj;
  return 0;
}

// ---------------------------------------------------------------------------
// get_contr_permutations (tensor_algebra_cpu.F90:5613-5755).  Outputs are
// 1-based, entry 0 is the permutation sign, as in the reference:
// dprm (N2O) for the destination, lprm/rprm (O2N) for the inputs.
// ---------------------------------------------------------------------------
static bool contr_pattern_ok(int lrank, int rrank, const int* cptrn) {
  int jl = lrank + rrank;
  if (jl <= 0) return true;
  std::vector<int> jkey(jl + 1, 0);
  int jc = 0;
  for (int j0 = 1; j0 <= jl; ++j0) {
    int j1 = cptrn[j0 - 1];
    if (j1 < 0) {
      if (j0 <= lrank) {
        if (-j1 > rrank) return false;
        if (cptrn[lrank + (-j1) - 1] != -j0) return false;
      } else {
        if (-j1 > lrank) return false;
        if (cptrn[(-j1) - 1] != -(j0 - lrank)) return false;
      }
    } else if (j1 > 0 && j1 <= jl) {
      ++jc;
      if (jkey[j1] == 0) jkey[j1] = 1; else return false;
    } else {
      return false;
    }
  }
  for (int j0 = 1; j0 <= jc; ++j0) if (jkey[j0] != 1) return false;
  return true;
}

int orc_contr_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank, const int* cptrn,
                           int conj_bits, int* dprm, int* lprm, int* rprm, int* ncd, int* nlu,
                           int* nru) {
  if (!(contr_pattern_ok(lrank, rrank, cptrn) && lrank >= 0 && rrank >= 0)) return 1;
  bool left_conj = (conj_bits >> 1) & 1, right_conj = (conj_bits >> 2) & 1;
  if (conj_bits & 1) { left_conj = !left_conj; right_conj = !right_conj; }
  if (gemm_tl == 0 && left_conj) return 2;
  int drank = 0; dprm[0] = 1;
  for (int i = 1; i <= lrank; ++i) if (cptrn[i - 1] > 0) { ++drank; dprm[drank] = cptrn[i - 1]; }
  *nlu = drank;
  bool simple = (drank >= 2);
  for (int i = lrank + 1; i <= lrank + rrank; ++i) {
    if (cptrn[i - 1] > 0) {
      ++drank; dprm[drank] = cptrn[i - 1];
      if (cptrn[i - 1] <= *nlu) simple = false;
    }
  }
  if (simple) for (int j = 1; j <= drank; ++j) dprm[j] = j;
  rprm[0] = 1; *nru = 0; *ncd = 0;
  int j = 0;
  if (rrank > 0) {
    for (int i = 1; i <= rrank; ++i) if (cptrn[lrank + i - 1] < 0) { ++j; rprm[i] = j; }
    *ncd = j;
    *nru = rrank - *ncd;
    if (simple && *nru >= 2) {
      for (int i = 1; i <= rrank; ++i)
        if (cptrn[lrank + i - 1] > 0) rprm[i] = *ncd + (cptrn[lrank + i - 1] - *nlu);
    } else {
      for (int i = 1; i <= rrank; ++i) if (cptrn[lrank + i - 1] > 0) { ++j; rprm[i] = j; }
    }
  }
  lprm[0] = 1;
  if (lrank > 0) {
    // contracted dimensions of L are ordered like their partners in R
    // (the reference sorts them with merge_sort_key_int; the keys are distinct)
    std::vector<std::pair<int, int>> keyed;  // (partner position in R, L position)
    for (int i = 1; i <= lrank; ++i) if (cptrn[i - 1] < 0) keyed.push_back({-cptrn[i - 1], i});
    std::sort(keyed.begin(), keyed.end());
    int jj = 0;
    for (auto& kv : keyed) lprm[kv.second] = ++jj;
    j = jj;
    if (simple && *nlu >= 2) {
      for (int i = 1; i <= lrank; ++i) if (cptrn[i - 1] > 0) lprm[i] = *ncd + cptrn[i - 1];
    } else {
      for (int i = 1; i <= lrank; ++i) if (cptrn[i - 1] > 0) { ++j; lprm[i] = j; }
    }
  }
  if (gemm_tl == 0) {
    for (int i = 1; i <= lrank; ++i) lprm[i] = (lprm[i] <= *ncd) ? lprm[i] + *nlu : lprm[i] - *ncd;
  }
  if (gemm_tr != 0 || right_conj) {
    for (int i = 1; i <= rrank; ++i) rprm[i] = (rprm[i] <= *ncd) ? rprm[i] + *nru : rprm[i] - *ncd;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Permutation (tensor_block_copy, tensor_algebra_cpu.F90:3151-3310, and the
// dlf kernels :7453-8502): out(y) = in(x) with y(o2n(i)) = x(i); o2n 1-based.
// Complex data is conjugated when conj != 0.  Exact copy.
// ---------------------------------------------------------------------------
}  // extern "C"

template <typename T>
static void permute_t(int rank, const int* dims, const int* o2n, const T* in, T* out,
                      bool conj_c, int nthreads) {
  int64_t vol = 1;
  for (int i = 0; i < rank; ++i) vol *= dims[i];
  if (rank == 0) { out[0] = in[0]; return; }
  int64_t bout[MAXR];
  {
    int n2o[MAXR + 1];
    for (int i = 1; i <= rank; ++i) n2o[o2n[i - 1]] = i;
    int64_t bs = 1;
    int64_t bpos[MAXR + 1];
    for (int p = 1; p <= rank; ++p) { bpos[p] = bs; bs *= dims[n2o[p] - 1]; }
    for (int i = 1; i <= rank; ++i) bout[i - 1] = bpos[o2n[i - 1]];
  }
  // Outer loop over input dims 1..rank-1 grouped into chunks of dim 0.
  const int64_t d0 = dims[0];
  const int64_t rows = vol / d0;
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int64_t row = 0; row < rows; ++row) {
    int64_t r = row, ooff = 0;
    for (int i = 1; i < rank; ++i) { int64_t x = r % dims[i]; r /= dims[i]; ooff += x * bout[i]; }
    const T* src = in + row * d0;
    const int64_t s0 = bout[0];
    for (int64_t x0 = 0; x0 < d0; ++x0) {
      T v = src[x0];
      if (conj_c) {
        // complex stored as two scalars; T here is a 2-scalar struct
        v.im = -v.im;
      }
      out[ooff + x0 * s0] = v;
    }
  }
}

struct c4e { float re; float im; };
struct c8e { double re; double im; };

// Real element types: identical loop, no conjugation.
template <typename T>
static void permute_real(int rank, const int* dims, const int* o2n, const T* src, T* dst, int nthreads) {
  if (rank == 0) { dst[0] = src[0]; return; }
  int n2o[MAXR + 1]; int64_t bpos[MAXR + 1], bout[MAXR];
  for (int i = 1; i <= rank; ++i) n2o[o2n[i - 1]] = i;
  int64_t bs = 1;
  for (int p = 1; p <= rank; ++p) { bpos[p] = bs; bs *= dims[n2o[p] - 1]; }
  for (int i = 1; i <= rank; ++i) bout[i - 1] = bpos[o2n[i - 1]];
  const int64_t d0 = dims[0], rows = bs / d0;
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int64_t row = 0; row < rows; ++row) {
    int64_t r = row, ooff = 0;
    for (int i = 1; i < rank; ++i) { int64_t x = r % dims[i]; r /= dims[i]; ooff += x * bout[i]; }
    for (int64_t x0 = 0; x0 < d0; ++x0) dst[ooff + x0 * bout[0]] = src[row * d0 + x0];
  }
}

extern "C" {

int orc_permute(int dtk, int rank, const int* dims, const int* o2n, const void* in, void* out,
                           int conj, int nthreads) {
  if (nthreads <= 0) nthreads = 1;
  switch (dtk) {
    case R4: permute_real<float>(rank, dims, o2n, (const float*)in, (float*)out, nthreads); return 0;
    case R8: permute_real<double>(rank, dims, o2n, (const double*)in, (double*)out, nthreads); return 0;
    case C4: permute_t<c4e>(rank, dims, o2n, (const c4e*)in, (c4e*)out, conj != 0, nthreads); return 0;
    case C8: permute_t<c8e>(rank, dims, o2n, (const c8e*)in, (c8e*)out, conj != 0, nthreads); return 0;
  }
  return 1;
}

// ---------------------------------------------------------------------------
// Elementwise add (tensor_block_add, tensor_algebra_cpu.F90:3312-3673) as the
// C API reaches it (cpu_tensor_block_add, talshf.F90:1857-1903, always passes
// the scale factor): accumulate d = d + l*a, overwrite d = l*a.  R4 takes
// a = real(cmplx8_to_real8(scale), 4); C4 takes a = cmplx(scale, kind=4).
// conj_bits: bit0 D, bit1 L; a conjugated D flips the conjugation of L.
// ---------------------------------------------------------------------------
int orc_add(int dtk, int64_t vol, void* d, const void* l, double sr, double si, int conj_bits,
            int accumulative, int nthreads) {
  if (nthreads <= 0) nthreads = 1;
  bool dconj = conj_bits & 1, lconj = (conj_bits >> 1) & 1;
  if (dconj) lconj = !lconj;
  switch (dtk) {
    case R4: {
      float a = (float)cmplx8_to_real8(sr, si);
      float* D = (float*)d; const float* L = (const float*)l;
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int64_t i = 0; i < vol; ++i) { float t = L[i] * a; D[i] = accumulative ? D[i] + t : t; }
      return 0;
    }
    case R8: {
      double a = cmplx8_to_real8(sr, si);
      double* D = (double*)d; const double* L = (const double*)l;
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int64_t i = 0; i < vol; ++i) { double t = L[i] * a; D[i] = accumulative ? D[i] + t : t; }
      return 0;
    }
    case C4: {
      cplx<float> a{(float)sr, (float)si};
      cplx<float>* D = (cplx<float>*)d; const cplx<float>* L = (const cplx<float>*)l;
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int64_t i = 0; i < vol; ++i) {
        cplx<float> x = lconj ? cconj(L[i]) : L[i];
        cplx<float> t = cmul(x, a);
        D[i] = accumulative ? cadd(D[i], t) : t;
      }
      return 0;
    }
    case C8: {
      cplx<double> a{sr, si};
      cplx<double>* D = (cplx<double>*)d; const cplx<double>* L = (const cplx<double>*)l;
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int64_t i = 0; i < vol; ++i) {
        cplx<double> x = lconj ? cconj(L[i]) : L[i];
        cplx<double> t = cmul(x, a);
        D[i] = accumulative ? cadd(D[i], t) : t;
      }
      return 0;
    }
  }
  return 1;
}

// cpu_tensor_block_add (talshf.F90:1857-1903): permute L by the digital
// pattern (O2N) into a temporary when it is not the identity, then add.
int orc_tensor_add(const int* cptrn, int dtk, int rank, const int* ldims, void* d, const void* l,
                   double sr, double si, int conj_bits, int nthreads) {
  int64_t vol = 1;
  for (int i = 0; i < rank; ++i) vol *= ldims[i];
  bool permute = false;
  for (int i = 0; i < rank; ++i) if (cptrn[i] != i + 1) { permute = true; break; }
  if (!permute) return orc_add(dtk, vol, d, l, sr, si, conj_bits, 1, nthreads);
  std::vector<char> tmp((size_t)vol * elem_size(dtk));
  int e = orc_permute(dtk, rank, ldims, cptrn, l, tmp.data(), 0, nthreads);
  if (e) return e;
  return orc_add(dtk, vol, d, tmp.data(), sr, si, conj_bits, 1, nthreads);
}

// tensor_block_scale (tensor_algebra_cpu.F90:1821-1890): d = d*a.
int orc_scale(int dtk, int64_t vol, void* d, double sr, double si) {
  switch (dtk) {
    case R4: {
      const float a = (float)cmplx8_to_real8(sr, si);
      float* D = (float*)d;
      for (int64_t i = 0; i < vol; ++i) D[i] = D[i] * a;
      return 0;
    }
    case R8: {
      const double a = cmplx8_to_real8(sr, si);
      double* D = (double*)d;
      for (int64_t i = 0; i < vol; ++i) D[i] = D[i] * a;
      return 0;
    }
    case C4: {
      const cplx<float> a{(float)sr, (float)si};
      cplx<float>* D = (cplx<float>*)d;
      for (int64_t i = 0; i < vol; ++i) D[i] = cmul(D[i], a);
      return 0;
    }
    case C8: {
      const cplx<double> a{sr, si};
      cplx<double>* D = (cplx<double>*)d;
      for (int64_t i = 0; i < vol; ++i) D[i] = cmul(D[i], a);
      return 0;
    }
  }
  return 1;
}

// tensor_block_init (tensor_algebra_cpu.F90:955-1395): d = val.
int orc_init(int dtk, int64_t vol, void* d, double vr, double vi) {
  switch (dtk) {
    case R4: {
      float* D = (float*)d;
      const float v = (float)vr;
      for (int64_t i = 0; i < vol; ++i) D[i] = v;
      return 0;
    }
    case R8: {
      double* D = (double*)d;
      for (int64_t i = 0; i < vol; ++i) D[i] = vr;
      return 0;
    }
    case C4: {
      cplx<float>* D = (cplx<float>*)d;
      const cplx<float> v{(float)vr, (float)vi};
      for (int64_t i = 0; i < vol; ++i) D[i] = v;
      return 0;
    }
    case C8: {
      cplx<double>* D = (cplx<double>*)d;
      const cplx<double> v{vr, vi};
      for (int64_t i = 0; i < vol; ++i) D[i] = v;
      return 0;
    }
  }
  return 1;
}

// Norms (tensor_block_norm1/norm2, tensor_algebra_cpu.F90:1933-2129), summed
// in double here (the reference's OpenMP reduction order is unspecified).
// which: 1 -> sum |x| (complex modulus), 2 -> sum |x|^2.
double orc_norm(int dtk, int64_t vol, const void* d, int which) {
  double s = 0.0;
  for (int64_t i = 0; i < vol; ++i) {
    double re = 0, im = 0;
    switch (dtk) {
      case R4: re = ((const float*)d)[i]; break;
      case R8: re = ((const double*)d)[i]; break;
      case C4: re = ((const float*)d)[2 * i]; im = ((const float*)d)[2 * i + 1]; break;
      case C8: re = ((const double*)d)[2 * i]; im = ((const double*)d)[2 * i + 1]; break;
    }
    s += (which == 1) ? std::hypot(re, im) : re * re + im * im;
  }
  return s;
}

}  // extern "C"

// ===========================================================================
// Contraction (tensor_block_contract, tensor_algebra_cpu.F90:3675-4294):
// D = beta*D + alpha * op(L) * op(R) with beta = 1 (accumulative) or 0,
// op = conjugation per conj_bits (bit0 D flips L and R), executed as TTGT:
// permute L to (contracted, uncontracted) = K x M, R to K x N, C = L^T R
// (the reference's GEMM('T','N'), :4005), then scatter C into D.
// ===========================================================================
namespace {

struct Matricization {
  int drank, lrank, rrank;
  int64_t M, N, K;
  std::vector<int64_t> lm, lk, rn, rk, dm, dn;  // element offsets per row/col index
};

// Builds offset tables: element (m,k) of op(L)^T lives at L[lm[m] + lk[k]],
// (k,n) of R at R[rk[k] + rn[n]], (m,n) of C at D[dm[m] + dn[n]].
// m enumerates L's uncontracted dims (L order, first fastest), n enumerates
// R's uncontracted dims (R order), k enumerates contracted dims in R's order.
bool matricize(const int* cptrn, int drank, const int* ddims, int lrank, const int* ldims,
               int rrank, const int* rdims, Matricization& mz) {
  mz.drank = drank; mz.lrank = lrank; mz.rrank = rrank;
  int64_t lb[MAXR], rb[MAXR], db[MAXR];
  int64_t s = 1; for (int i = 0; i < lrank; ++i) { lb[i] = s; s *= ldims[i]; }
  s = 1; for (int i = 0; i < rrank; ++i) { rb[i] = s; s *= rdims[i]; }
  s = 1; for (int i = 0; i < drank; ++i) { db[i] = s; s *= ddims[i]; }
  std::vector<int> mdims, ndims, kdims;        // extents
  std::vector<int64_t> mls, mds, nrs, nds, krs, kls;  // strides
  for (int i = 0; i < lrank; ++i) {
    int c = cptrn[i];
    if (c > 0) {
      if (c > drank || ddims[c - 1] != ldims[i]) return false;
      mdims.push_back(ldims[i]); mls.push_back(lb[i]); mds.push_back(db[c - 1]);
    }
  }
  for (int i = 0; i < rrank; ++i) {
    int c = cptrn[lrank + i];
    if (c > 0) {
      if (c > drank || ddims[c - 1] != rdims[i]) return false;
      ndims.push_back(rdims[i]); nrs.push_back(rb[i]); nds.push_back(db[c - 1]);
    } else {
      int lp = -c;
      if (lp < 1 || lp > lrank || ldims[lp - 1] != rdims[i]) return false;
      kdims.push_back(rdims[i]); krs.push_back(rb[i]); kls.push_back(lb[lp - 1]);
    }
  }
  auto table = [](const std::vector<int>& ext, const std::vector<int64_t>& st, std::vector<int64_t>& out) {
    int64_t v = 1; for (int e : ext) v *= e;
    out.assign(v, 0);
    for (int64_t idx = 0; idx < v; ++idx) {
      int64_t r = idx, off = 0;
      for (size_t j = 0; j < ext.size(); ++j) { int64_t x = r % ext[j]; r /= ext[j]; off += x * st[j]; }
      out[idx] = off;
    }
    return v;
  };
  mz.M = table(mdims, mls, mz.lm); table(mdims, mds, mz.dm);
  mz.N = table(ndims, nrs, mz.rn); table(ndims, nds, mz.dn);
  mz.K = table(kdims, krs, mz.rk); table(kdims, kls, mz.lk);
  return true;
}

// Double-double helpers (Dekker/Knuth error-free transformations).
struct dd { double hi, lo; };
inline dd two_sum(double a, double b) { double s = a + b; double bb = s - a; double e = (a - (s - bb)) + (b - bb); return {s, e}; }
inline dd two_prod(double a, double b) { double p = a * b; double e = std::fma(a, b, -p); return {p, e}; }
inline dd dd_add(dd a, dd b) { dd s = two_sum(a.hi, b.hi); double e = s.lo + a.lo + b.lo; return two_sum(s.hi, e); }
inline dd dd_mul_d(dd a, double b) { dd p = two_prod(a.hi, b); p.lo += a.lo * b; return two_sum(p.hi, p.lo); }

template <typename R>
int contract_real(const Matricization& mz, R* D, const R* L, const R* Rt, double alpha,
                  int accumulative, int mode, int nthreads) {
  // mode 0: sums in the data type, k in order (the oracle's GEMM);
  // mode 1: double-double sums, result rounded once (the FP64 error oracle).
  const R a = (R)alpha;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t n = 0; n < mz.N; ++n) {
    for (int64_t m = 0; m < mz.M; ++m) {
      const int64_t doff = mz.dm[m] + mz.dn[n];
      if (mode == 0) {
        R acc = 0;
        for (int64_t k = 0; k < mz.K; ++k) acc = acc + L[mz.lm[m] + mz.lk[k]] * Rt[mz.rk[k] + mz.rn[n]];
        D[doff] = accumulative ? (R)(a * acc + D[doff]) : (R)(a * acc);
      } else {
        dd acc{0.0, 0.0};
        for (int64_t k = 0; k < mz.K; ++k)
          acc = dd_add(acc, two_prod((double)L[mz.lm[m] + mz.lk[k]], (double)Rt[mz.rk[k] + mz.rn[n]]));
        dd r = dd_mul_d(acc, alpha);
        if (accumulative) r = dd_add(r, dd{(double)D[doff], 0.0});
        D[doff] = (R)(r.hi + r.lo);
      }
    }
  }
  return 0;
}

template <typename R>
int contract_cplx(const Matricization& mz, R* D, const R* L, const R* Rt, double ar, double ai,
                  bool lconj, bool rconj, int accumulative, int mode, int nthreads) {
  const cplx<R> a{(R)ar, (R)ai};
  const cplx<R>* Lc = (const cplx<R>*)L;
  const cplx<R>* Rc = (const cplx<R>*)Rt;
  cplx<R>* Dc = (cplx<R>*)D;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t n = 0; n < mz.N; ++n) {
    for (int64_t m = 0; m < mz.M; ++m) {
      const int64_t doff = mz.dm[m] + mz.dn[n];
      if (mode == 0) {
        cplx<R> acc{0, 0};
        for (int64_t k = 0; k < mz.K; ++k) {
          cplx<R> x = Lc[mz.lm[m] + mz.lk[k]], y = Rc[mz.rk[k] + mz.rn[n]];
          if (lconj) x = cconj(x);
          if (rconj) y = cconj(y);
          acc = cadd(acc, cmul(x, y));
        }
        cplx<R> t = cmul(a, acc);
        Dc[doff] = accumulative ? cadd(t, Dc[doff]) : t;
      } else {
        dd sr{0, 0}, si{0, 0};
        for (int64_t k = 0; k < mz.K; ++k) {
          cplx<R> x = Lc[mz.lm[m] + mz.lk[k]], y = Rc[mz.rk[k] + mz.rn[n]];
          double xr = x.re, xi = lconj ? -(double)x.im : (double)x.im;
          double yr = y.re, yi = rconj ? -(double)y.im : (double)y.im;
          sr = dd_add(sr, two_prod(xr, yr)); sr = dd_add(sr, two_prod(-xi, yi));
          si = dd_add(si, two_prod(xr, yi)); si = dd_add(si, two_prod(xi, yr));
        }
        dd rr = dd_add(dd_mul_d(sr, ar), dd_mul_d(si, -ai));
        dd ri = dd_add(dd_mul_d(si, ar), dd_mul_d(sr, ai));
        if (accumulative) { rr = dd_add(rr, dd{(double)Dc[doff].re, 0}); ri = dd_add(ri, dd{(double)Dc[doff].im, 0}); }
        Dc[doff] = cplx<R>{(R)(rr.hi + rr.lo), (R)(ri.hi + ri.lo)};
      }
    }
  }
  return 0;
}

}  // namespace

extern "C" {

// mode 0: the oracle's own TTGT-order GEMM in the tensor's data type;
// mode 1: double-double accumulation, rounded once (the FP64 error oracle).
int orc_contract(const int* cptrn, int dtk, int drank, const int* ddims, void* d, int lrank,
                 const int* ldims, const void* l, int rrank, const int* rdims, const void* r,
                 double ar, double ai, int conj_bits, int accumulative, int mode, int nthreads) {
  if (nthreads <= 0) nthreads = 1;
  Matricization mz;
  if (!matricize(cptrn, drank, ddims, lrank, ldims, rrank, rdims, mz)) return 8;
  bool dconj = conj_bits & 1, lconj = (conj_bits >> 1) & 1, rconj = (conj_bits >> 2) & 1;
  if (dconj) { lconj = !lconj; rconj = !rconj; }
  switch (dtk) {
    case R4: return contract_real<float>(mz, (float*)d, (const float*)l, (const float*)r,
                                         cmplx8_to_real8(ar, ai), accumulative, mode, nthreads);
    case R8: return contract_real<double>(mz, (double*)d, (const double*)l, (const double*)r,
                                          cmplx8_to_real8(ar, ai), accumulative, mode, nthreads);
    case C4: return contract_cplx<float>(mz, (float*)d, (const float*)l, (const float*)r, ar, ai,
                                         lconj, rconj, accumulative, mode, nthreads);
    case C8: return contract_cplx<double>(mz, (double*)d, (const double*)l, (const double*)r, ar, ai,
                                          lconj, rconj, accumulative, mode, nthreads);
  }
  return 6;
}

// ---------------------------------------------------------------------------
// CPU baseline: the reference's OpenMP + BLAS CP-TAL contraction path
// (tensor_block_contract :3675-4163: permute L, R (and D) with the
// cache-efficient OpenMP transposes, then ?gemm('T','N'), then permute D back)
// using the OpenBLAS bundled with scipy through dlopen.  Real data kinds.
// ---------------------------------------------------------------------------
typedef void (*dgemm_t)(const char*, const char*, const int*, const int*, const int*, const double*,
                        const double*, const int*, const double*, const int*, const double*, double*,
                        const int*, size_t, size_t);
typedef void (*sgemm_t)(const char*, const char*, const int*, const int*, const int*, const float*,
                        const float*, const int*, const float*, const int*, const float*, float*,
                        const int*, size_t, size_t);
typedef void (*setthr_t)(int);
static void* g_blas = nullptr;
static dgemm_t g_dgemm = nullptr;
static sgemm_t g_sgemm = nullptr;
static setthr_t g_setthr = nullptr;

int orc_blas_load(const char* path) {
  if (g_blas) return 0;
  g_blas = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!g_blas) return 1;
  g_dgemm = (dgemm_t)dlsym(g_blas, "scipy_dgemm_");
  g_sgemm = (sgemm_t)dlsym(g_blas, "scipy_sgemm_");
  g_setthr = (setthr_t)dlsym(g_blas, "scipy_openblas_set_num_threads");
  return (g_dgemm && g_sgemm) ? 0 : 2;
}

int orc_permute_blocked(int dtk, int rank, const int* dims, const int* o2n, const void* in, void* out,
                        int nthreads);

int orc_contract_blas(const int* cptrn, int dtk, int drank, const int* ddims, void* d, int lrank,
                      const int* ldims, const void* l, int rrank, const int* rdims, const void* r,
                      double ar, double ai, int accumulative, int nthreads) {
  if (!g_dgemm) return 100;
  if (dtk != R8 && dtk != R4) return 101;
  if (g_setthr) g_setthr(nthreads);
  int dprm[MAXR + 1], lprm[MAXR + 1], rprm[MAXR + 1], ncd, nlu, nru;
  int e = orc_contr_permutations(1, 0, lrank, rrank, cptrn, 0, dprm, lprm, rprm, &ncd, &nlu, &nru);
  if (e) return e;
  const size_t es = elem_size(dtk);
  int64_t K = 1, M = 1, N = 1;
  std::vector<int> lt(lrank), rt(rrank);
  for (int i = 0; i < lrank; ++i) lt[lprm[i + 1] - 1] = ldims[i];
  for (int i = 0; i < rrank; ++i) rt[rprm[i + 1] - 1] = rdims[i];
  for (int i = 0; i < ncd; ++i) K *= rt[i];
  for (int i = ncd; i < lrank; ++i) M *= lt[i];
  for (int i = ncd; i < rrank; ++i) N *= rt[i];
  // temporaries are not initialised (like the reference's allocate); the
  // permutations are the cache-blocked OpenMP transposes of
  // tensor_block_copy_dlf_r8 (tensor_algebra_cpu.F90:7764-7834)
  std::unique_ptr<char[]> Ltb(new char[M * K * es]), Rtb(new char[K * N * es]), Ctb(new char[M * N * es]);
  char *Lt = Ltb.get(), *Rt = Rtb.get(), *Ct = Ctb.get();
  orc_permute_blocked(dtk, lrank, ldims, lprm + 1, l, Lt, nthreads);
  orc_permute_blocked(dtk, rrank, rdims, rprm + 1, r, Rt, nthreads);
  // C dims are (L-uncontracted, R-uncontracted); C dim j maps to D dim dprm[j].
  std::vector<int> cdims(drank), c2d(drank);
  for (int j = 0; j < drank; ++j) { cdims[j] = ddims[dprm[j + 1] - 1]; c2d[j] = dprm[j + 1]; }
  bool dtr = false;
  for (int j = 0; j < drank; ++j) if (c2d[j] != j + 1) dtr = true;
  if (accumulative) {
    if (dtr) {
      std::vector<int> d2c(drank);
      for (int j = 0; j < drank; ++j) d2c[c2d[j] - 1] = j + 1;
      orc_permute_blocked(dtk, drank, ddims, d2c.data(), d, Ct, nthreads);
    } else {
      std::memcpy(Ct, d, M * N * es);
    }
  }
  int m = (int)M, n = (int)N, k = (int)K;
  if (dtk == R8) {
    double a = cmplx8_to_real8(ar, ai), b = accumulative ? 1.0 : 0.0;
    g_dgemm("T", "N", &m, &n, &k, &a, (const double*)Lt, &k, (const double*)Rt, &k, &b, (double*)Ct, &m, 1, 1);
  } else {
    float a = (float)cmplx8_to_real8(ar, ai), b = accumulative ? 1.0f : 0.0f;
    g_sgemm("T", "N", &m, &n, &k, &a, (const float*)Lt, &k, (const float*)Rt, &k, &b, (float*)Ct, &m, 1, 1);
  }
  if (dtr) orc_permute_blocked(dtk, drank, cdims.data(), c2d.data(), Ct, d, nthreads);
  else std::memcpy(d, Ct, M * N * es);
  return 0;
}

// Cache-blocked OpenMP permutation used as the timed CPU baseline
// (tensor_block_copy_dlf_r8, tensor_algebra_cpu.F90:7699-7940): the tensor is
// traversed in blocks spanning the input-minor and output-minor dimensions so
// both sides stay in cache, with the outer volume split across threads.
int orc_permute_blocked(int dtk, int rank, const int* dims, const int* o2n, const void* in,
                        void* out, int nthreads) {
  const int es = elem_size(dtk);
  if (rank <= 1) { int64_t v = rank ? dims[0] : 1; std::memcpy(out, in, v * es); return 0; }
  int n2o[MAXR + 1]; int64_t bpos[MAXR + 1], bout[MAXR], bin[MAXR];
  for (int i = 1; i <= rank; ++i) n2o[o2n[i - 1]] = i;
  int64_t bs = 1;
  for (int p = 1; p <= rank; ++p) { bpos[p] = bs; bs *= dims[n2o[p] - 1]; }
  for (int i = 1; i <= rank; ++i) bout[i - 1] = bpos[o2n[i - 1]];
  bs = 1; for (int i = 0; i < rank; ++i) { bin[i] = bs; bs *= dims[i]; }
  const int q = n2o[1] - 1;  // input dim that becomes output-fastest
  if (q == 0) return orc_permute(dtk, rank, dims, o2n, in, out, 0, nthreads);
  const int64_t B = 32;  // block of the two minor dimensions
  const int64_t d0 = dims[0], dq = dims[q];
  const int64_t outer = bs / (d0 * dq);
  const char* src = (const char*)in; char* dst = (char*)out;
#pragma omp parallel for schedule(static) collapse(2) num_threads(nthreads)
  for (int64_t o = 0; o < outer; ++o) {
    for (int64_t bq = 0; bq < (dq + B - 1) / B; ++bq) {
      int64_t r = o, ioff = 0, ooff = 0;
      for (int i = 1; i < rank; ++i) {
        if (i == q) continue;
        int64_t x = r % dims[i]; r /= dims[i]; ioff += x * bin[i]; ooff += x * bout[i];
      }
      for (int64_t b0 = 0; b0 < d0; b0 += B) {
        for (int64_t xq = bq * B; xq < std::min(dq, bq * B + B); ++xq) {
          const int64_t io = ioff + xq * bin[q], oo = ooff + xq * bout[q];
          for (int64_t x0 = b0; x0 < std::min(d0, b0 + B); ++x0)
            std::memcpy(dst + (oo + x0 * bout[0]) * es, src + (io + x0) * es, es);
        }
      }
    }
  }
  return 0;
}

int orc_elem_size(int dtk) { return elem_size(dtk); }

// Seeded U[lo,hi) doubles in parallel: the splitmix64 stream of
// splitmix64_uniform (oracle/__init__.py) and tb_fill_uniform, value i from
// state seed + (i+1) * golden gamma, 53-bit fraction; same bits.
void orc_fill_uniform(int64_t n, uint64_t seed, double lo, double hi, double* out, int nthreads) {
  if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int64_t i = 0; i < n; ++i) {
    uint64_t z = seed + (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    out[i] = lo + (hi - lo) * u;
  }
}

// Batched FP64 error oracle: out[i] = sum_k l[i*K + k] * r[i*K + k] with
// double-double accumulation, rounded once (R8: doubles; C8: complex
// products of interleaved pairs).  Used to check sampled elements of large
// contractions, one K-long dot product per sampled D element.
int orc_dd_dot_batch(int dtk, int64_t n, int64_t K, const void* l, const void* r, void* out, int nthreads) {
  if (dtk != R8 && dtk != C8) return 6;
  if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t i = 0; i < n; ++i) {
    if (dtk == R8) {
      const double* x = (const double*)l + i * K;
      const double* y = (const double*)r + i * K;
      dd acc{0.0, 0.0};
      for (int64_t k = 0; k < K; ++k) acc = dd_add(acc, two_prod(x[k], y[k]));
      ((double*)out)[i] = acc.hi + acc.lo;
    } else {
      const double* x = (const double*)l + 2 * i * K;
      const double* y = (const double*)r + 2 * i * K;
      dd sr{0, 0}, si{0, 0};
      for (int64_t k = 0; k < K; ++k) {
        const double xr = x[2 * k], xi = x[2 * k + 1], yr = y[2 * k], yi = y[2 * k + 1];
        sr = dd_add(sr, two_prod(xr, yr)); sr = dd_add(sr, two_prod(-xi, yi));
        si = dd_add(si, two_prod(xr, yi)); si = dd_add(si, two_prod(xi, yr));
      }
      ((double*)out)[2 * i] = sr.hi + sr.lo;
      ((double*)out)[2 * i + 1] = si.hi + si.lo;
    }
  }
  return 0;
}

}  // extern "C"
