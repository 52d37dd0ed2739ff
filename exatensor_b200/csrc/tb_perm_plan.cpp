// tb_perm_plan.cpp -- builds permutation plans (host code, no CUDA).
#include "tb_perm_plan.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/talsh_b200.h"

namespace tb {

int build_perm_plan(int es, int rank, const int64_t* dims_in, const int64_t* sin_in,
                    const int64_t* sout_in, PermParams* pp, int vmin_kb, int vmax_kb, int min_run) {
  PermParams& P = *pp;
  std::memset(&P, 0, sizeof(P));
  P.es = es;
  // 1. drop unit dims, merge neighbours that stay neighbours
  std::vector<int64_t> D, SI, SO;
  for (int i = 0; i < rank; ++i) {
    if (dims_in[i] <= 0) return TB_ERR_INVALID_ARGS;
    if (dims_in[i] == 1) continue;
    if (!D.empty() && SI.back() * D.back() == sin_in[i] && SO.back() * D.back() == sout_in[i]) {
      D.back() *= dims_in[i];
    } else {
      D.push_back(dims_in[i]); SI.push_back(sin_in[i]); SO.push_back(sout_in[i]);
    }
  }
  if (D.empty()) { D.push_back(1); SI.push_back(1); SO.push_back(1); }
  const int r = (int)D.size();
  if (r > kPlanMaxRank) return TB_ERR_INVALID_ARGS;
  if (SI[0] != 1) return TB_ERR_NOT_IMPLEMENTED;
  std::vector<int> Q(r);
  for (int i = 0; i < r; ++i) Q[i] = i;
  std::stable_sort(Q.begin(), Q.end(), [&](int x, int y) { return SO[x] < SO[y]; });
  if (SO[Q[0]] != 1) return TB_ERR_NOT_IMPLEMENTED;
  // minimum contiguous run of the load and store blocks (elements): 256 bytes
  // unless the caller (or TB_PERM_MINRUN, a tuning knob) asks for another
  static const int64_t run_env = [] {
    const char* e = std::getenv("TB_PERM_MINRUN");
    const long v = e ? std::atol(e) : 0;
    return (int64_t)(v >= 32 && v <= 4096 ? v : 256);
  }();
  const int64_t T = std::max<int64_t>(1, (min_run > 0 ? min_run : run_env) / es);
  // tile volume bounds (bytes; 16 KB .. 32 KB unless TB_PERM_VMIN_KB /
  // TB_PERM_VMAX_KB say otherwise -- tuning knobs that leave results unchanged)
  auto knob = [](const char* name, long dflt) {
    const char* e = std::getenv(name);
    const long v = e ? std::atol(e) : 0;
    return (int64_t)(v >= 4 && v <= 96 ? v : dflt) * 1024;
  };
  static const int64_t vmin_env = knob("TB_PERM_VMIN_KB", 16), vmax_env = knob("TB_PERM_VMAX_KB", 32);
  // explicit bounds (the measured plan choice) override the defaults
  const int64_t vmin_bytes = vmin_kb > 0 ? (int64_t)vmin_kb * 1024 : vmin_env;
  const int64_t vmax_bytes = vmax_kb > 0 ? (int64_t)vmax_kb * 1024 : vmax_env;
  const int64_t Vmax = std::max<int64_t>(1, vmax_bytes / es), Vmin = std::min(Vmax, std::max<int64_t>(1, vmin_bytes / es));
  std::vector<int64_t> t(r, 1);
  auto cdiv = [](int64_t x, int64_t y) { return (x + y - 1) / y; };
  // Even split: the smallest extent >= want that tiles D in the same number
  // of pieces as want does (76 with want 32 -> 26: 26+26+24, not 32+32+12).
  auto even = [&](int64_t D, int64_t want) {
    want = std::max<int64_t>(1, std::min(D, want));
    return cdiv(D, cdiv(D, want));
  };
  // Store-run extent: a divisor of D in [want, 1.5 want] if there is one
  // (5776 with want 32 -> 38: no partial tiles), else an even split into
  // pieces of at least want (90 with want 64 -> 90): store runs never fall
  // below the minimum run.
  auto even_up = [&](int64_t D, int64_t want) {
    want = std::max<int64_t>(1, std::min(D, want));
    for (int64_t x = want; x <= std::min(D, want + want / 2); ++x)
      if (D % x == 0) return x;
    return cdiv(D, std::max<int64_t>(1, D / want));
  };
  // 2. load block: input dims 0..a
  int a = 0;
  {
    int64_t vol = 1;
    for (a = 0; a < r; ++a) {
      if (vol * D[a] <= T && a < r - 1) { t[a] = D[a]; vol *= D[a]; continue; }
      t[a] = even(D[a], cdiv(T, vol));
      break;
    }
    if (a == r) a = r - 1;
  }
  // 3. store block: output-order prefix (must be dense in the output)
  std::vector<char> inB(r, 0);
  int blast = -1;
  {
    int64_t volB = 1;
    for (int j = 0; j < r; ++j) {
      const int i = Q[j];
      if (SO[i] != volB) break;  // not dense: the store run ends before i
      if (i < a || (i == a && t[a] == D[a]) || (i > a && t[i] == D[i])) {
        inB[i] = 1; blast = i; volB *= D[i];
        if (volB >= T) break;
        continue;
      }
      if (i == a) {
        t[a] = std::max(t[a], even_up(D[a], cdiv(T, volB)));
        inB[a] = 1; blast = a; volB *= t[a];
        if (t[a] == D[a] && volB < T) continue;  // became whole: the run may grow further
        break;
      }
      if (volB * D[i] <= T) { t[i] = D[i]; inB[i] = 1; blast = i; volB *= D[i]; continue; }
      t[i] = even_up(D[i], cdiv(T, volB));
      inB[i] = 1; blast = i; volB *= t[i];
      break;
    }
  }
  if (blast < 0) return TB_ERR_NOT_IMPLEMENTED;
  auto vol_of = [&]() { int64_t v = 1; for (int i = 0; i < r; ++i) v *= t[i]; return v; };
  // 4a. the fastest dimension stays fastest (the load and store blocks end on
  // the same dim): the permutation moves whole runs of it, so make those runs
  // long -- that dim up to Vmax, then the next input dim as the row direction.
  if (a == blast) {
    const int64_t others = vol_of() / t[a];
    t[a] = std::max(t[a], even(D[a], std::max<int64_t>(1, Vmax / others)));
    if (vol_of() < Vmin && a + 1 < r && t[a + 1] == 1) {
      // a divisor of the extent, so that this dim is never partial (only the
      // load and store blocks' last dims may be: pa, pb)
      int64_t want = std::max<int64_t>(1, Vmax / vol_of()), best = 1;
      for (int64_t x = std::min(want, D[a + 1]); x >= 1; --x)
        if (D[a + 1] % x == 0) { best = x; break; }
      t[a + 1] = best;
    }
  }
  // 4. extend the tile to Vmin elements: whole small dims first, then the
  // partial dims, then a divisor of a dim outside both blocks (so that no tile
  // is partial in it: when the load and store blocks cover the same dims, the
  // tile would otherwise stay as small as they are, e.g. 18 x 18 of an 18^6
  // tensor)
  for (int guard = 0; guard < 4 * r + 8; ++guard) {
    int64_t V = vol_of();
    if (V >= Vmin) break;
    bool grown = false;
    for (int i = 0; i < r && !grown; ++i) {
      if (t[i] == 1 && D[i] > 1 && V * D[i] <= Vmax) { t[i] = D[i]; grown = true; }
    }
    if (grown) continue;
    for (int which = 0; which < 2 && !grown; ++which) {
      const int d = which == 0 ? a : blast;
      if (t[d] < D[d]) {
        const int64_t f = std::min(cdiv(D[d], t[d]), cdiv(Vmin, V));
        if (f > 1) { const int64_t nt = even(D[d], t[d] * f); if (nt > t[d]) { t[d] = nt; grown = true; } }
      }
    }
    for (int i = 0; i < r && !grown; ++i) {
      if (t[i] != 1 || D[i] <= 1 || i <= a || inB[i]) continue;
      for (int64_t x = std::min(D[i] - 1, Vmax / V); x >= 2; --x)
        if (D[i] % x == 0) { t[i] = x; grown = true; break; }
    }
    if (!grown) break;
  }
  // 5a. a partial load-block dimension gets rows of whole 16-byte units where
  // the extent allows (so that rows can move as 16-byte copies)
  if (t[a] < D[a]) {
    int64_t pA = 1;
    for (int i = 0; i < a; ++i) pA *= D[i];
    int64_t m = 16, x = pA * es;
    while (x % 2 == 0 && m > 1) { x /= 2; m /= 2; }  // m = 16 / gcd(pA*es, 16)
    const int64_t up = cdiv(t[a], m) * m;
    if (up <= D[a] && up != t[a]) {
      const int64_t Vn = vol_of() / t[a] * up;
      if (Vn <= Vmax) t[a] = up;
    }
  }
  // 5. bulk-copy alignment: when the load block ends on a whole dimension and
  // its rows are not a multiple of 16 bytes, extend it into the next input
  // dimension by the smallest extent that makes them so (shrinking the store
  // block's partial extent if the tile would grow past Vmax).
  {
    int64_t pA = 1;
    for (int i = 0; i < a; ++i) pA *= D[i];
    // rows of whole 8-byte units of 4-byte elements move as 8-byte copies:
    // no need to grow the load block for them
    const bool rows8_ok = es < 8 && (pA * t[a] * es) % 8 == 0;
    if ((pA * t[a] * es) % 16 != 0 && !rows8_ok && t[a] == D[a] && a + 1 < r) {
      const int64_t pA2 = pA * D[a];
      int64_t g = 16, x = pA2 * es;
      while (x % 2 == 0 && g > 1) { x /= 2; g /= 2; }  // g = 16 / gcd(pA2*es, 16)
      int64_t nt = t[a + 1] > 1 ? cdiv(t[a + 1], g) * g : g;
      if (nt <= D[a + 1]) {
        int64_t Vn = vol_of() / t[a + 1] * nt;
        const int64_t tblast0 = blast >= 0 ? t[blast] : 0;
        if (Vn > Vmax && blast > a + 1 && t[blast] > 1) {  // only a store dim outside the load block
          const int64_t pBfull = [&]() { int64_t p = 1; for (int j = 0; j < r; ++j) if (inB[j] && j != blast) p *= t[j]; return p; }();
          const int64_t tb = std::max<int64_t>(cdiv(T, pBfull), t[blast] * Vmax / Vn);
          if (tb < t[blast]) { t[blast] = tb; Vn = vol_of() / t[a + 1] * nt; }
        }
        if (Vn <= Vmax) { t[a + 1] = nt; a = a + 1; }
        else if (blast >= 0) t[blast] = tblast0;  // extension rejected: keep the store block as it was
      }
    }
  }
  // 5b. partial dims that a nearby divisor tiles exactly: tiles at a
  // dimension's end are partial and take the kernel's general (slower) code,
  // so a partial extent moves to a divisor of its dimension within a factor
  // two when the tile stays within Vmax and keeps its vector-aligned rows
  // (76 with 26: 38, no partial tile).  The largest such tile is taken.
  {
    int64_t pA = 1;
    for (int i = 0; i < a; ++i) pA *= D[i];
    auto row_class = [&](int64_t ta) {  // 16: rows of 16-byte units, 8: of 8-byte units (4-byte elements)
      const int64_t bytes = pA * ta * es;
      return bytes % 16 == 0 ? 16 : (es < 8 && bytes % 8 == 0 ? 8 : 0);
    };
    int dims_to_fix[2] = {blast, a};
    for (int k = 0; k < 2; ++k) {
      const int d = dims_to_fix[k];
      if (d < 0 || t[d] >= D[d] || D[d] % t[d] == 0 || cdiv(D[d], t[d]) > 16) continue;  // few partial tiles
      if (k == 1 && d == blast) continue;  // same dim as the store block's last: already done
      const int64_t V = vol_of(), cur = t[d];
      int64_t best = 0, bestV = 0;
      for (int64_t x = std::max<int64_t>(1, cur / 2); x <= std::min(D[d], 2 * cur); ++x) {
        if (D[d] % x != 0) continue;
        const int64_t Vn = V / cur * x;
        if (Vn > Vmax || Vn < Vmin / 2) continue;
        if (d == a && row_class(x) < row_class(cur)) continue;
        if (d == blast && x * (V / cur) < 1) continue;
        if (Vn > bestV) { best = x; bestV = Vn; }
      }
      if (best) t[d] = best;
    }
  }
  // 6. chunk structure
  const int pa = (t[a] < D[a]) ? a : -1;
  const int pb = (t[blast] < D[blast]) ? blast : -1;
  int64_t prodA = 1;
  for (int i = 0; i < a; ++i) prodA *= D[i];
  const int64_t LA = prodA * t[a];
  // Shared-memory layout: load chunk c occupies row c with stride lap.  The
  // row stride is padded so that transposed reads (consecutive output
  // elements one row apart) spread over the banks: an odd number of 4-byte
  // words per row, or for bulk-copy rows an odd number of 16-byte units.
  // Rows of whole 8-byte units (4-byte elements) use an odd number of
  // 8-byte units per row instead, so that 8-byte copies stay aligned.
  const bool bulk_rows = (LA * es) % 16 == 0;
  const bool rows8 = !bulk_rows && es < 8 && (LA * es) % 8 == 0;
  int64_t lap;
  if (bulk_rows) {
    const int64_t u = 16 / es;  // elements per 16 bytes (>= 1)
    lap = LA;
    if (((lap * es) / 16) % 2 == 0) lap += u;
  } else if (rows8) {
    const int64_t u = 8 / es;
    lap = LA;
    if (((lap * es) / 8) % 2 == 0) lap += u;
  } else {
    lap = (LA % 2 == 1) ? LA : LA + 1;
  }
  // position strides (load block within a row, rest dims across rows)
  std::vector<int64_t> est(r, 0);
  {
    int64_t s = 1;
    for (int i = 0; i <= a; ++i) { est[i] = s; s *= t[i]; }
    s = lap;
    for (int i = a + 1; i < r; ++i) if (t[i] > 1) { est[i] = s; s *= t[i]; }
  }
  const int64_t V = vol_of();
  std::vector<int> Bdims;  // store block dims in output order
  for (int j = 0; j < r; ++j) if (inB[Q[j]]) Bdims.push_back(Q[j]);
  int64_t LB = 1;
  for (int d : Bdims) LB *= t[d];
  // store positions j' decompose on the store block's last dim (blast):
  // j' = (full store-block dims before blast) + prodB * digit(blast)
  int64_t prodB = 1;
  for (int d : Bdims) if (d != blast) prodB *= t[d];
  const int64_t nA = V / LA, nB = V / LB;
  if (nA > kMaxChunks || nB > kMaxChunks || prodB > kMaxEjf || V > (int64_t)1 << 28)
    return TB_ERR_NOT_IMPLEMENTED;
  P.rank = r; P.V = (int)V; P.LA = (int)LA; P.nA = (int)nA; P.LB = (int)LB; P.nB = (int)nB;
  P.pa = pa; P.pb = pb; P.prodA = (int)prodA; P.prodB = (int)prodB; P.ejf_n = (int)prodB;
  P.ej_pb_stride = (int)est[blast];
  P.lap = (int)lap;
  {
    // bulk-copy eligibility: rows of whole 16-byte units that start on 16-byte
    // boundaries everywhere, and a tensor whose byte size is a multiple of 16
    // (so rounding a partial row up to 16 bytes never leaves the tensor)
    int64_t tot = 1;
    for (int i = 0; i < r; ++i) tot *= D[i];
    P.total = tot;
    bool ok = bulk_rows && (tot * es) % 16 == 0 && (prodA * t[a] * es) % 16 == 0;
    for (int i = a + 1; i < r; ++i) if ((SI[i] * es) % 16 != 0) ok = false;
    P.tma_ok = ok ? 1 : 0;
    // the same for 8-byte copies of 4-byte elements (also when the rows are
    // whole 16-byte units but the row starts are only 8-byte aligned)
    bool ok8 = !ok && (rows8 || bulk_rows) && es < 8 && (tot * es) % 8 == 0 && (prodA * t[a] * es) % 8 == 0;
    for (int i = a + 1; i < r; ++i) if ((SI[i] * es) % 8 != 0) ok8 = false;
    P.vec8 = ok8 ? 1 : 0;
  }
  for (int i = 0; i < r; ++i) { P.dims[i] = D[i]; P.tile[i] = t[i]; P.sin[i] = SI[i]; P.sout[i] = SO[i]; }
  magic32((uint32_t)LA, &P.la_magic, &P.la_shift);
  magic32((uint32_t)LB, &P.lb_magic, &P.lb_shift);
  magic32((uint32_t)prodB, &P.pb_magic, &P.pb_shift);
  // load chunks: rest dims (tile dims outside the load block) in input order
  std::vector<int> restA;
  for (int i = a + 1; i < r; ++i) if (t[i] > 1) restA.push_back(i);
  for (int64_t c = 0; c < nA; ++c) {
    int64_t x = c, off = 0; int dpb = -1;
    for (int d : restA) { int64_t dg = x % t[d]; x /= t[d]; off += dg * SI[d]; if (d == pb) dpb = (int)dg; }
    P.ld_base[c] = off; P.ld_dpb[c] = (int16_t)dpb;
  }
  // store chunks: tile dims outside the store block, in output order
  std::vector<int> restB;
  for (int j = 0; j < r; ++j) { int d = Q[j]; if (t[d] > 1 && !inB[d]) restB.push_back(d); }
  for (int64_t c = 0; c < nB; ++c) {
    int64_t x = c, off = 0, eb = 0; int dpa = -1;
    for (int d : restB) {
      int64_t dg = x % t[d]; x /= t[d];
      off += dg * SO[d]; eb += dg * est[d];
      if (d == pa) dpa = (int)dg;
    }
    P.st_base[c] = off; P.st_ebase[c] = (int32_t)eb; P.st_dpa[c] = (int16_t)dpa;
  }
  P.lin2d = (restA.size() <= 1 && restB.size() <= 1 && prodB == 1) ? 1 : 0;
  P.row_is_pb = (!restA.empty() && restA[0] == pb) ? 1 : 0;
  P.chunk_is_pa = (!restB.empty() && restB[0] == pa) ? 1 : 0;
  P.row_sin = restA.empty() ? 0 : SI[restA[0]];
  P.chunk_sout = restB.empty() ? 0 : SO[restB[0]];
  P.chunk_eb = restB.empty() ? 0 : (int32_t)est[restB[0]];
  P.vbytes = P.tma_ok ? 16 : (P.vec8 ? 8 : 0);
  P.vec2d = (P.lin2d && P.vbytes && es <= P.vbytes && P.chunk_eb == 1 &&
             (P.ej_pb_stride * (int64_t)es) % P.vbytes == 0 && nB <= LA && (LA * es) % P.vbytes == 0) ? 1 : 0;
  P.nvec = P.vbytes ? (int)((LA * es + P.vbytes - 1) / P.vbytes) : 0;
  magic32((uint32_t)std::max(1, P.nvec), &P.nv_magic, &P.nv_shift);
  // row copies: store chunk c is load row c (same dim, same run), rows of
  // whole vectors
  P.rows2d = (P.lin2d && P.vbytes && es <= P.vbytes && nA == nB && LA == LB && P.ej_pb_stride == 1 &&
              (P.chunk_eb == lap || nA == 1) && (LA * es) % P.vbytes == 0) ? 1 : 0;
  {
    bool ov = P.rows2d && (P.chunk_sout * es) % P.vbytes == 0;
    for (int i = 0; ov && i < r; ++i)
      if (t[i] < D[i] && (t[i] * SO[i] * es) % P.vbytes != 0) ov = false;  // tile steps along grid dims
    P.out_vec = ov ? 1 : 0;
  }
  // positions inside a store chunk: store-block dims before blast
  for (int64_t j = 0; j < prodB; ++j) {
    int64_t x = j, e = 0;
    for (int d : Bdims) { if (d == blast) continue; int64_t dg = x % t[d]; x /= t[d]; e += dg * est[d]; }
    P.ejf[j] = (int32_t)e;
  }
  // 6. tile grid: consecutive tiles step along the dims in output order, so
  // that the CTAs running at one time write neighbouring output runs (the
  // write side of a permutation is the less forgiving one; measured +15% on
  // rank-4 R8 permutations over input order).  TB_PERM_GRID=in selects input
  // order (a tuning knob; results are identical).
  static const bool grid_out = [] {
    const char* e = std::getenv("TB_PERM_GRID");
    return !(e && std::strcmp(e, "in") == 0);
  }();
  int g = 0; int64_t nt = 1;
  for (int jj = 0; jj < r; ++jj) {
    const int i = grid_out ? Q[jj] : jj;
    const int64_t ext = cdiv(D[i], t[i]);
    if (ext > 1) { P.gdim[g] = i; P.gext[g] = ext; P.gdiv[g].init((uint64_t)ext); ++g; nt *= ext; }
  }
  P.ngd = g; P.ntiles = nt;
  P.gd32 = nt < ((int64_t)1 << 31) ? 1 : 0;
  for (int k = 0; k < g; ++k) magic32((uint32_t)std::min<int64_t>(P.gext[k], (int64_t)1 << 31), &P.gmag[k], &P.gsh[k]);
  return 0;
}

int build_perm_plan_o2n(int es, int rank, const int* dims, const int* cptrn, PermParams* p, int vmin_kb,
                        int vmax_kb, int min_run) {
  if (rank < 0 || rank > kPlanMaxRank) return TB_ERR_INVALID_ARGS;
  int64_t D[kPlanMaxRank], SI[kPlanMaxRank], SO[kPlanMaxRank], pos[kPlanMaxRank + 1];
  int seen[kPlanMaxRank + 1] = {0};
  for (int i = 0; i < rank; ++i) {
    if (cptrn[i] < 1 || cptrn[i] > rank || seen[cptrn[i]]) return TB_ERR_PATTERN;
    seen[cptrn[i]] = 1;
  }
  int64_t s = 1;
  for (int i = 0; i < rank; ++i) { D[i] = dims[i]; SI[i] = s; s *= dims[i]; }
  // output extents by position, then strides by position
  int64_t oe[kPlanMaxRank];
  for (int i = 0; i < rank; ++i) oe[cptrn[i] - 1] = dims[i];
  s = 1;
  for (int q = 0; q < rank; ++q) { pos[q] = s; s *= oe[q]; }
  for (int i = 0; i < rank; ++i) SO[i] = pos[cptrn[i] - 1];
  return build_perm_plan(es, rank, D, SI, SO, p, vmin_kb, vmax_kb, min_run);
}

int perm_glist_vector_bytes(const PermParams& P, int in_align, int nthr) {
  const int es = P.es;
  int vb = es;
  if (P.tma_ok && es < 16 && in_align % 16 == 0) vb = 16;
  else if (P.vec8 && es < 8 && in_align % 8 == 0) vb = 8;
  if (((int64_t)P.LA * es) % vb != 0) vb = es;
  const int64_t nld = (int64_t)P.nA * ((int64_t)P.LA * es / vb);
  const int64_t cap = (int64_t)kGListEntries * nthr;
  if (P.V > cap || nld > cap) return 0;
  int64_t maxl = 0, maxs = 0;
  for (int c = 0; c < P.nA; ++c) maxl = std::max<int64_t>(maxl, P.ld_base[c]);
  for (int c = 0; c < P.nB; ++c) maxs = std::max<int64_t>(maxs, P.st_base[c]);
  const int64_t lim = (int64_t)1 << 31;
  if (maxl + P.LA >= lim || maxs + P.LB >= lim) return 0;
  for (int c = 0; c < P.nA; ++c) if (P.ld_base[c] < 0) return 0;
  for (int c = 0; c < P.nB; ++c) if (P.st_base[c] < 0) return 0;
  return vb;
}

int perm2d_list_entries(const PermParams& P, bool rows, int nthr) {
  if (!P.lin2d || P.vbytes <= 0 || P.es > P.vbytes || P.nvec <= 0) return 0;
  const int64_t VW = P.vbytes / P.es;
  int64_t nld = (int64_t)P.nA * P.nvec, nst, maxb_ld, maxb_st;
  maxb_ld = (int64_t)(P.nA - 1) * P.row_sin + (int64_t)P.nvec * VW;
  if (rows) {
    if (!P.rows2d) return 0;
    nst = (int64_t)P.nB * P.nvec;
    maxb_st = (int64_t)(P.nB - 1) * P.chunk_sout + (int64_t)P.nvec * VW;
  } else {
    if (!P.vec2d || P.nB % VW != 0) return 0;
    nst = (int64_t)P.LB * (P.nB / VW);
    maxb_st = (int64_t)P.LB + (int64_t)P.nB * P.chunk_sout;
  }
  const int64_t lim = (int64_t)1 << 31;
  // shared-memory offsets are below the stage size; global ones must fit int32
  if (maxb_ld >= lim || maxb_st >= lim || P.row_sin < 0 || P.chunk_sout < 0) return 0;
  const int64_t need = std::max(nld, nst);
  if (need <= 8 * (int64_t)nthr) return 8;
  if (need <= 16 * (int64_t)nthr) return 16;
  return 0;
}

}  // namespace tb
