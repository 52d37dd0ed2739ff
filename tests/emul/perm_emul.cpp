// CPU emulation of perm_tile_kernel's index arithmetic (exatensor_b200/csrc/
// tb_permute.cuh) driven by the product's own plan builder (tb_perm_plan.cpp).
// For each case it replays the kernel's tile loop, load phase and store phase
// thread by thread, checks every shared-memory and table index against its
// bound, and checks that each output element is written exactly once with the
// input element a reference O2N permutation puts there.
// Usage: perm_emul <es> <rank> d1..dn p1..pn  -> prints "OK <tiles> <V>" or an error.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include "../../exatensor_b200/csrc/tb_perm_plan.h"

using namespace tb;

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const int es = atoi(argv[1]);
  const int rank = atoi(argv[2]);
  std::vector<int> dims(rank), perm(rank);
  for (int i = 0; i < rank; ++i) dims[i] = atoi(argv[3 + i]);
  for (int i = 0; i < rank; ++i) perm[i] = atoi(argv[3 + rank + i]);
  static PermParams P;
  int e = build_perm_plan_o2n(es, rank, dims.data(), perm.data(), &P);
  if (e) { printf("DECLINED %d\n", e); return 0; }
  long long vol = 1;
  for (int d : dims) vol *= d;
  // reference output positions
  std::vector<long long> oe(rank), pos(rank), sout(rank);
  for (int i = 0; i < rank; ++i) oe[perm[i] - 1] = dims[i];
  long long s = 1;
  for (int q = 0; q < rank; ++q) { pos[q] = s; s *= oe[q]; }
  for (int i = 0; i < rank; ++i) sout[i] = pos[perm[i] - 1];
  std::vector<long long> ref(vol);  // ref[out] = in index
  for (long long i = 0; i < vol; ++i) {
    long long r = i, o = 0;
    for (int d = 0; d < rank; ++d) { long long x = r % dims[d]; r /= dims[d]; o += x * sout[d]; }
    ref[o] = i;
  }
  std::vector<long long> out(vol, -1), out2(P.lin2d ? vol : 0, -1);
  const bool vecpath = P.lin2d && (P.vec2d || P.rows2d);
  std::vector<long long> out3(vecpath ? vol : 0, -1);
  // Full-tile offset lists of perm2d_kernel (perm_list_entry), replayed for
  // every thread: the N entries of each thread together must cover the
  // tile's (outer, inner) grid exactly once, with the offsets the formulas
  // give, and the global ones must fit in 32 bits.
  const int NLIST = vecpath ? perm2d_list_entries(P, P.rows2d != 0, 256) : 0;
  struct Grid { int nq, np; long long Aq, Ap, Bq, Bp; };
  Grid gl{}, gs{};
  if (vecpath) {
    const int VB = P.vbytes, VW = VB / es;
    if (P.vec2d && P.rows2d) { printf("FAIL vec2d and rows2d both set\n"); return 1; }
    if (P.rows2d && (P.nA != P.nB || P.LA != P.LB || P.ej_pb_stride != 1 ||
                     (P.nA > 1 && (P.chunk_eb != P.lap || P.chunk_sout == 0)) || (P.LA * es) % VB != 0)) {
      printf("FAIL rows2d shape\n"); return 1;
    }
    gl = {P.nvec, P.nA, VB, (long long)P.lap * es, VW, P.row_sin};
    if (P.rows2d) gs = {P.nvec, P.nB, VB, (long long)P.chunk_eb * es, VW, P.chunk_sout};
    else gs = {P.LB, P.nB / VW, (long long)P.ej_pb_stride * es, VB, 1, (long long)VW * P.chunk_sout};
    if (NLIST != 0 && NLIST != 8 && NLIST != 16) { printf("FAIL list entries %d\n", NLIST); return 1; }
    if (NLIST && !P.rows2d && P.nB % VW != 0) { printf("FAIL lists with a ragged column group\n"); return 1; }
    auto check_list = [&](const Grid& g, const char* what) {
      std::vector<int> seen((size_t)g.nq * g.np, 0);
      for (int tid = 0; tid < 256; ++tid)
        for (int i = 0; i < NLIST; ++i) {
          const long long lin = (long long)tid + (long long)i * 256;
          if (lin >= (long long)g.nq * g.np) break;
          uint32_t a; int32_t b;
          perm_list_entry((int)lin, g.nq, (uint32_t)g.Aq, (uint32_t)g.Ap, (int32_t)g.Bq, (int32_t)g.Bp, &a, &b);
          const long long q = lin % g.nq, pp = lin / g.nq;
          if ((long long)a != pp * g.Ap + q * g.Aq || (long long)b != pp * g.Bp + q * g.Bq) {
            printf("FAIL %s list offsets %d %d\n", what, tid, i); exit(1);
          }
          seen[lin]++;
        }
      for (size_t i = 0; i < seen.size(); ++i)
        if (seen[i] != 1) { printf("FAIL %s list coverage %zu %d\n", what, i, seen[i]); exit(1); }
    };
    if (NLIST) { check_list(gl, "load"); check_list(gs, P.rows2d ? "row store" : "column store"); }
  }
  // General-plan list kernel (perm_glist_kernel): replayed for every plan that
  // fits its lists (16-byte-aligned input), whichever kernel the launcher
  // picks for it -- full tiles through the lists, partial tiles through the
  // table-driven store below.
  const int GVB = perm_glist_vector_bytes(P, 16, 256);
  std::vector<long long> out4(GVB ? vol : 0, -1);
  // Row-copy kernel (perm_rowcopy_kernel): plans whose store chunk c is load
  // row c move each row global to global; replayed for every such plan.
  const bool ROWCOPY = P.lin2d && P.nA == P.nB && P.LA == P.LB && P.ej_pb_stride == 1 &&
                       (P.chunk_eb == P.lap || P.nA == 1);
  std::vector<long long> out5(ROWCOPY ? vol : 0, -1);
  const int V = P.V, LA = P.LA, LB = P.LB;
  const long long bufn = (long long)P.nA * P.lap;
  std::vector<long long> buf(bufn, -1);
  auto fail = [&](const char* m, long long a, long long b) { printf("FAIL %s %lld %lld\n", m, a, b); exit(1); };
  if (P.lap < LA) fail("row stride", P.lap, LA);
  if (P.nA > kMaxChunks || P.nB > kMaxChunks || P.ejf_n > kMaxEjf) fail("table size", P.nA, P.nB);
  if ((long long)P.LA * P.nA != V || (long long)P.LB * P.nB != V) fail("chunk product", LA, LB);
  for (long long tile = 0; tile < P.ntiles; ++tile) {
    long long in_base = 0, out_base = 0;
    int rem_a = 1 << 30, rem_b = 1 << 30;
    unsigned long long r = tile;
    for (int g = 0; g < P.ngd; ++g) {
      unsigned long long q = P.gdiv[g].div(r);
      if (q != r / (unsigned long long)P.gext[g]) fail("fastdiv", r, P.gext[g]);
      if (P.gd32) {
        if (r >= (1ull << 31)) fail("gd32 with a tile index past 2^31", r, tile);
        if (fdiv32((uint32_t)r, P.gmag[g], P.gsh[g]) != q) fail("fdiv32 grid", r, P.gext[g]);
      }
      long long x = (long long)(r - q * P.gext[g]);
      r = q;
      int d = P.gdim[g];
      long long org = x * P.tile[d];
      in_base += org * P.sin[d];
      out_base += org * P.sout[d];
      long long rem = P.dims[d] - org;
      if (d == P.pa) rem_a = (int)(rem < P.tile[d] ? rem : P.tile[d]);
      if (d == P.pb) rem_b = (int)(rem < P.tile[d] ? rem : P.tile[d]);
    }
    const bool full = (P.pa < 0 || rem_a >= P.tile[P.pa]) && (P.pb < 0 || rem_b >= P.tile[P.pb]);
    std::fill(buf.begin(), buf.end(), -1);
    for (int ee = 0; ee < V; ++ee) {
      int c = (int)fdiv32((uint32_t)ee, P.la_magic, P.la_shift);
      if (c != ee / LA) fail("fdiv32 LA", ee, LA);
      int j = ee - c * LA;
      bool ok = true;
      if (!full) {
        if (P.pa >= 0) { int da = j / P.prodA; ok = da < rem_a; if (P.pb == P.pa) ok = ok && da < rem_b; }
        if (P.pb >= 0 && P.pb != P.pa) ok = ok && P.ld_dpb[c] < rem_b;
      }
      if (ok) {
        long long src = in_base + P.ld_base[c] + j;
        if (src < 0 || src >= vol) fail("load oob", src, tile);
        long long p = (long long)c * P.lap + j;
        if (p >= bufn) fail("smem oob", p, bufn);
        buf[p] = src;
      }
    }
    if (P.tma_ok || P.vec8) {
      // vector-copy replay: each valid row is copied with its byte length
      // rounded up to the vector (16 bytes, or 8 for vec8); the copy must stay
      // inside the tensor and inside its smem row, both ends aligned
      const long long vb = P.tma_ok ? 16 : 8;
      if (P.vec8 && (es >= 8 || P.tma_ok)) fail("vec8 with wide elements or tma", es, P.tma_ok);
      for (int c = 0; c < P.nA; ++c) {
        bool ok = true;
        if (!full && P.pb >= 0 && P.pb != P.pa) ok = P.ld_dpb[c] < rem_b;
        if (!ok) continue;
        long long len = (!full && P.pa >= 0) ? (long long)P.prodA * std::min(rem_a, P.pb == P.pa ? rem_b : rem_a)
                                              : (long long)LA;
        long long bytes = (len * es + vb - 1) / vb * vb;
        long long src = in_base + P.ld_base[c];
        if ((src * es) % vb != 0) fail("vector source misaligned", src, c);
        if (src * es + bytes > vol * es) fail("vector copy leaves the tensor", src, bytes);
        if (bytes > (long long)P.lap * es) fail("vector copy overflows its row", bytes, P.lap);
        if (((long long)c * P.lap * es) % vb != 0) fail("vector destination misaligned", c, P.lap);
      }
    }
    // store phase as perm_store: 8 warps, (chunk, block) units, strided positions
    {
      const int lpc = P.LB >= 24 ? 32 : (P.LB >= 12 ? 16 : 8), cpw = 32 / lpc;
      const int blk = P.LB <= 512 ? P.LB : (512 / P.ejf_n) * P.ejf_n;
      if (blk < 1 || (blk != P.LB && blk % P.ejf_n != 0)) fail("block not a multiple of prodB", blk, P.ejf_n);
      const int nblk = (P.LB + blk - 1) / blk;
      const int qlim = (!full && P.pb >= 0) ? (P.pa == P.pb ? std::min(rem_a, rem_b) : rem_b) : (1 << 30);
      const bool dpa_check = !full && P.pa >= 0 && P.pa != P.pb;
      const int units = P.nB * nblk;
      for (int warp = 0; warp < 8; ++warp)
        for (int lane = 0; lane < 32; ++lane) {
          const int sub = lane / lpc, l = lane % lpc;
          for (int u = warp * cpw + sub; u < units; u += 8 * cpw) {
            const int c = u / nblk, j0 = (u - c * nblk) * blk;
            if (dpa_check && P.st_dpa[c] >= rem_a) continue;
            const int jmax = std::min(j0 + blk, LB);
            for (int j = j0 + l; j < jmax; j += lpc) {
              const int q = (int)fdiv32((uint32_t)j, P.pb_magic, P.pb_shift);
              if (q != j / P.ejf_n) fail("fdiv32 prodB", j, P.ejf_n);
              if (q >= qlim) break;
              const long long ee = (long long)P.st_ebase[c] + P.ejf[j - q * P.ejf_n] + (long long)q * P.ej_pb_stride;
              if (P.ejf_n == 1 && ee != (long long)P.st_ebase[c] + (long long)j * P.ej_pb_stride) fail("pB1 form", j, c);
              if (ee < 0 || ee >= bufn) fail("smem position oob", ee, bufn);
              const long long dst = out_base + P.st_base[c] + j;
              if (dst < 0 || dst >= vol) fail("store oob", dst, tile);
              if (buf[ee] < 0) fail("store reads unloaded smem", ee, tile);
              if (out[dst] != -1) fail("double write", dst, tile);
              out[dst] = buf[ee];
              if (GVB && !full) out4[dst] = buf[ee];  // the list kernel's partial tiles
            }
          }
        }
    }
    if (GVB && full) {
      const int VW = GVB / es, nvec = LA / VW, nld_all = P.nA * nvec;
      if ((long long)LA % VW) fail("glist rows not whole vectors", LA, VW);
      if (P.V > kGListEntries * 256 || nld_all > kGListEntries * 256) fail("glist lists too short", P.V, nld_all);
      std::vector<long long> gbuf(bufn, -1);
      for (int tid = 0; tid < 256; ++tid)
        for (int i = 0; i < kGListEntries; ++i) {
          const int v = tid + i * 256;
          if (v >= nld_all) break;
          const int c = v / nvec, x = v - c * nvec;
          const long long a = ((long long)c * P.lap + (long long)x * VW) * es;  // shared-memory bytes
          const long long b = P.ld_base[c] + (long long)x * VW;                  // tile-relative element
          if (a % GVB) fail("glist load smem misaligned", a, tid);
          if (((in_base + b) * es) % GVB) fail("glist load source misaligned", in_base + b, tid);
          if ((long long)x * VW + VW > P.lap || a / es + VW > bufn) fail("glist load smem oob", a, tid);
          if (b >= ((long long)1 << 31)) fail("glist load offset beyond 32 bits", b, tid);
          if (in_base + b < 0 || in_base + b + VW > vol) fail("glist load leaves the tensor", in_base + b, tid);
          for (int t = 0; t < VW; ++t) gbuf[a / es + t] = in_base + b + t;
        }
      for (int tid = 0; tid < 256; ++tid)
        for (int i = 0; i < kGListEntries; ++i) {
          const int e = tid + i * 256;
          if (e >= V) break;
          const int cc = e / LB, j = e - cc * LB, q = j / P.prodB;
          const long long pos = (long long)P.st_ebase[cc] + P.ejf[j - q * P.prodB] + (long long)q * P.ej_pb_stride;
          const long long rel = P.st_base[cc] + j;
          if (pos < 0 || pos >= bufn) fail("glist store smem oob", pos, tid);
          if (rel >= ((long long)1 << 31)) fail("glist store offset beyond 32 bits", rel, tid);
          const long long dst = out_base + rel;
          if (dst < 0 || dst >= vol) fail("glist store oob", dst, tid);
          if (gbuf[pos] < 0) fail("glist store reads unloaded smem", pos, tid);
          if (out4[dst] != -1) fail("glist double write", dst, tid);
          out4[dst] = gbuf[pos];
        }
    }
    if (ROWCOPY) {
      for (int c = 0; c < P.nA; ++c) {
        if (!full && P.pb >= 0 && P.pb != P.pa && P.row_is_pb && c >= rem_b) continue;
        long long len = P.LA;
        if (!full && P.pa >= 0) len = (long long)P.prodA * (P.pb == P.pa ? std::min(rem_a, rem_b) : rem_a);
        for (long long j = 0; j < len; ++j) {
          const long long src = in_base + (long long)c * P.row_sin + j;
          const long long dst = out_base + (long long)c * P.chunk_sout + j;
          if (src < 0 || src >= vol) fail("rowcopy load oob", src, tile);
          if (dst < 0 || dst >= vol) fail("rowcopy store oob", dst, tile);
          if (out5[dst] != -1) fail("rowcopy double write", dst, tile);
          out5[dst] = src;
        }
      }
    }
    // two-dimensional kernel replay (perm2d_kernel): rows, chunks and
    // positions by formula instead of the chunk tables
    if (P.vec2d) {
      // 16-byte column groups: the widest group read stays inside a row, rows
      // and groups are 16-byte aligned, and full-row vectors fit the row
      const int VB = P.vbytes, VW = VB / es;
      if (VB != 16 && VB != 8) fail("vec2d vector bytes", VB, 0);
      if (VW < 1) fail("vec2d element wider than the vector", es, VB);
      if (!P.lin2d || P.chunk_eb != 1) fail("vec2d without unit chunk step", P.chunk_eb, 0);
      if ((long long)((P.nB + VW - 1) / VW) * VW > P.lap) fail("vec2d group beyond row", P.nB, P.lap);
      if (((long long)P.ej_pb_stride * es) % VB || ((long long)P.lap * es) % VB) fail("vec2d row alignment", P.lap, 0);
      if ((long long)P.nvec * VB > (long long)P.lap * es) fail("vec2d vectors beyond row", P.nvec, P.lap);
      if (P.nvec != (P.LA * es + VB - 1) / VB) fail("vec2d nvec", P.nvec, P.LA);
      if (!(VB == 16 ? P.tma_ok : P.vec8)) fail("vec2d without aligned copies", VB, 0);
      for (int v = 0; v < P.nA * P.nvec; v += 7)
        if ((int)fdiv32((uint32_t)v, P.nv_magic, P.nv_shift) != v / P.nvec) fail("fdiv32 nvec", v, P.nvec);
    }
    if (vecpath && full && NLIST) {
      // full tile through the lists: vector loads, then vector reads of the
      // stage feeding the row-copy or column-group stores
      const int VB = P.vbytes, VW = VB / es;
      std::vector<long long> vbuf(bufn, -1);
      for (int tid = 0; tid < 256; ++tid)
        for (int i = 0; i < NLIST; ++i) {
          const int lin = tid + i * 256;
          if (lin >= gl.nq * gl.np) break;
          uint32_t a; int32_t b;
          perm_list_entry(lin, gl.nq, (uint32_t)gl.Aq, (uint32_t)gl.Ap, (int32_t)gl.Bq, (int32_t)gl.Bp, &a, &b);
          if (a % VB != 0) fail("list load smem misaligned", a, tid);
          const long long src = in_base + b;
          if ((src * es) % VB != 0) fail("list load source misaligned", src, tid);
          if (src < 0 || (src * es + VB) > vol * es) fail("list load leaves the tensor", src, tid);
          const long long e0 = a / es;
          if (e0 + VW > bufn) fail("list load smem oob", e0, bufn);
          for (int t = 0; t < VW; ++t)
            if (src + t < vol) vbuf[e0 + t] = src + t;  // past a row's end: padding, never stored
        }
      for (int tid = 0; tid < 256; ++tid)
        for (int i = 0; i < NLIST; ++i) {
          const int lin = tid + i * 256;
          if (lin >= gs.nq * gs.np) break;
          uint32_t a; int32_t b;
          perm_list_entry(lin, gs.nq, (uint32_t)gs.Aq, (uint32_t)gs.Ap, (int32_t)gs.Bq, (int32_t)gs.Bp, &a, &b);
          if (a % VB != 0) fail("list store smem misaligned", a, tid);
          const long long e0 = a / es;
          if (e0 + VW > bufn) fail("list store smem oob", e0, bufn);
          for (int t = 0; t < VW; ++t) {
            const long long rel = P.rows2d ? (long long)b + t : (long long)b + (long long)t * P.chunk_sout;
            if (rel >= ((long long)1 << 31)) fail("list store offset beyond 32 bits", rel, tid);
            const long long dst = out_base + rel;
            if (P.rows2d && P.out_vec && t == 0 && ((out_base + b) * es) % VB != 0) fail("row store misaligned", dst, tid);
            if (dst < 0 || dst >= vol) fail("list store oob", dst, tid);
            if (vbuf[e0 + t] < 0) fail("list store reads unloaded smem", e0 + t, tid);
            if (out3[dst] != -1) fail("list double write", dst, tid);
            out3[dst] = vbuf[e0 + t];
          }
        }
    }
    if (P.lin2d) {
      int rows = P.nA;
      if (!full && P.pb >= 0 && P.pb != P.pa && P.row_is_pb) rows = std::min(rows, rem_b);
      for (int c = 0; c < P.nA; ++c) {
        const bool tab_ok = !(!full && P.pb >= 0 && P.pb != P.pa) || P.ld_dpb[c] < rem_b;
        if ((c < rows) != tab_ok) fail("2d row count", c, rows);
        if (P.ld_base[c] != (long long)c * P.row_sin) fail("2d row stride", c, P.row_sin);
      }
      int chunks = P.nB;
      if (!full && P.pa >= 0 && P.pa != P.pb && P.chunk_is_pa) chunks = std::min(chunks, rem_a);
      const int qlim = (!full && P.pb >= 0) ? (P.pa == P.pb ? std::min(rem_a, rem_b) : rem_b) : (1 << 30);
      const int jlim = std::min(LB, qlim);
      for (int c = 0; c < P.nB; ++c) {
        const bool tab_ok = !(!full && P.pa >= 0 && P.pa != P.pb) || P.st_dpa[c] < rem_a;
        if ((c < chunks) != tab_ok) fail("2d chunk count", c, chunks);
        if (c >= chunks) continue;
        if (P.st_base[c] != (long long)c * P.chunk_sout || P.st_ebase[c] != c * P.chunk_eb) fail("2d chunk stride", c, 0);
        for (int j = 0; j < jlim; ++j) {
          const long long ee = (long long)c * P.chunk_eb + (long long)j * P.ej_pb_stride;
          if (ee < 0 || ee >= bufn) fail("2d smem oob", ee, bufn);
          const long long dst = out_base + (long long)c * P.chunk_sout + j;
          if (dst < 0 || dst >= vol) fail("2d store oob", dst, tile);
          if (buf[ee] < 0) fail("2d store reads unloaded smem", ee, tile);
          if (out2[dst] != -1) fail("2d double write", dst, tile);
          out2[dst] = buf[ee];
          if (vecpath && (!full || !NLIST)) out3[dst] = buf[ee];  // the general 2-D code
        }
      }
    }
  }
  for (long long o = 0; o < vol; ++o) {
    if (out[o] != ref[o]) fail("wrong value at", o, out[o]);
    if (P.lin2d && out2[o] != ref[o]) fail("2d wrong value at", o, out2[o]);
    if (vecpath && out3[o] != ref[o]) fail("walk wrong value at", o, out3[o]);
    if (GVB && out4[o] != ref[o]) fail("glist wrong value at", o, out4[o]);
    if (ROWCOPY && out5[o] != ref[o]) fail("rowcopy wrong value at", o, out5[o]);
  }
  printf("OK %lld %d %d %d tma=%d vec8=%d lin2d=%d vec2d=%d rows2d=%d lists=%d glist=%d rowcopy=%d\n",
         (long long)P.ntiles, V, LA, LB, P.tma_ok, P.vec8, P.lin2d, P.vec2d, P.rows2d, NLIST, GVB, (int)ROWCOPY);
  return 0;
}
