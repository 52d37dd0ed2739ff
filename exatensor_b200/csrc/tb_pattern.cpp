// tb_pattern.cpp -- symbolic index patterns and contraction matricization.
//
// Grammar (TALSH/tensor_algebra_cpu.F90:5307-5531, get_contr_pattern_dig):
// a pattern names one destination and one or two input tensors, each written
// NAME(idx,idx,...) with indices separated by ',' or '|'; text outside the
// parentheses is ignored.  A '+' between a tensor name and its '(' requests
// complex conjugation (bit 0 = D, bit 1 = L, bit 2 = R).  An index label is
// alphanumeric and may end in one '+' (contravariant), which is ignored for
// matching.  In a contraction every label occurs either in D and in exactly
// one input (uncontracted), in D and in both inputs (hyper-index), or in
// both inputs but not in D (contracted); in a copy/add every label occurs
// once in D and once in L.  The digital pattern gives, for each input
// dimension, its destination position (>0) or minus its partner's position
// in the other input (<0).
#include "tb_pattern.h"

#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/talsh_b200.h"

namespace tb {

namespace {

bool is_alnum(char c) {
  return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9');
}

struct Arg {
  bool conj = false;
  std::vector<std::string> labels;
};

// Splits the pattern into parenthesised argument lists.
int tokenize(const char* s, std::vector<Arg>& args) {
  const int n = (int)std::strlen(s);
  int i = 0;
  while (i < n) {
    while (i < n && s[i] != '(') ++i;
    if (i >= n) break;
    Arg a;
    a.conj = (i >= 2 && s[i - 1] == '+' && (is_alnum(s[i - 2]) || s[i - 2] == '_'));
    int j = i + 1;
    std::string cur;
    bool sep_seen = false, closed = false;
    for (; j < n; ++j) {
      const char c = s[j];
      if (c == ',' || c == '|' || c == ')') {
        if (c == ')' && cur.empty() && !sep_seen) { closed = true; break; }  // "T()"
        if (cur.empty()) return 2;
        // label: alphanumeric, optional single trailing '+'
        std::string lb = cur;
        if (lb.back() == '+') lb.pop_back();
        if (lb.empty()) return 2;
        for (char ch : lb) if (!is_alnum(ch)) return 2;
        a.labels.push_back(lb);
        cur.clear();
        if (c == ')') { closed = true; break; }
        sep_seen = true;
      } else {
        cur.push_back(c);
      }
    }
    if (!closed) return 5;
    args.push_back(a);
    if (args.size() > 3) return 1;
    i = j + 1;
  }
  return 0;
}

}  // namespace

int parse_pattern(const char* pattern, ParsedPattern* out) {
  ParsedPattern& P = *out;
  P = ParsedPattern();
  if (!pattern) return 16;
  std::string s(pattern);
  while (!s.empty() && s.back() == ' ') s.pop_back();
  if (s.empty()) return 16;
  std::vector<Arg> args;
  if (int e = tokenize(s.c_str(), args)) return e;
  if (args.size() < 2) return 15;
  const int nin = (int)args.size() - 1;
  for (size_t t = 0; t < args.size(); ++t)
    if ((int)args[t].labels.size() > kPatternMaxRank) return 17;
  P.drank = (int)args[0].labels.size();
  P.lrank = (int)args[1].labels.size();
  P.rrank = nin == 2 ? (int)args[2].labels.size() : -1;
  P.conj_bits = (args[0].conj ? 1 : 0) | (args[1].conj ? 2 : 0) | (nin == 2 && args[2].conj ? 4 : 0);
  // label -> positions (1-based) in each argument
  struct Occ { int pos[3] = {0, 0, 0}; int count[3] = {0, 0, 0}; };
  std::unordered_map<std::string, Occ> occ;
  for (size_t t = 0; t < args.size(); ++t)
    for (size_t k = 0; k < args[t].labels.size(); ++k) {
      Occ& o = occ[args[t].labels[k]];
      o.count[t]++;
      if (!o.pos[t]) o.pos[t] = (int)k + 1;
    }
  const int L = P.lrank;
  for (size_t t = 1; t < args.size(); ++t) {
    for (size_t k = 0; k < args[t].labels.size(); ++k) {
      const Occ& o = occ[args[t].labels[k]];
      for (int q = 0; q < 3; ++q) if (o.count[q] > 1) return 10;  // repeated within one tensor
      const int slot = (t == 1 ? 0 : L) + (int)k;
      if (o.count[0] == 1) {
        P.cptrn[slot] = o.pos[0];                       // uncontracted (hyper if in both inputs)
        if (nin == 2 && o.count[1] && o.count[2]) P.hyper = true;
      } else {
        if (nin == 1) return 13;
        const int other = (t == 1) ? 2 : 1;
        if (!o.count[other]) return 11;                 // appears once only
        P.cptrn[slot] = -o.pos[other];                  // contracted
      }
    }
  }
  // every destination label must appear in an input
  for (size_t k = 0; k < args[0].labels.size(); ++k) {
    const Occ& o = occ[args[0].labels[k]];
    if (o.count[0] > 1) return 10;
    if (!o.count[1] && (nin == 1 || !o.count[2])) return nin == 1 ? 14 : 11;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Matricization of a contraction: D(m,n) = sum_k L(m,k) R(k,n), where m runs
// over L's uncontracted dims, n over R's uncontracted dims and k over the
// contracted dims.  Offsets of every operand factor into one term per group,
// so any index order is a pair of offset tables (the fused gather/epilogue)
// or a permutation into a matrix layout (TTGT).
// ---------------------------------------------------------------------------
int matricize(const int* cptrn, int drank, const int* ddims, int lrank, const int* ldims, int rrank,
              const int* rdims, Matricization* mz) {
  Matricization& Z = *mz;
  Z = Matricization();
  if (drank < 0 || lrank < 0 || rrank < 0 || drank > kPatternMaxRank || lrank > kPatternMaxRank ||
      rrank > kPatternMaxRank)
    return TB_ERR_INVALID_ARGS;
  int64_t lb[kPatternMaxRank], rb[kPatternMaxRank], db[kPatternMaxRank];
  int64_t s = 1;
  for (int i = 0; i < lrank; ++i) { if (ldims[i] <= 0) return TB_ERR_INVALID_ARGS; lb[i] = s; s *= ldims[i]; }
  s = 1;
  for (int i = 0; i < rrank; ++i) { if (rdims[i] <= 0) return TB_ERR_INVALID_ARGS; rb[i] = s; s *= rdims[i]; }
  s = 1;
  for (int i = 0; i < drank; ++i) { if (ddims[i] <= 0) return TB_ERR_INVALID_ARGS; db[i] = s; s *= ddims[i]; }
  int dused[kPatternMaxRank + 1] = {0};
  for (int i = 0; i < lrank; ++i) {
    const int c = cptrn[i];
    if (c > 0) {
      if (c > drank || ddims[c - 1] != ldims[i] || dused[c]) return TB_ERR_PATTERN;
      dused[c] = 1;
      Z.m.push_back({ldims[i], lb[i], db[c - 1], c - 1, i});
    } else {
      const int rp = -c;
      if (rp < 1 || rp > rrank || cptrn[lrank + rp - 1] != -(i + 1) || rdims[rp - 1] != ldims[i])
        return TB_ERR_PATTERN;
    }
  }
  for (int i = 0; i < rrank; ++i) {
    const int c = cptrn[lrank + i];
    if (c > 0) {
      if (c > drank || ddims[c - 1] != rdims[i] || dused[c]) return TB_ERR_PATTERN;
      dused[c] = 1;
      Z.n.push_back({rdims[i], rb[i], db[c - 1], c - 1, i});
    } else {
      const int lp = -c;
      if (lp < 1 || lp > lrank || cptrn[lp - 1] != -(i + 1)) return TB_ERR_PATTERN;
      Z.k.push_back({rdims[i], lb[lp - 1], rb[i], lp - 1, i});  // (extent, L stride, R stride)
    }
  }
  for (int q = 1; q <= drank; ++q) if (!dused[q]) return TB_ERR_PATTERN;
  Z.M = 1; for (auto& g : Z.m) Z.M *= g.ext;
  Z.N = 1; for (auto& g : Z.n) Z.N *= g.ext;
  Z.K = 1; for (auto& g : Z.k) Z.K *= g.ext;
  Z.drank = drank; Z.lrank = lrank; Z.rrank = rrank;
  return 0;
}

}  // namespace tb

extern "C" int tb_parse_pattern(const char* pattern, int* cptrn, int* drank, int* lrank, int* rrank,
                                int* conj_bits) {
  tb::ParsedPattern P;
  int e = tb::parse_pattern(pattern, &P);
  if (e) {
    tb::set_error("pattern parse error %d in \"%s\"", e, pattern ? pattern : "(null)");
    return TB_ERR_PATTERN;
  }
  const int n = P.lrank + (P.rrank > 0 ? P.rrank : 0);
  for (int i = 0; i < n; ++i) cptrn[i] = P.cptrn[i];
  if (drank) *drank = P.drank;
  if (lrank) *lrank = P.lrank;
  if (rrank) *rrank = P.rrank;
  if (conj_bits) *conj_bits = P.conj_bits;
  return 0;
}
