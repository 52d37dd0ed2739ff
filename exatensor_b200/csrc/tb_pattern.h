// tb_pattern.h -- host-side index-pattern parsing and contraction matricization.
#pragma once
#include <cstdint>
#include <vector>

namespace tb {

constexpr int kPatternMaxRank = 56;

void set_error(const char* fmt, ...);

struct ParsedPattern {
  int drank = -1, lrank = -1, rrank = -1;  // rrank = -1 for unary (copy/add) patterns
  int conj_bits = 0;                       // bit0 D, bit1 L, bit2 R
  bool hyper = false;                      // an index present in D, L and R
  int cptrn[2 * kPatternMaxRank] = {0};    // digital pattern (lrank + rrank entries)
};

// Returns 0 or a nonzero parse error code.
int parse_pattern(const char* pattern, ParsedPattern* out);

// One index group of a matricized contraction.
struct MGroup {
  int64_t ext;    // extent
  int64_t s1;     // stride in the first tensor of the group (L for m and k, R for n)
  int64_t s2;     // stride in the second tensor (D for m and n, R for k)
  int dpos;       // position in D (m, n) or in L (k)
  int src;        // position in the owning input
};

struct Matricization {
  int drank = 0, lrank = 0, rrank = 0;
  int64_t M = 1, N = 1, K = 1;
  std::vector<MGroup> m;  // L-uncontracted dims (L order): s1 = L stride, s2 = D stride
  std::vector<MGroup> n;  // R-uncontracted dims (R order): s1 = R stride, s2 = D stride
  std::vector<MGroup> k;  // contracted dims (R order):    s1 = L stride, s2 = R stride
};

// Validates a digital contraction pattern against the shapes and fills mz.
int matricize(const int* cptrn, int drank, const int* ddims, int lrank, const int* ldims, int rrank,
              const int* rdims, Matricization* mz);

}  // namespace tb
