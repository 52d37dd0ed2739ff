// Prints the fields of a permutation plan built by the product's planner
// (tb_perm_plan.cpp) that decide which kernel path its tiles take.
// Usage: perm_plan_info <es> <rank> d1..dn p1..pn
//   -> "lin2d vec2d rows2d lists LB es partial_small ntiles"
// partial_small: dims split into 2..16 tiles whose extent the tile does not divide.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../../exatensor_b200/csrc/tb_perm_plan.h"

using namespace tb;

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const int es = atoi(argv[1]), rank = atoi(argv[2]);
  std::vector<int> dims(rank), perm(rank);
  for (int i = 0; i < rank; ++i) dims[i] = atoi(argv[3 + i]);
  for (int i = 0; i < rank; ++i) perm[i] = atoi(argv[3 + rank + i]);
  static PermParams P;
  if (int e = build_perm_plan_o2n(es, rank, dims.data(), perm.data(), &P)) { printf("DECLINED %d\n", e); return 0; }
  int partial_small = 0;
  for (int i = 0; i < P.rank; ++i) {
    const long long n = (P.dims[i] + P.tile[i] - 1) / P.tile[i];
    if (n >= 2 && n <= 16 && P.dims[i] % P.tile[i] != 0) ++partial_small;
  }
  const int lists = P.rows2d ? perm2d_list_entries(P, true, 256) : (P.vec2d ? perm2d_list_entries(P, false, 256) : 0);
  printf("%d %d %d %d %d %d %d %lld\n", P.lin2d, P.vec2d, P.rows2d, lists, P.LB, P.es, partial_small,
         (long long)P.ntiles);
  return 0;
}
