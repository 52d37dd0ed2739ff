// tb_tc.cu -- tensor-core (tcgen05) contraction path.
#include "tb_common.cuh"
#include "tb_contract.h"

namespace tb {

int select_method(int, const Matricization&, const tb_plan_t*) { return TB_METHOD_TTGT; }

int contract_fused(const Matricization&, int, const int*, void*, const int*, const void*, const int*, const void*,
                   double, double, bool, int, int, const tb_plan_t*, cudaStream_t, tb_contract_stats_t*) {
  set_error("fused tensor-core contraction not available for this request");
  return TB_ERR_NOT_IMPLEMENTED;
}

}  // namespace tb
