// tb_contract.h -- contraction driver internals shared with the tensor-core path.
#pragma once
#include <cuda_runtime.h>

#include "../../include/talsh_b200.h"
#include "tb_pattern.h"

namespace tb {

int contract_impl(const int* cptrn, int dtk, int drank, const int* ddims, void* d, int lrank, const int* ldims,
                  const void* l, int rrank, const int* rdims, const void* r, double ar, double ai, int conj_bits,
                  int accumulative, const tb_plan_t* plan, cudaStream_t s);

// Chooses TB_METHOD_TTGT or TB_METHOD_FUSED for a matricized contraction.
int select_method(int dtk, const Matricization& Z, const tb_plan_t* plan);

// Tensor-core contraction with fused operand gathers and epilogue.
// Returns TB_ERR_NOT_IMPLEMENTED when the shape is outside its scope.
int contract_fused(const Matricization& Z, int dtk, const int* ddims, void* d, const int* ldims, const void* l,
                   const int* rdims, const void* r, double ar, double ai, bool accumulate, int lconj, int rconj,
                   const tb_plan_t* plan, cudaStream_t s, tb_contract_stats_t* stats);

// Learned plan selection (tb_select.cu).
int descriptor_of(const Matricization& Z, int dtk, float* features);
// -1 when no selector is installed; else 0 with the chosen plan index, whether
// the two best predictions are too close to call (and autotuning is on), and a
// cache key of the descriptor.
// Candidate plans (the network's outputs, TB_SELECT_PLANS of them): 0 TTGT,
// 1 tensor cores with N tile 128, 2 with N tile 256, 3 (kCandPair) the
// 256-wide tile on SM pairs (cta_group::2, 256-row tiles), 4 (kCandSlices)
// the 256-wide tile with 6 INT8 slices (FP64 only).
constexpr int kCandPair = 3;
constexpr int kCandSlices = 4;
constexpr int kNumCandidates = 5;
// The network's choice for a descriptor (idx), or the cached measured one;
// tune_mask: candidates to time before choosing (0: none).
int selector_pick(const float* features, int* idx, unsigned* tune_mask, uint64_t* key);
void selector_remember(uint64_t key, int idx);
void selector_autoload();

}  // namespace tb
