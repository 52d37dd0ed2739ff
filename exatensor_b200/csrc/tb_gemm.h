// tb_gemm.h -- GEMM cores used by the contraction driver.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace tb {

// Plain GEMM in the tensor's own type (TTGT form), both operands K-major:
// C[m + n*ldc] = (ar,ai) * sum_k op(A[k + m*lda]) op(B[k + n*ldb]) + (br,bi) * C.
int gemm_plain_tn(int dtk, int64_t M, int64_t N, int64_t K, const void* A, int64_t lda, const void* B,
                  int64_t ldb, void* C, int64_t ldc, double ar, double ai, double br, double bi, int lconj,
                  int rconj, cudaStream_t s);

}  // namespace tb
