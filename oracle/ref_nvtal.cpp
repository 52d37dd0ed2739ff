// ref_nvtal.cpp -- TEST INFRASTRUCTURE ONLY: a C harness over the reference's
// own NV-TAL device path (ExaTENSOR TALSH/tensor_algebra_gpu_nvidia.cu with
// TALSH/tensor_algebra_gpu.cpp, mem_manager.cpp and timer.cpp), which
// oracle/Makefile compiles from the reference's sources, unchanged, into
// oracle/_ref/libnvtal_ref.so in the reference's default configuration (its
// contractions call cuBLAS GEMMs, :6899-7024).  The tests call these
// functions to compare this library's results with the reference's GPU kernels
// on the same inputs:
//   ref_copy      gpu_tensor_block_copy        (TALSH/tensor_algebra_gpu_nvidia.cu:4806)
//   ref_add       gpu_tensor_block_add         (:5203)
//   ref_contract  gpu_tensor_block_contract_dlf (:5847)
// each driven the way the reference's NV-TAL test does (TALSH/test.cpp:1016-1110):
// arg_buf_allocate, tensBlck_create/construct/attach_body, cuda_task_create,
// the operation, cuda_task_wait.  Tensor bodies are the caller's host arrays,
// attached as external memory; copy controls COPY_TT / COPY_TTT move them to
// the GPU and the result back.
//
// NV-TAL calls one Fortran routine of the CPU path, get_contr_permutations
// (TALSH/tensor_algebra_cpu.F90:5613, bind(c)), for adds and contractions.  No
// Fortran compiler exists here, so it is supplied by the oracle's C++
// restatement of that routine (orc_contr_permutations in talsh_oracle.cpp),
// with the same arguments and a nonzero ierr on an invalid pattern.
// Nothing under exatensor_b200/ links or loads this library.
#include "device_algebra.h"
#include "mem_manager.h"
#include "tensor_algebra.h"

extern "C" int orc_contr_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank, const int* cptrn,
                                      int conj_bits, int* dprm, int* lprm, int* rprm, int* ncd, int* nlu, int* nru);

extern "C" void get_contr_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank, const int* cptrn,
                                       int conj_bits, int* dprm, int* lprm, int* rprm, int* ncd, int* nlu, int* nru,
                                       int* ierr) {
  *ierr = orc_contr_permutations(gemm_tl, gemm_tr, lrank, rrank, cptrn, conj_bits, dprm, lprm, rprm, ncd, nlu, nru);
}

namespace {

int g_ready = 0;

// A tensor block of the given shape whose body is an external host array.
int make_block(int dtk, int rank, const int* dims, const void* body, tensBlck_t** out) {
  tensBlck_t* t = nullptr;
  int e = tensBlck_create(&t);
  if (e) return 100 + e;
  e = tensBlck_construct(t, YEP, rank, dims);
  if (!e) e = tensBlck_attach_body(t, dtk, -1, const_cast<void*>(body));
  if (e) {
    tensBlck_destroy(t);
    return 200 + e;
  }
  *out = t;
  return 0;
}

// Waits for a scheduled task; 0 when it completed.
int finish(int sched, cudaTask_t* task) {
  int e = sched;
  if (!e) {
    const int st = cuda_task_wait(task);
    if (st != CUDA_TASK_COMPLETED) e = 1000 + cuda_task_error_code(task);
  }
  cuda_task_destroy(task);
  return e;
}

}  // namespace

extern "C" {

// NV-TAL initialisation on one GPU with a 1 GiB pinned host argument buffer.
int ref_init(int gpu) {
  if (g_ready) return 0;
  size_t host_buf = (size_t)1 << 30;
  int host_args = 0;
  const int e = arg_buf_allocate(&host_buf, &host_args, gpu, gpu);
  if (!e) g_ready = 1;
  return e;
}

// d = permute(l) (o2n: input dimension i goes to output position o2n[i]).
int ref_copy(int dtk, int rank, const int* ldims, const int* o2n, const void* l, void* d, int conj_bits) {
  if (!g_ready) return -1;
  int ddims[MAX_TENSOR_RANK];
  for (int i = 0; i < rank; ++i) ddims[o2n[i] - 1] = ldims[i];
  tensBlck_t *lt = nullptr, *dt = nullptr;
  int e = make_block(dtk, rank, ldims, l, &lt);
  if (!e) e = make_block(dtk, rank, ddims, d, &dt);
  cudaTask_t* task = nullptr;
  if (!e) e = cuda_task_create(&task);
  if (!e) e = finish(gpu_tensor_block_copy(o2n, lt, dt, COPY_TT, task, 0, conj_bits), task);
  if (lt) tensBlck_destroy(lt);
  if (dt) tensBlck_destroy(dt);
  return e;
}

// d += scale * permute(l).
int ref_add(int dtk, int rank, const int* ldims, const int* o2n, void* d, const void* l, double sr, double si,
            int conj_bits) {
  if (!g_ready) return -1;
  int ddims[MAX_TENSOR_RANK];
  for (int i = 0; i < rank; ++i) ddims[o2n[i] - 1] = ldims[i];
  tensBlck_t *lt = nullptr, *dt = nullptr;
  int e = make_block(dtk, rank, ldims, l, &lt);
  if (!e) e = make_block(dtk, rank, ddims, d, &dt);
  cudaTask_t* task = nullptr;
  if (!e) e = cuda_task_create(&task);
  if (!e) e = finish(gpu_tensor_block_add(o2n, lt, dt, COPY_TT, task, 0, sr, si, conj_bits), task);
  if (lt) tensBlck_destroy(lt);
  if (dt) tensBlck_destroy(dt);
  return e;
}

// d = beta * d + scale * l * r by the digital pattern cptrn (beta = 1 when accumulative).
int ref_contract(const int* cptrn, int dtk, int drank, const int* ddims, void* d, int lrank, const int* ldims,
                 const void* l, int rrank, const int* rdims, const void* r, double sr, double si, int conj_bits,
                 int accumulative) {
  if (!g_ready) return -1;
  tensBlck_t *lt = nullptr, *rt = nullptr, *dt = nullptr;
  int e = make_block(dtk, lrank, ldims, l, &lt);
  if (!e) e = make_block(dtk, rrank, rdims, r, &rt);
  if (!e) e = make_block(dtk, drank, ddims, d, &dt);
  cudaTask_t* task = nullptr;
  if (!e) e = cuda_task_create(&task);
  if (!e)
    e = finish(gpu_tensor_block_contract_dlf(cptrn, lt, rt, dt, COPY_TTT, task, 0, sr, si, conj_bits, accumulative),
               task);
  if (lt) tensBlck_destroy(lt);
  if (rt) tensBlck_destroy(rt);
  if (dt) tensBlck_destroy(dt);
  return e;
}

}  // extern "C"
