/* talsh_b200.h -- device-level C ABI of the B200 tensor-algebra library.
 *
 * These entry points replace TAL-SH's NV-TAL device calls
 * (TALSH/device_algebra.h:259-273, implemented in
 * TALSH/tensor_algebra_gpu_nvidia.cu) with plain pointers and sizes: device
 * pointers to dense tensor bodies in TAL-SH's "dlf" layout (dimension 1 is
 * the fastest, complex numbers interleaved), extents as int arrays, digital
 * index patterns exactly as get_contr_pattern_dig produces them
 * (TALSH/tensor_algebra_cpu.F90:5307), the TAL-SH data kinds R4=4, R8=8,
 * C4=14, C8=18, and an optional cudaStream_t passed as void* (NULL = the
 * legacy default stream).  Every call is asynchronous on that stream unless
 * stated otherwise and returns 0 on success or a TB_ERR_* code; nothing falls
 * back to the host.
 *
 * The talsh.h API (include/talsh.h) is built on top of these calls.
 */
#ifndef TALSH_B200_H_
#define TALSH_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (0 = success). */
#define TB_SUCCESS 0
#define TB_ERR_INVALID_ARGS 1     /* bad pointer, rank, extent, data kind or pattern */
#define TB_ERR_PATTERN 2          /* malformed symbolic or digital index pattern */
#define TB_ERR_CUDA 3             /* CUDA runtime error (see tb_last_error) */
#define TB_ERR_NOT_IMPLEMENTED 4  /* valid request this library does not execute */
#define TB_ERR_DEVICE 5           /* a kernel recorded a device-side error */
#define TB_ERR_NO_MEMORY 6        /* scratch allocation failed (maps to TRY_LATER) */
#define TB_ERR_LIMIT 7            /* request exceeds a documented limit */

/* Contraction methods. */
#define TB_METHOD_AUTO 0      /* plan selector decides */
#define TB_METHOD_TTGT 1      /* plain: permute, GEMM in the tensor's own type, permute back */
#define TB_METHOD_FUSED 2     /* tensor cores: fused gather/epilogue; split-BF16 (R4/C4), modular
                                 residues or INT8 slices (R8/C8) */

/* Contraction plan (all-zero = automatic). */
typedef struct {
  int method;      /* TB_METHOD_* */
  int slices;      /* INT8 slices per FP64 operand for R8/C8 fused (0 = default) */
  int tile_n;      /* tensor-core N tile: 0 (default), 128 or 256 */
  int bf16_terms;  /* split-BF16 products for R4/C4 fused: 0 (default = 3) */
  int tile_m;      /* tensor-core M tile: 0 (default), 128 (one SM) or 256 (an SM pair) */
  int moduli;      /* R8/C8 fused: 0 (default) = modular residues (Ozaki scheme II) where the
                      contraction allows, with the fewest moduli that keep 46 bits per operand;
                      8..15 = that many moduli; -1 = INT8 slices (Ozaki scheme I) instead.
                      A positive `slices` also selects INT8 slices. */
  int reserved[2];
} tb_plan_t;

/* Last error message of the calling thread ("" if none). */
const char* tb_last_error(void);

/* Number of kernels this library has launched in the process (all threads). */
long long tb_launch_count(void);

/* Opt-in CUDA-event timing of the dominant GEMM kernel launches made by the
 * calling thread (events on the launching stream).  tb_timing_read
 * synchronises on the recorded events, returns their summed duration and
 * count, and clears the record. */
int tb_timing_enable(int on);
int tb_timing_read(double* total_ms, int* count);

/* Select and initialise a GPU for the calling thread (kind-specific id). */
int tb_device_init(int gpu);
/* Reads and clears the device-side error word; returns TB_ERR_DEVICE if set. */
int tb_device_check(void* stream);

/* Valid data kind -> element size in bytes (0 if invalid). */
int tb_data_kind_size(int data_kind);

/* Parse a symbolic pattern ("D(a,b)+=L(c,a)*R(c,b)") into TAL-SH's digital
 * form.  Replaces talsh_get_contr_ptrn_str2dig (TALSH/talshf.F90:619).
 * cptrn must hold 2*MAX_TENSOR_RANK ints.  rrank is -1 for unary patterns. */
int tb_parse_pattern(const char* pattern, int* cptrn, int* drank, int* lrank, int* rrank,
                     int* conj_bits);

/* out = permute(in): copy with an O2N index permutation given as the digital
 * copy pattern (1-based, cptrn[i] = destination position of input dim i).
 * conj_bits bit0 (D) xor bit1 (L) conjugates complex data.  Bit-exact.
 * The first copy of 32 MB or more with a given shape, permutation and
 * element size times a few plans on the stream and waits for them (one host
 * synchronisation per shape; not while the stream is capturing; the copy is
 * done when it returns); later calls are asynchronous.  TB_PERM_TUNE=0
 * turns that off.
 * Replaces gpu_tensor_block_copy (TALSH/tensor_algebra_gpu_nvidia.cu:4806;
 * kernel gpu_tensor_block_copy_dlf__ :1126). */
int tb_tensor_copy(int data_kind, int rank, const int* in_dims, const int* cptrn,
                   const void* in, void* out, int conj_bits, void* stream);

/* Naive one-element-per-thread scatter permutation (the reference's
 * gpu_tensor_block_copy_scatter_dlf__, :2173).  Same result as tb_tensor_copy. */
int tb_tensor_copy_scatter(int data_kind, int rank, const int* in_dims, const int* cptrn,
                           const void* in, void* out, int conj_bits, void* stream);

/* d = d + permute(l) * scale, one fused pass, bit-exact against the
 * reference's permute-then-add (two roundings, no FMA).  l_dims are the
 * extents of l; cptrn is the digital addition pattern (O2N, 1-based).
 * Replaces gpu_tensor_block_add (TALSH/tensor_algebra_gpu_nvidia.cu:5203). */
int tb_tensor_add(int data_kind, int rank, const int* l_dims, const int* cptrn, void* d,
                  const void* l, double scale_real, double scale_imag, int conj_bits,
                  void* stream);

/* d = value (gpu_tensor_block_init, :4262). */
int tb_tensor_init(int data_kind, size_t volume, void* d, double val_real, double val_imag,
                   void* stream);

/* d = d * scale (gpu_tensor_block_scale, :4525). */
int tb_tensor_scale(int data_kind, size_t volume, void* d, double scale_real,
                    double scale_imag, void* stream);

/* Deterministic norms: which = 1 -> sum |x|, which = 2 -> sum |x|^2, written
 * to *result (host memory); this call synchronises the stream.  Device-side
 * counterpart of talshTensorImageNorm1_cpu (TALSH/talshc.cpp:6207). */
int tb_tensor_norm(int data_kind, size_t volume, const void* d, int which, double* result,
                   void* stream);

/* Tensor contraction D = beta*D + alpha * op(L) * op(R) with beta = 1 when
 * accumulative != 0, else 0.  cptrn is the digital contraction pattern
 * (lrank+rrank entries), conj_bits bit0 D, bit1 L, bit2 R.  plan may be
 * NULL (TB_METHOD_AUTO).  With AUTO, a large contraction (>= 2^34 FLOP) whose
 * shape comes back may, on its second call, time candidate plans with
 * alpha = 0, beta = 1 and wait for them (one host synchronisation per
 * shape; not while the stream is capturing) before running the fastest.
 * Replaces gpu_tensor_block_contract_dlf
 * (TALSH/tensor_algebra_gpu_nvidia.cu:5847). */
int tb_tensor_contract(const int* cptrn, int data_kind, int drank, const int* d_dims, void* d,
                       int lrank, const int* l_dims, const void* l, int rrank,
                       const int* r_dims, const void* r, double alpha_real, double alpha_imag,
                       int conj_bits, int accumulative, const tb_plan_t* plan, void* stream);

/* Contraction with a symbolic pattern (parses, then tb_tensor_contract). */
int tb_tensor_contract_str(const char* pattern, int data_kind, int drank, const int* d_dims,
                           void* d, int lrank, const int* l_dims, const void* l, int rrank,
                           const int* r_dims, const void* r, double alpha_real,
                           double alpha_imag, int accumulative, const tb_plan_t* plan,
                           void* stream);

/* Size of the static per-device scratch array of tb_tensor_contract_noalloc. */
#define TB_NOALLOC_ARENA_BYTES (64ull << 20)

/* Plain (TTGT) contraction that allocates no memory.  It has no counterpart in
 * the reference, whose contractions always draw their scratch from TAL-SH's
 * device buffer pool.  It is for callers that may not allocate device memory
 * while they run: code that has reserved all device memory up front, or that
 * runs where an allocation would synchronise the device or is not permitted.
 * Arguments and results are those of tb_tensor_contract, with the method
 * fixed to TTGT (permute, GEMM in the tensor's own type, permute back).
 *   - The permuted copies of L and R, the product matrix and the dot-product
 *     partials live in one static device array of TB_NOALLOC_ARENA_BYTES,
 *     which every GPU that loads this library holds until the process exits.
 *     A contraction whose (M*K + N*K + M*N) * element size, each term rounded
 *     up to 256 bytes, exceeds it is rejected with TB_ERR_LIMIT before any
 *     work is queued; tb_tensor_contract has no such limit.
 *   - tb_device_init must have run on the device first (it creates the
 *     device error word this call reports through); else TB_ERR_INVALID_ARGS.
 *   - The first call on each device looks up the array's device address (and
 *     may load the library's GPU code there); make that first call before any
 *     stream capture.
 *   - Every call uses the same array and finds the previous call's data in
 *     it.  Calls queued on one stream run in order and are safe; calls that
 *     can overlap on the GPU (different streams, other host threads) race. */
int tb_tensor_contract_noalloc(const int* cptrn, int data_kind, int drank, const int* d_dims,
                               void* d, int lrank, const int* l_dims, const void* l, int rrank,
                               const int* r_dims, const void* r, double alpha_real,
                               double alpha_imag, int conj_bits, int accumulative, void* stream);

/* ---- block-sparse contractions -------------------------------------------
 * A block-sparse contraction is a list of block tasks D_blk += alpha * L_blk *
 * R_blk under one index pattern; tasks with the same d pointer add into the
 * same output block.  ExaTENSOR's TAVP-WRK runs such lists as one
 * talsh_tensor_contract per block (INTERVIRT/tavp_worker.F90:9420-9518, call
 * at :9467); these calls run the whole list as one grouped tensor-core
 * launch (R8: INT8 slices, R4: split BF16), replayed from a CUDA graph. */
typedef struct {
  void* d;           /* output block body (device, dlf) */
  const void* l;     /* left operand block body */
  const void* r;     /* right operand block body */
  int d_dims[8];     /* extents; ranks come from the pattern (<= 8) */
  int l_dims[8];
  int r_dims[8];
} tb_block_task_t;

typedef struct tb_bsc_plan_s tb_bsc_plan_t;

typedef struct {
  int tasks, left_blocks, right_blocks, out_blocks, work_items;
  int slices;        /* INT8 slices (R8) */
  int tile_n;        /* GEMM N tile */
  double flops;      /* sum of 2*M*N*K over the tasks */
  float tune_ms[4];  /* autotuner timings: (tile 128, 6 slices), (128, 7), (256, 6), (256, 7) */
} tb_bsc_info_t;

/* Builds the plan: distinct operand blocks, offset tables, tensor maps and the
 * work list (device memory owned by the plan; blocks must stay allocated).
 * beta = accumulative ? 1 : 0 applies to every output block once per execution.
 * plan may set slices (R8, 2..7, default 6; planes are allocated for
 * max(slices, 6)) and tile_n (128 or 256). */
int tb_bsc_plan_create(const char* pattern, int data_kind, int ntasks, const tb_block_task_t* tasks,
                       double alpha_real, double alpha_imag, int accumulative, const tb_plan_t* plan,
                       tb_bsc_plan_t** out, void* stream);
/* Runs the contraction on stream: operand conversion + one grouped GEMM,
 * captured into a CUDA graph on the first call and replayed afterwards. */
int tb_bsc_execute(tb_bsc_plan_t* plan, void* stream);
/* The same launches queued directly on the stream (no graph). */
int tb_bsc_execute_stream(tb_bsc_plan_t* plan, void* stream);
/* Times the tile-width candidates (and 6 vs 7 slices when the planes hold 7)
 * on the plan's data, with alpha = 0 and beta = 1 so that D is unchanged, and
 * keeps the fastest. */
int tb_bsc_autotune(tb_bsc_plan_t* plan, void* stream);
int tb_bsc_plan_info(const tb_bsc_plan_t* plan, tb_bsc_info_t* info);
int tb_bsc_plan_destroy(tb_bsc_plan_t* plan);

/* Diagnostic of the calling thread's last talshTensorContractXL: the D
 * dimension its output was decomposed along and the number of slabs, or -1
 * and 0 when it ran undecomposed. */
int tb_xl_last_split(int* d_dim, int* slabs);

/* ---- block-task lists from segment metadata --------------------------------
 * A block-sparse tensor splits index k into nseg[k] segments of extents
 * seg_ext (all indices' segments concatenated, index 0 first); a present block
 * is one segment number per index (keys, nblocks x rank, index 0 first) with
 * its dense body (dlf layout) in device memory. */
typedef struct {
  int rank;
  const int* nseg;       /* [rank] */
  const int* seg_ext;    /* [sum of nseg] */
  int nblocks;
  const int* keys;       /* [nblocks][rank] */
  void* const* bodies;   /* [nblocks] */
} tb_block_list_t;

/* The block tasks of the contraction `pattern` over block-sparse D, L and R:
 * every (L block, R block) pair whose contracted segments agree, with the D
 * block their uncontracted segments name (pairs whose D block is absent give
 * no task).  Replaces the matching of TensContractionSplitFunc
 * (INTRAVIRT/tensor_recursive.F90:9202-9784), whose sub-contraction list
 * TAVP-WRK executes block by block (INTERVIRT/tavp_worker.F90:9420).  Writes
 * at most max_tasks tasks and the total count to *ntasks; tasks = NULL,
 * max_tasks = 0 only counts.  Errors: segmentations that differ between the
 * tensors carrying an index, out-of-range segment numbers, repeated D keys
 * (TB_ERR_INVALID_ARGS); too small an array (TB_ERR_LIMIT, *ntasks = the
 * count).  Host code only: no device work. */
int tb_bsc_tasks_from_blocks(const char* pattern, const tb_block_list_t* d, const tb_block_list_t* l,
                             const tb_block_list_t* r, int max_tasks, tb_block_task_t* tasks, int* ntasks);

/* ---- caller-side batching ------------------------------------------------
 * Collects block contractions (one pattern, data kind, alpha and
 * accumulation) that a caller would issue one by one -- TAVP-WRK's
 * talsh_tensor_contract per block (INTERVIRT/tavp_worker.F90:9467) -- and
 * runs them at flush time as one grouped launch (R8, R4: tb_bsc_plan_create
 * and tb_bsc_execute), or as a loop of tb_tensor_contract_str calls for the
 * data kinds the grouped kernel does not take.  A flushed list equal to one
 * flushed before (same tasks, same order) reuses its plan and CUDA graph; on
 * its second use the plan's tile and slice choice is timed once.  The
 * accumulative flag applies to each output block once per flush.  Blocks
 * must stay allocated while a cached plan may run them. */
typedef struct tb_batch_s tb_batch_t;
typedef struct {
  long long tasks;         /* tasks flushed */
  int grouped_flushes, loop_flushes, plans_built, plan_reuses, autotunes, cached_plans;
} tb_batch_stats_t;
int tb_batch_create(const char* pattern, int data_kind, double alpha_real, double alpha_imag, int accumulative,
                    const tb_plan_t* plan, tb_batch_t** out);
int tb_batch_add(tb_batch_t* batch, int ntasks, const tb_block_task_t* tasks);
/* Tasks queued since the last flush (-1 for a null batch). */
int tb_batch_pending(const tb_batch_t* batch);
int tb_batch_flush(tb_batch_t* batch, void* stream);
int tb_batch_get_stats(const tb_batch_t* batch, tb_batch_stats_t* stats);
/* Destroys the cached plans (after the device finishes their work). */
int tb_batch_destroy(tb_batch_t* batch);

/* ---- learned plan selection ---------------------------------------------
 * No counterpart in the reference, which always runs TTGT through cuBLAS.
 * A contraction descriptor (TB_DESC_FEATURES floats) feeds a 3-layer MLP that
 * predicts the log-runtime of each candidate plan: 0 TTGT; tensor cores with
 * 1 the 128-wide N tile, 2 the 256-wide N tile, 3 the 256-wide tile on SM
 * pairs (256-row tiles), 4 the 256-wide tile with 6 INT8 slices instead of
 * modular residues (FP64 data only).  TB_METHOD_AUTO then takes the fastest
 * predicted plan.  Every candidate meets the accuracy bounds, so the choice
 * changes speed, not what is computed beyond those bounds. */
#define TB_DESC_FEATURES 16
#define TB_SELECT_PLANS 5

/* Descriptor of a contraction (host only, no GPU work). */
int tb_contract_descriptor(const int* cptrn, int data_kind, int drank, const int* d_dims, int lrank,
                           const int* l_dims, int rrank, const int* r_dims, float* features);

/* The network: hand-written CUDA forward, backward (deterministic) and Adam
 * kernels.  Parameters are W1 b1 W2 b2 W3 b3 with W_l stored [in][out]. */
typedef struct tb_mlp_s tb_mlp_t;
int tb_mlp_create(int n_in, int n_hidden, int n_out, int max_batch, uint64_t seed, tb_mlp_t** out);
int tb_mlp_destroy(tb_mlp_t* net);
long long tb_mlp_num_params(const tb_mlp_t* net);
int tb_mlp_get_params(const tb_mlp_t* net, float* host, int grads);  /* grads != 0: last gradients */
int tb_mlp_set_params(tb_mlp_t* net, const float* host);
/* y[batch][n_out] = net(x[batch][n_in]); device pointers, asynchronous. */
int tb_mlp_forward(tb_mlp_t* net, const float* x, int batch, float* y, void* stream);
/* Mean squared error over the labelled targets (NaN = unlabelled) and its
 * gradients for one batch (<= max_batch); *loss (host) if non-NULL syncs. */
int tb_mlp_backward(tb_mlp_t* net, const float* x, const float* targets, int batch, float* loss, void* stream);
int tb_mlp_adam_step(tb_mlp_t* net, float lr, float beta1, float beta2, float eps, void* stream);

/* Installs a trained selector for TB_METHOD_AUTO: the parameters of a
 * (TB_DESC_FEATURES -> hidden -> hidden -> TB_SELECT_PLANS) network and the
 * feature normalisation (x - mean) / scale.  params = NULL removes it (the
 * rule-based choice returns).  margin: when other plans' predictions lie
 * within this of the best (in natural-log units), autotune != 0 and the
 * contraction is large (about 1.7e10 FLOP or more), the second call with the
 * same descriptor times those plans (alpha = 0, beta = 1 runs, D unchanged)
 * and caches the winner; one-off shapes keep the prediction. */
int tb_selector_install(int n_hidden, const float* params, const float* mean, const float* scale, float margin,
                        int autotune);
/* The selector's choice for a descriptor: plan index (as listed above; plan 4
 * only for FP64 descriptors) and the predicted log-runtimes (may be NULL). */
int tb_selector_choose(const float* features, float* predicted);
/* Host time of one selection (descriptor already built), averaged over iters
 * calls of the inference that TB_METHOD_AUTO runs; -1 without a selector. */
int tb_selector_time(const float* features, int iters, double* us_per_call);
/* Installs a selector from a weights file ("TBSEL001" header, features,
 * hidden, outputs, margin, autotune, mean, scale, parameters).  tb_device_init
 * loads selector_weights.bin from the library's directory when present
 * (TB_SELECTOR=0 disables this, TB_SELECTOR=<path> names another file). */
int tb_selector_load(const char* path);

/* Seeded U[lo,hi) fill on the device (splitmix64 stream, 53-bit fractions);
 * complex kinds fill real and imaginary parts from consecutive draws. */
int tb_fill_uniform(int data_kind, size_t volume, void* d, uint64_t seed, double lo, double hi,
                    void* stream);

/* Statistics of the last tb_tensor_contract on this thread. */
typedef struct {
  int method;        /* TB_METHOD_TTGT or TB_METHOD_FUSED actually executed */
  int slices;        /* INT8 slices (R8/C8 fused) */
  int passes;        /* accumulator passes of the tensor-core GEMM */
  int gemm_launches; /* GEMM kernel launches */
  long long m, n, k; /* matricized sizes (real-expanded for complex on tensor cores) */
  double flops;      /* 2*M*N*K (real) or 8*M*N*K (complex), the reference's accounting */
  int products;      /* plane products the tensor-core GEMM ran (INT8 slice pairs or BF16
                        terms); its tensor-core work is products * flops */
  int tile_n;        /* tensor-core N tile of the executed plan */
  int tile_m;        /* tensor-core M tile: 128 (one SM) or 256 (an SM pair, cta_group::2) */
  int moduli;        /* R8/C8 fused with modular residues: moduli (one INT8 GEMM each); 0 otherwise */
  int residue_bits;  /* ... and the bits p kept per operand (|X| <= 2^p) */
} tb_contract_stats_t;
int tb_last_contract_stats(tb_contract_stats_t* stats);

/* Tensor-core throughput probes (diagnostics; no counterpart in the
 * reference, which has no tensor-core code): the rooflines of the
 * contraction kernels, measured on this GPU.  Each runs `iters` MMAs per
 * issuing unit with operands resident on chip (no global memory traffic)
 * once untimed, then once between CUDA events on `stream`, synchronizes, and
 * returns the rate in operations per second (2*M*N*K per MMA) and the timed
 * launch's milliseconds (ms may be NULL).
 *   TB_PEAK_I8    tcgen05.mma kind::i8, M 128 x N 256 x K 32, one CTA per SM
 *   TB_PEAK_BF16  tcgen05.mma kind::f16 with BF16 inputs, M 128 x N 256 x K 16
 *   TB_PEAK_F64   mma.sync m8n8k4 FP64 (DMMA), four chains per warp */
#define TB_PEAK_I8 1
#define TB_PEAK_BF16 2
#define TB_PEAK_F64 3
int tb_peak_measure(int kind, long long iters, double* ops_per_s, double* ms, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TALSH_B200_H_ */
