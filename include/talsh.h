/* talsh.h -- TAL-SH user-level C API served by the B200 library.
 *
 * Drop-in subset of the reference's TALSH/talsh.h (:143-596) for the
 * single-process tensor-algebra path: tensors with host and GPU images,
 * tasks, and the Init/Scale/Copy/Add/Contract operations with TAL-SH's index
 * pattern strings and copy-control semantics.  Declarations, return codes and
 * argument meanings follow the reference; each group cites the reference
 * declaration it replaces.  Operations execute on NVIDIA GPUs only: a request
 * for the Host device returns TALSH_NOT_AVAILABLE (there is no CPU path).
 */
#ifndef TALSH_H_
#define TALSH_H_

#include "tensor_algebra.h"

#define TALSH_MAX_DEV_PRESENT 16

/* Error codes (TALSH/talsh.h:26-41) */
#define TALSH_SUCCESS 0
#define TALSH_FAILURE -666
#define TALSH_NOT_AVAILABLE -888
#define TALSH_NOT_IMPLEMENTED -999
#define TALSH_NOT_INITIALIZED 1000000
#define TALSH_ALREADY_INITIALIZED 1000001
#define TALSH_INVALID_ARGS 1000002
#define TALSH_INTEGER_OVERFLOW 1000003
#define TALSH_OBJECT_NOT_EMPTY 1000004
#define TALSH_OBJECT_IS_EMPTY 1000005
#define TALSH_IN_PROGRESS 1000006
#define TALSH_NOT_ALLOWED 1000007
#define TALSH_LIMIT_EXCEEDED 1000008
#define TALSH_NOT_FOUND 1000009
#define TALSH_OBJECT_BROKEN 1000010
#define TALSH_INVALID_REQUEST 1000011

/* Task status (TALSH/talsh.h:43-50) */
#define TALSH_TASK_ERROR 1999999
#define TALSH_TASK_EMPTY 2000000
#define TALSH_TASK_SCHEDULED 2000001
#define TALSH_TASK_STARTED 2000002
#define TALSH_TASK_INPUT_READY 2000003
#define TALSH_TASK_OUTPUT_READY 2000004
#define TALSH_TASK_COMPLETED 2000005

/* Dense tensor with images on several devices (TALSH/talsh.h:87-94) */
typedef struct {
  talsh_tens_shape_t* shape_p;
  talsh_dev_rsc_t* dev_rsc;
  int* data_kind;
  int* avail;
  int dev_rsc_len;
  int ndev;
} talsh_tens_t;

typedef struct {
  talsh_tens_t* tens_p;
  int source_image;
} talshTensArg_t;

/* Task handle (TALSH/talsh.h:110-121) */
typedef struct {
  void* task_p;
  int task_error;
  int dev_kind;
  int data_kind;
  int coherence;
  int num_args;
  talshTensArg_t tens_args[MAX_TENSOR_OPERANDS];
  double data_vol;
  double flops;
  double exec_time;
} talsh_task_t;

#ifdef __cplusplus
extern "C" {
#define TALSH_DEF(x) = x
#else
#define TALSH_DEF(x)
#endif

/* Control (TALSH/talsh.h:150-166) */
int talshValidDataKind(int datk, int* datk_size);
int talshInit(size_t* host_buf_size, int* host_arg_max, int ngpus, int gpu_list[], int nmics, int mic_list[],
              int namds, int amd_list[]);
int talshShutdown(void);
/* Fast math selects the tensor-core (split-BF16 / INT8-slice) contraction form */
int talshEnableFastMath(int dev_kind, int dev_id TALSH_DEF(DEV_DEFAULT));
int talshDisableFastMath(int dev_kind, int dev_id TALSH_DEF(DEV_DEFAULT));
int talshQueryFastMath(int dev_kind, int dev_id);
int talshDeviceCount(int dev_kind, int* dev_count);
int talshFlatDevId(int dev_kind, int dev_num);
int talshKindDevId(int dev_id, int* dev_kind);
size_t talshDeviceMemorySize(int dev_num, int dev_kind TALSH_DEF(DEV_NULL));
double talshDeviceGetFlops(int dev_kind TALSH_DEF(DEV_DEFAULT), int dev_id TALSH_DEF(DEV_DEFAULT));
int talshStats(int dev_id TALSH_DEF(-1), int dev_kind TALSH_DEF(DEV_NULL));

/* Tensor blocks (TALSH/talsh.h:232-314) */
int talshTensorCreate(talsh_tens_t** tens_block);
int talshTensorClean(talsh_tens_t* tens_block);
int talshTensorIsEmpty(const talsh_tens_t* tens_block);
int talshTensorConstruct(talsh_tens_t* tens_block, int data_kind, int tens_rank, const int tens_dims[],
                         int dev_id TALSH_DEF(0), void* ext_mem TALSH_DEF(NULL), int in_hab TALSH_DEF(-1),
                         talsh_tens_init_i init_method TALSH_DEF(NULL), double init_val_real TALSH_DEF(0.0),
                         double init_val_imag TALSH_DEF(0.0));
int talshTensorConstruct_(talsh_tens_t* tens_block, int data_kind, int tens_rank, const int tens_dims[], int dev_id,
                          void* ext_mem, int in_hab, talsh_tens_init_i init_method, double init_val_real,
                          double init_val_imag);
int talshTensorImportData(talsh_tens_t* tens_block, int data_kind, const void* ext_data);
int talshTensorDestruct(talsh_tens_t* tens_block);
int talshTensorDestroy(talsh_tens_t* tens_block);
int talshTensorRank(const talsh_tens_t* tens_block);
size_t talshTensorVolume(const talsh_tens_t* tens_block);
size_t talshTensorSizeAllImages(const talsh_tens_t* tens_block, int* num_images);
const int* talshTensorDimExtents(const talsh_tens_t* tens_block, int* rank);
int talshTensorDataKind(const talsh_tens_t* tens_block, int* num_images, int* data_kinds);
int talshTensorInUse(const talsh_tens_t* tens_block);
int talshTensorPresence(const talsh_tens_t* tens_block, int* ncopies, int copies[], int data_kinds[],
                        int dev_kind TALSH_DEF(DEV_NULL), int dev_id TALSH_DEF(-1));
int talshTensorGetBodyAccess(talsh_tens_t* tens_block, void** body_p, int data_kind, int dev_id,
                             int dev_kind TALSH_DEF(DEV_NULL));
int talshTensorGetBodyAccessConst(const talsh_tens_t* tens_block, const void** body_p, int data_kind, int dev_id,
                                  int dev_kind TALSH_DEF(DEV_NULL));
int talshTensorGetScalar(talsh_tens_t* tens_block, double* scalar_real, double* scalar_imag);

/* Tasks (TALSH/talsh.h:331-369) */
int talshTaskCreate(talsh_task_t** talsh_task);
int talshTaskClean(talsh_task_t* talsh_task);
int talshTaskIsEmpty(const talsh_task_t* talsh_task);
int talshTaskDestruct(talsh_task_t* talsh_task);
int talshTaskDestroy(talsh_task_t* talsh_task);
int talshTaskDevId(talsh_task_t* talsh_task, int* dev_kind TALSH_DEF(NULL));
int talshTaskStatus(talsh_task_t* talsh_task);
int talshTaskComplete(talsh_task_t* talsh_task, int* stats, int* ierr);
int talshTaskWait(talsh_task_t* talsh_task, int* stats);
int talshTasksWait(int ntasks, talsh_task_t talsh_tasks[], int stats[]);
int talshTaskTime(talsh_task_t* talsh_task, double* total, double* comput TALSH_DEF(NULL),
                  double* input TALSH_DEF(NULL), double* output TALSH_DEF(NULL), double* mmul TALSH_DEF(NULL));

/* Placement (TALSH/talsh.h:427-451) */
int talshTensorPlace(talsh_tens_t* tens, int dev_id, int dev_kind TALSH_DEF(DEV_NULL), void* dev_mem TALSH_DEF(NULL),
                     int copy_ctrl TALSH_DEF(COPY_M), talsh_task_t* talsh_task TALSH_DEF(NULL));
int talshTensorDiscard(talsh_tens_t* tens, int dev_id, int dev_kind TALSH_DEF(DEV_NULL));
int talshTensorDiscardOther(talsh_tens_t* tens, int dev_id, int dev_kind TALSH_DEF(DEV_NULL));

/* Operations (TALSH/talsh.h:452-541) */
int talshTensorInit(talsh_tens_t* dtens, double val_real, double val_imag, int dev_id TALSH_DEF(DEV_DEFAULT),
                    int dev_kind TALSH_DEF(DEV_DEFAULT), int copy_ctrl TALSH_DEF(COPY_M),
                    talsh_task_t* talsh_task TALSH_DEF(NULL));
int talshTensorScale(talsh_tens_t* dtens, double val_real, double val_imag, int dev_id TALSH_DEF(DEV_DEFAULT),
                     int dev_kind TALSH_DEF(DEV_DEFAULT), int copy_ctrl TALSH_DEF(COPY_M),
                     talsh_task_t* talsh_task TALSH_DEF(NULL));
int talshTensorCopy(const char* cptrn, talsh_tens_t* dtens, talsh_tens_t* ltens, int dev_id TALSH_DEF(DEV_DEFAULT),
                    int dev_kind TALSH_DEF(DEV_DEFAULT), int copy_ctrl TALSH_DEF(COPY_MT),
                    talsh_task_t* talsh_task TALSH_DEF(NULL));
int talshTensorAdd(const char* cptrn, talsh_tens_t* dtens, talsh_tens_t* ltens, double scale_real TALSH_DEF(1.0),
                   double scale_imag TALSH_DEF(0.0), int dev_id TALSH_DEF(DEV_DEFAULT),
                   int dev_kind TALSH_DEF(DEV_DEFAULT), int copy_ctrl TALSH_DEF(COPY_MT),
                   talsh_task_t* talsh_task TALSH_DEF(NULL));
int talshTensorContract(const char* cptrn, talsh_tens_t* dtens, talsh_tens_t* ltens, talsh_tens_t* rtens,
                        double scale_real TALSH_DEF(1.0), double scale_imag TALSH_DEF(0.0),
                        int dev_id TALSH_DEF(DEV_DEFAULT), int dev_kind TALSH_DEF(DEV_DEFAULT),
                        int copy_ctrl TALSH_DEF(COPY_MTT), int accumulative TALSH_DEF(YEP),
                        talsh_task_t* talsh_task TALSH_DEF(NULL));
int talshTensorContractXL(const char* cptrn, talsh_tens_t* dtens, talsh_tens_t* ltens, talsh_tens_t* rtens,
                          double scale_real TALSH_DEF(1.0), double scale_imag TALSH_DEF(0.0),
                          int dev_id TALSH_DEF(DEV_DEFAULT), int dev_kind TALSH_DEF(DEV_DEFAULT),
                          int accumulative TALSH_DEF(YEP));

/* Debugging: 1-norm of the Host image (TALSH/talsh.h:594) */
double talshTensorImageNorm1_cpu(const talsh_tens_t* talsh_tens);

#ifdef __cplusplus
}
#endif

#endif /* TALSH_H_ */
