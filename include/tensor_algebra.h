/* tensor_algebra.h -- TAL-SH constants and interoperable types used by talsh.h.
 *
 * Values and struct layouts are those of the reference's
 * TALSH/tensor_algebra.h (data kinds :67-72, device kinds :75-86, aliases
 * :94-112, coherence control :119-203, types :206-250) so that existing
 * callers compile against this library unchanged.  The dense layout is
 * "dlf": dimension 1 is the fastest, complex numbers are interleaved.
 */
#ifndef TENSOR_ALGEBRA_H_
#define TENSOR_ALGEBRA_H_

#include <stddef.h>
#include <stdint.h>

#define MAX_TENSOR_RANK 56
#define MAX_TENSOR_OPERANDS 4
#define MAX_CONTRACTION_PATTERN_LEN 1024
#define MAX_MLNDS_PER_TENS 4

/* Data kinds */
#define NO_TYPE 0
#define R4 4
#define R8 8
#define C4 14
#define C8 18

/* Device kinds and flat device numbering: Host {0}, NVIDIA GPU {1..8}, ... */
#define MAX_GPUS_PER_NODE 8
#define MAX_MICS_PER_NODE 8
#define MAX_AMDS_PER_NODE 8
#define DEV_NULL -1
#define DEV_DEFAULT DEV_NULL
#define DEV_HOST 0
#define DEV_NVIDIA_GPU 1
#define DEV_INTEL_MIC 2
#define DEV_AMD_GPU 3
#define DEV_MAX (1 + MAX_GPUS_PER_NODE + MAX_MICS_PER_NODE + MAX_AMDS_PER_NODE)

/* Aliases */
#define NOPE 0
#define YEP 1
#define DEVICE_UNABLE -546372819
#define TRY_LATER -918273645
#define NOT_CLEAN -192837465

/* Coherence (copy) control: two bits per argument, D most senior.
 * D: discard the argument everywhere after the task; M: discard it from the
 * source device if that differs from the execution device; T: discard it from
 * the execution device if that differs from the source device; K: keep both. */
#define COPY_D 0
#define COPY_M 1
#define COPY_T 2
#define COPY_K 3
#define COPY_DD 0
#define COPY_DM 1
#define COPY_DT 2
#define COPY_DK 3
#define COPY_MD 4
#define COPY_MM 5
#define COPY_MT 6
#define COPY_MK 7
#define COPY_TD 8
#define COPY_TM 9
#define COPY_TT 10
#define COPY_TK 11
#define COPY_KD 12
#define COPY_KM 13
#define COPY_KT 14
#define COPY_KK 15
#define COPY_DDD 0
#define COPY_MMM 21
#define COPY_MMT 22
#define COPY_MTT 26
#define COPY_MKK 31
#define COPY_TTT 42
#define COPY_TTK 43
#define COPY_KKK 63

typedef struct {
  int num_dim;       /* rank (>=0), -1: empty */
  size_t* offsets;
} talsh_tens_signature_t;

typedef struct {
  int num_dim;       /* rank (>=0), -1: empty */
  int* dims;         /* extents */
  int* divs;         /* dividers (not used by this library) */
  int* grps;         /* groups (not used by this library) */
} talsh_tens_shape_t;

typedef struct {
  void* base;
  size_t volume;
  int data_kind;
} talsh_tens_data_t;

typedef struct {
  int dev_id;        /* flat device id, -1: none */
  void* gmem_p;      /* body pointer on that device */
  int buf_entry;     /* -1: not in an argument buffer */
  int mem_attached;  /* 0: allocated by the library, 1: attached external memory */
} talsh_dev_rsc_t;

typedef int (*talsh_tens_init_i)(const talsh_tens_data_t* tens_data, const talsh_tens_shape_t* tens_shape,
                                 const talsh_tens_signature_t* tens_signature);

#endif /* TENSOR_ALGEBRA_H_ */
