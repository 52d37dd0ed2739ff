// talsh_api.cpp -- the talsh.h user API on top of the tb_* device calls.
//
// Mirrors TAL-SH's C dispatch layer (TALSH/talshc.cpp): tensors own up to
// TALSH_MAX_DEV_PRESENT body images (host and GPU), operations pick a source
// image per argument (talsh_choose_image_for_device, talshc.cpp:490), move
// data to the execution GPU, run the tb_* kernels on that GPU's stream and
// apply the copy-control coherence rules (tensor_algebra.h:119-203) when the
// task completes.  A NULL task makes a call blocking (talshc.cpp:5285).
// Host requests return TALSH_NOT_AVAILABLE: nothing computes on the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <vector>

#include "../../include/talsh.h"
#include "../../include/talsh_b200.h"
#include "tb_pattern.h"

namespace {

struct DevState {
  bool on = false;
  cudaStream_t stream = nullptr;
  cudaStream_t xstream = nullptr;  // host-to-device slices of streamed contractions
  bool fast_math = true;
  double flops = 0.0;
};

bool g_on = false;
int g_ngpu = 0;
DevState g_dev[MAX_GPUS_PER_NODE];
std::recursive_mutex g_mu;

struct TaskImpl {
  int gpu = -1;
  bool done = false;
  int err = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // start, inputs ready, computed, outputs ready
  std::vector<std::function<void()>> finalize;               // coherence actions after completion
};

int elem_size(int dtk) { return tb_data_kind_size(dtk); }

size_t volume_of(const talsh_tens_t* t) {
  if (!t || !t->shape_p || t->shape_p->num_dim < 0) return 0;
  size_t v = 1;
  for (int i = 0; i < t->shape_p->num_dim; ++i) v *= (size_t)t->shape_p->dims[i];
  return v;
}

int flat_gpu(int gpu) { return 1 + gpu; }
int gpu_of_flat(int flat) { return (flat >= 1 && flat <= MAX_GPUS_PER_NODE) ? flat - 1 : -1; }

int map_tb(int e) {
  switch (e) {
    case TB_SUCCESS: return TALSH_SUCCESS;
    case TB_ERR_INVALID_ARGS: case TB_ERR_PATTERN: return TALSH_INVALID_ARGS;
    case TB_ERR_NOT_IMPLEMENTED: return TALSH_NOT_IMPLEMENTED;
    case TB_ERR_NO_MEMORY: return TRY_LATER;
    case TB_ERR_LIMIT: return TALSH_LIMIT_EXCEEDED;
    default: return TALSH_FAILURE;
  }
}

// ---- images ------------------------------------------------------------------
int find_image(const talsh_tens_t* t, int flat_dev) {
  for (int i = 0; i < t->ndev; ++i)
    if (t->dev_rsc[i].dev_id == flat_dev && t->avail[i] == YEP) return i;
  return -1;
}

void free_image_memory(talsh_dev_rsc_t& r, cudaStream_t s) {
  if (!r.gmem_p || r.mem_attached) return;
  if (r.dev_id == 0) {
    cudaFreeHost(r.gmem_p);
  } else {
    const int g = gpu_of_flat(r.dev_id);
    if (g >= 0) { cudaSetDevice(g); cudaFreeAsync(r.gmem_p, s ? s : g_dev[g].stream); }
  }
  r.gmem_p = nullptr;
}

void remove_image(talsh_tens_t* t, int idx, cudaStream_t s = nullptr) {
  free_image_memory(t->dev_rsc[idx], s);
  for (int i = idx; i + 1 < t->ndev; ++i) {
    t->dev_rsc[i] = t->dev_rsc[i + 1];
    t->data_kind[i] = t->data_kind[i + 1];
    t->avail[i] = t->avail[i + 1];
  }
  --t->ndev;
}

int add_image(talsh_tens_t* t, int flat_dev, void* p, int dtk, int attached) {
  if (t->ndev >= t->dev_rsc_len) return -1;
  const int i = t->ndev++;
  t->dev_rsc[i].dev_id = flat_dev;
  t->dev_rsc[i].gmem_p = p;
  t->dev_rsc[i].buf_entry = -1;
  t->dev_rsc[i].mem_attached = attached;
  t->data_kind[i] = dtk;
  t->avail[i] = YEP;
  return i;
}

int alloc_on(int flat_dev, size_t bytes, void** p, cudaStream_t s) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  if (flat_dev == 0) {
    if (g_ngpu > 0) { if (cudaMallocHost(p, bytes) != cudaSuccess) { cudaGetLastError(); return TRY_LATER; } }
    else { *p = std::malloc(bytes); if (!*p) return TRY_LATER; }
    return 0;
  }
  const int g = gpu_of_flat(flat_dev);
  if (g < 0 || !g_dev[g].on) return TALSH_INVALID_ARGS;
  cudaSetDevice(g);
  if (cudaMallocAsync(p, bytes, s ? s : g_dev[g].stream) != cudaSuccess) { cudaGetLastError(); return TRY_LATER; }
  return 0;
}

}  // namespace

// =============================================================================
// Control
// =============================================================================
extern "C" int talshValidDataKind(int datk, int* datk_size) {
  const int s = elem_size(datk);
  if (datk_size) *datk_size = s;
  return s > 0 ? YEP : NOPE;
}

extern "C" int talshInit(size_t* host_buf_size, int* host_arg_max, int ngpus, int gpu_list[], int nmics,
                         int mic_list[], int namds, int amd_list[]) {
  (void)mic_list; (void)amd_list;
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (g_on) return TALSH_ALREADY_INITIALIZED;
  if (nmics > 0 || namds > 0) return TALSH_NOT_AVAILABLE;
  if (ngpus < 0 || ngpus > MAX_GPUS_PER_NODE || (ngpus > 0 && !gpu_list)) return TALSH_INVALID_ARGS;
  for (int i = 0; i < ngpus; ++i) {
    const int g = gpu_list[i];
    if (g < 0 || g >= MAX_GPUS_PER_NODE) return TALSH_INVALID_ARGS;
    if (tb_device_init(g) != TB_SUCCESS) return TALSH_FAILURE;
    if (cudaStreamCreateWithFlags(&g_dev[g].stream, cudaStreamNonBlocking) != cudaSuccess) return TALSH_FAILURE;
    g_dev[g].on = true;
    g_dev[g].flops = 0.0;
  }
  g_ngpu = ngpus;
  if (host_arg_max) *host_arg_max = 1 << 20;
  (void)host_buf_size;  // host images are allocated on demand in pinned memory
  g_on = true;
  return TALSH_SUCCESS;
}

extern "C" int talshShutdown(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g_on) return TALSH_NOT_INITIALIZED;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) {
    if (!g_dev[g].on) continue;
    cudaSetDevice(g);
    cudaStreamSynchronize(g_dev[g].stream);
    cudaStreamDestroy(g_dev[g].stream);
    if (g_dev[g].xstream) { cudaStreamSynchronize(g_dev[g].xstream); cudaStreamDestroy(g_dev[g].xstream); }
    g_dev[g] = DevState();
  }
  g_ngpu = 0;
  g_on = false;
  return TALSH_SUCCESS;
}

extern "C" int talshEnableFastMath(int dev_kind, int dev_id) {
  if (dev_kind != DEV_NVIDIA_GPU) return TALSH_NOT_AVAILABLE;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g)
    if (g_dev[g].on && (dev_id == DEV_DEFAULT || dev_id == g)) g_dev[g].fast_math = true;
  return TALSH_SUCCESS;
}

extern "C" int talshDisableFastMath(int dev_kind, int dev_id) {
  if (dev_kind != DEV_NVIDIA_GPU) return TALSH_NOT_AVAILABLE;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g)
    if (g_dev[g].on && (dev_id == DEV_DEFAULT || dev_id == g)) g_dev[g].fast_math = false;
  return TALSH_SUCCESS;
}

extern "C" int talshQueryFastMath(int dev_kind, int dev_id) {
  if (dev_kind != DEV_NVIDIA_GPU || dev_id < 0 || dev_id >= MAX_GPUS_PER_NODE) return NOPE;
  return g_dev[dev_id].fast_math ? YEP : NOPE;
}

extern "C" int talshDeviceCount(int dev_kind, int* dev_count) {
  if (!dev_count) return TALSH_INVALID_ARGS;
  *dev_count = 0;
  if (dev_kind == DEV_HOST) { *dev_count = 1; return TALSH_SUCCESS; }
  if (dev_kind == DEV_NVIDIA_GPU) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); n = 0; }
    *dev_count = n > MAX_GPUS_PER_NODE ? MAX_GPUS_PER_NODE : n;
    return TALSH_SUCCESS;
  }
  if (dev_kind == DEV_INTEL_MIC || dev_kind == DEV_AMD_GPU) return TALSH_SUCCESS;
  return TALSH_INVALID_ARGS;
}

extern "C" int talshFlatDevId(int dev_kind, int dev_num) {
  // tensor_algebra_gpu.cpp:225-276 device-id codec
  switch (dev_kind) {
    case DEV_HOST: return dev_num == 0 ? 0 : DEV_MAX;
    case DEV_NVIDIA_GPU: return (dev_num >= 0 && dev_num < MAX_GPUS_PER_NODE) ? 1 + dev_num : DEV_MAX;
    case DEV_INTEL_MIC: return (dev_num >= 0 && dev_num < MAX_MICS_PER_NODE) ? 1 + MAX_GPUS_PER_NODE + dev_num : DEV_MAX;
    case DEV_AMD_GPU:
      return (dev_num >= 0 && dev_num < MAX_AMDS_PER_NODE) ? 1 + MAX_GPUS_PER_NODE + MAX_MICS_PER_NODE + dev_num : DEV_MAX;
  }
  return DEV_MAX;
}

extern "C" int talshKindDevId(int dev_id, int* dev_kind) {
  if (dev_id == 0) { if (dev_kind) *dev_kind = DEV_HOST; return 0; }
  if (dev_id >= 1 && dev_id <= MAX_GPUS_PER_NODE) { if (dev_kind) *dev_kind = DEV_NVIDIA_GPU; return dev_id - 1; }
  int b = 1 + MAX_GPUS_PER_NODE;
  if (dev_id >= b && dev_id < b + MAX_MICS_PER_NODE) { if (dev_kind) *dev_kind = DEV_INTEL_MIC; return dev_id - b; }
  b += MAX_MICS_PER_NODE;
  if (dev_id >= b && dev_id < b + MAX_AMDS_PER_NODE) { if (dev_kind) *dev_kind = DEV_AMD_GPU; return dev_id - b; }
  if (dev_kind) *dev_kind = DEV_NULL;
  return -1;
}

extern "C" size_t talshDeviceMemorySize(int dev_num, int dev_kind) {
  if (dev_kind != DEV_NVIDIA_GPU) return 0;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev_num) != cudaSuccess) { cudaGetLastError(); return 0; }
  return p.totalGlobalMem;
}

extern "C" double talshDeviceGetFlops(int dev_kind, int dev_id) {
  double f = 0.0;
  if (dev_kind != DEV_NVIDIA_GPU && dev_kind != DEV_DEFAULT) return 0.0;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g)
    if (g_dev[g].on && (dev_id == DEV_DEFAULT || dev_id == g)) f += g_dev[g].flops;
  return f;
}

extern "C" int talshStats(int dev_id, int dev_kind) {
  (void)dev_kind;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g)
    if (g_dev[g].on && (dev_id < 0 || dev_id == g))
      printf("#MSG(TAL-SH::B200): GPU %d: %.6e flops executed\n", g, g_dev[g].flops);
  return TALSH_SUCCESS;
}

// =============================================================================
// Tensor blocks
// =============================================================================
extern "C" int talshTensorCreate(talsh_tens_t** tens_block) {
  if (!tens_block) return TALSH_INVALID_ARGS;
  *tens_block = (talsh_tens_t*)std::malloc(sizeof(talsh_tens_t));
  if (!*tens_block) return TRY_LATER;
  return talshTensorClean(*tens_block);
}

extern "C" int talshTensorClean(talsh_tens_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  t->shape_p = nullptr; t->dev_rsc = nullptr; t->data_kind = nullptr; t->avail = nullptr;
  t->dev_rsc_len = 0; t->ndev = 0;
  return TALSH_SUCCESS;
}

extern "C" int talshTensorIsEmpty(const talsh_tens_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  return t->shape_p == nullptr ? YEP : NOPE;
}

extern "C" int talshTensorConstruct(talsh_tens_t* t, int data_kind, int tens_rank, const int tens_dims[], int dev_id,
                                    void* ext_mem, int in_hab, talsh_tens_init_i init_method, double init_val_real,
                                    double init_val_imag) {
  (void)in_hab;
  if (!g_on) return TALSH_NOT_INITIALIZED;
  if (!t || tens_rank < 0 || tens_rank > MAX_TENSOR_RANK || (tens_rank > 0 && !tens_dims)) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) != YEP) return TALSH_OBJECT_NOT_EMPTY;
  if (data_kind != NO_TYPE && !elem_size(data_kind)) return TALSH_INVALID_ARGS;
  for (int i = 0; i < tens_rank; ++i) if (tens_dims[i] <= 0) return TALSH_INVALID_ARGS;
  if (dev_id < 0 || dev_id > MAX_GPUS_PER_NODE) return TALSH_INVALID_ARGS;
  if (dev_id > 0 && !g_dev[dev_id - 1].on) return TALSH_INVALID_ARGS;
  t->shape_p = (talsh_tens_shape_t*)std::calloc(1, sizeof(talsh_tens_shape_t));
  t->shape_p->num_dim = tens_rank;
  t->shape_p->dims = (int*)std::calloc(tens_rank > 0 ? tens_rank : 1, sizeof(int));
  for (int i = 0; i < tens_rank; ++i) t->shape_p->dims[i] = tens_dims[i];
  t->dev_rsc_len = TALSH_MAX_DEV_PRESENT;
  t->dev_rsc = (talsh_dev_rsc_t*)std::calloc(TALSH_MAX_DEV_PRESENT, sizeof(talsh_dev_rsc_t));
  t->data_kind = (int*)std::calloc(TALSH_MAX_DEV_PRESENT, sizeof(int));
  t->avail = (int*)std::calloc(TALSH_MAX_DEV_PRESENT, sizeof(int));
  t->ndev = 0;
  if (data_kind == NO_TYPE && !ext_mem) return TALSH_SUCCESS;  // body deferred
  const size_t vol = volume_of(t);
  const size_t bytes = vol * (size_t)elem_size(data_kind);
  if (ext_mem) {
    add_image(t, dev_id, ext_mem, data_kind, 1);
    return TALSH_SUCCESS;
  }
  void* p = nullptr;
  cudaStream_t s = dev_id > 0 ? g_dev[dev_id - 1].stream : nullptr;
  if (int e = alloc_on(dev_id, bytes, &p, s)) { talshTensorDestruct(t); return e; }
  add_image(t, dev_id, p, data_kind, 0);
  // initialise the new body
  if (dev_id == 0) {
    if (init_method) {
      talsh_tens_data_t td{p, vol, data_kind};
      talsh_tens_signature_t sig{tens_rank, nullptr};
      int e = init_method(&td, t->shape_p, &sig);
      if (e) return TALSH_FAILURE;
    } else {
      for (size_t i = 0; i < vol; ++i) {
        switch (data_kind) {
          case R4: ((float*)p)[i] = (float)init_val_real; break;
          case R8: ((double*)p)[i] = init_val_real; break;
          case C4: ((float*)p)[2 * i] = (float)init_val_real; ((float*)p)[2 * i + 1] = (float)init_val_imag; break;
          case C8: ((double*)p)[2 * i] = init_val_real; ((double*)p)[2 * i + 1] = init_val_imag; break;
        }
      }
    }
  } else {
    if (init_method) return TALSH_NOT_AVAILABLE;
    cudaSetDevice(dev_id - 1);
    if (tb_tensor_init(data_kind, vol, p, init_val_real, init_val_imag, s) != TB_SUCCESS) return TALSH_FAILURE;
    cudaStreamSynchronize(s);
  }
  return TALSH_SUCCESS;
}

extern "C" int talshTensorConstruct_(talsh_tens_t* t, int data_kind, int tens_rank, const int tens_dims[], int dev_id,
                                     void* ext_mem, int in_hab, talsh_tens_init_i init_method, double init_val_real,
                                     double init_val_imag) {
  return talshTensorConstruct(t, data_kind, tens_rank, tens_dims, dev_id, ext_mem, in_hab, init_method,
                              init_val_real, init_val_imag);
}

extern "C" int talshTensorImportData(talsh_tens_t* t, int data_kind, const void* ext_data) {
  if (!t || !ext_data) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) == YEP) return TALSH_OBJECT_IS_EMPTY;
  const int i = find_image(t, 0);
  if (i < 0 || t->data_kind[i] != data_kind) return TALSH_NOT_FOUND;
  std::memcpy(t->dev_rsc[i].gmem_p, ext_data, volume_of(t) * elem_size(data_kind));
  for (int j = t->ndev - 1; j >= 0; --j) if (j != i) remove_image(t, j);
  return TALSH_SUCCESS;
}

extern "C" int talshTensorDestruct(talsh_tens_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) if (g_dev[g].on) { cudaSetDevice(g); cudaStreamSynchronize(g_dev[g].stream); }
  while (t->ndev > 0) remove_image(t, t->ndev - 1);
  if (t->shape_p) { std::free(t->shape_p->dims); std::free(t->shape_p); }
  std::free(t->dev_rsc); std::free(t->data_kind); std::free(t->avail);
  return talshTensorClean(t);
}

extern "C" int talshTensorDestroy(talsh_tens_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  int e = talshTensorDestruct(t);
  std::free(t);
  return e;
}

extern "C" int talshTensorRank(const talsh_tens_t* t) {
  return (t && t->shape_p) ? t->shape_p->num_dim : -1;
}

extern "C" size_t talshTensorVolume(const talsh_tens_t* t) { return volume_of(t); }

extern "C" size_t talshTensorSizeAllImages(const talsh_tens_t* t, int* num_images) {
  if (!t) return 0;
  size_t s = 0;
  for (int i = 0; i < t->ndev; ++i) s += volume_of(t) * elem_size(t->data_kind[i]);
  if (num_images) *num_images = t->ndev;
  return s;
}

extern "C" const int* talshTensorDimExtents(const talsh_tens_t* t, int* rank) {
  if (!t || !t->shape_p) { if (rank) *rank = -1; return nullptr; }
  if (rank) *rank = t->shape_p->num_dim;
  return t->shape_p->dims;
}

extern "C" int talshTensorDataKind(const talsh_tens_t* t, int* num_images, int* data_kinds) {
  if (!t || !num_images) return TALSH_INVALID_ARGS;
  *num_images = t->ndev;
  if (data_kinds) for (int i = 0; i < t->ndev; ++i) data_kinds[i] = t->data_kind[i];
  return TALSH_SUCCESS;
}

extern "C" int talshTensorInUse(const talsh_tens_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  for (int i = 0; i < t->ndev; ++i) if (t->avail[i] != YEP) return YEP;
  return NOPE;
}

extern "C" int talshTensorPresence(const talsh_tens_t* t, int* ncopies, int copies[], int data_kinds[], int dev_kind,
                                   int dev_id) {
  if (!t || !ncopies) return TALSH_INVALID_ARGS;
  *ncopies = 0;
  for (int i = 0; i < t->ndev; ++i) {
    int k;
    const int num = talshKindDevId(t->dev_rsc[i].dev_id, &k);
    if (dev_kind != DEV_NULL && (k != dev_kind || (dev_id >= 0 && num != dev_id))) continue;
    if (copies) copies[*ncopies] = t->dev_rsc[i].dev_id;
    if (data_kinds) data_kinds[*ncopies] = t->data_kind[i];
    ++*ncopies;
  }
  return TALSH_SUCCESS;
}

extern "C" int talshTensorGetBodyAccess(talsh_tens_t* t, void** body_p, int data_kind, int dev_id, int dev_kind) {
  // talshc.cpp:1572-1604: returns the matching image and discards all others
  if (!g_on) return TALSH_NOT_INITIALIZED;
  if (!t || !body_p) return TALSH_INVALID_ARGS;
  *body_p = nullptr;
  if (talshTensorIsEmpty(t) == YEP) return TALSH_OBJECT_IS_EMPTY;
  if (dev_kind != DEV_NULL) dev_id = talshFlatDevId(dev_kind, dev_id);
  if (dev_id < 0 || dev_id >= DEV_MAX) return TALSH_INVALID_ARGS;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->dev_rsc[i].dev_id == dev_id && t->data_kind[i] == data_kind) {
      *body_p = t->dev_rsc[i].gmem_p;
      for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) if (g_dev[g].on) { cudaSetDevice(g); cudaStreamSynchronize(g_dev[g].stream); }
      for (int j = t->ndev - 1; j >= 0; --j) if (j != i) remove_image(t, j);
      return TALSH_SUCCESS;
    }
  }
  return TALSH_NOT_FOUND;
}

extern "C" int talshTensorGetBodyAccessConst(const talsh_tens_t* t, const void** body_p, int data_kind, int dev_id,
                                             int dev_kind) {
  if (!g_on) return TALSH_NOT_INITIALIZED;
  if (!t || !body_p) return TALSH_INVALID_ARGS;
  *body_p = nullptr;
  if (talshTensorIsEmpty(t) == YEP) return TALSH_OBJECT_IS_EMPTY;
  if (dev_kind != DEV_NULL) dev_id = talshFlatDevId(dev_kind, dev_id);
  for (int i = 0; i < t->ndev; ++i)
    if (t->dev_rsc[i].dev_id == dev_id && t->data_kind[i] == data_kind) {
      *body_p = t->dev_rsc[i].gmem_p;
      return TALSH_SUCCESS;
    }
  return TALSH_NOT_FOUND;
}

extern "C" double talshTensorImageNorm1_cpu(const talsh_tens_t* t) {
  // talshc.cpp:6207: sum of |x| over the Host image (a debugging helper)
  if (!t) return -1.0;
  const int i = find_image(t, 0);
  if (i < 0) return -1.0;
  const size_t vol = volume_of(t);
  const void* p = t->dev_rsc[i].gmem_p;
  double s = 0.0;
  for (size_t k = 0; k < vol; ++k) {
    switch (t->data_kind[i]) {
      case R4: s += std::fabs(((const float*)p)[k]); break;
      case R8: s += std::fabs(((const double*)p)[k]); break;
      case C4: s += std::hypot(((const float*)p)[2 * k], ((const float*)p)[2 * k + 1]); break;
      case C8: s += std::hypot(((const double*)p)[2 * k], ((const double*)p)[2 * k + 1]); break;
    }
  }
  return s;
}

// =============================================================================
// Tasks
// =============================================================================
namespace {

TaskImpl* impl(talsh_task_t* t) { return t ? (TaskImpl*)t->task_p : nullptr; }

void task_finish(talsh_task_t* t) {
  TaskImpl* ti = impl(t);
  if (!ti || ti->done) return;
  for (auto& f : ti->finalize) f();
  ti->finalize.clear();
  ti->done = true;
}

}  // namespace

extern "C" int talshTaskCreate(talsh_task_t** t) {
  if (!t) return TALSH_INVALID_ARGS;
  *t = (talsh_task_t*)std::malloc(sizeof(talsh_task_t));
  if (!*t) return TRY_LATER;
  return talshTaskClean(*t);
}

extern "C" int talshTaskClean(talsh_task_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  std::memset(t, 0, sizeof(*t));
  t->task_p = nullptr;
  t->task_error = -1;
  t->dev_kind = DEV_NULL;
  t->data_kind = NO_TYPE;
  t->coherence = -1;
  return TALSH_SUCCESS;
}

extern "C" int talshTaskIsEmpty(const talsh_task_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  return t->task_p == nullptr ? YEP : NOPE;
}

extern "C" int talshTaskDestruct(talsh_task_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  TaskImpl* ti = impl(t);
  if (ti) {
    if (!ti->done) {
      cudaSetDevice(ti->gpu);
      if (ti->ev[3]) cudaEventSynchronize(ti->ev[3]);
      task_finish(t);
    }
    for (auto& e : ti->ev) if (e) cudaEventDestroy(e);
    delete ti;
  }
  return talshTaskClean(t);
}

extern "C" int talshTaskDestroy(talsh_task_t* t) {
  if (!t) return TALSH_INVALID_ARGS;
  int e = talshTaskDestruct(t);
  std::free(t);
  return e;
}

extern "C" int talshTaskDevId(talsh_task_t* t, int* dev_kind) {
  TaskImpl* ti = impl(t);
  if (!ti) return DEV_NULL;
  if (dev_kind) { *dev_kind = DEV_NVIDIA_GPU; return ti->gpu; }
  return flat_gpu(ti->gpu);
}

extern "C" int talshTaskStatus(talsh_task_t* t) {
  TaskImpl* ti = impl(t);
  if (!ti) return TALSH_TASK_EMPTY;
  if (ti->done) return ti->err ? TALSH_TASK_ERROR : TALSH_TASK_COMPLETED;
  cudaSetDevice(ti->gpu);
  cudaError_t q = cudaEventQuery(ti->ev[3]);
  if (q == cudaErrorNotReady) return TALSH_TASK_SCHEDULED;
  if (q != cudaSuccess) { ti->err = TALSH_FAILURE; t->task_error = 1; }
  task_finish(t);
  if (!ti->err) t->task_error = 0;
  return ti->err ? TALSH_TASK_ERROR : TALSH_TASK_COMPLETED;
}

extern "C" int talshTaskComplete(talsh_task_t* t, int* stats, int* ierr) {
  if (ierr) *ierr = TALSH_SUCCESS;
  const int st = talshTaskStatus(t);
  if (stats) *stats = st;
  if (st == TALSH_TASK_EMPTY) { if (ierr) *ierr = TALSH_OBJECT_IS_EMPTY; return NOPE; }
  if (st == TALSH_TASK_ERROR && ierr) *ierr = TALSH_TASK_ERROR;
  return (st == TALSH_TASK_COMPLETED || st == TALSH_TASK_ERROR) ? YEP : NOPE;
}

extern "C" int talshTaskWait(talsh_task_t* t, int* stats) {
  TaskImpl* ti = impl(t);
  if (!ti) { if (stats) *stats = TALSH_TASK_EMPTY; return TALSH_OBJECT_IS_EMPTY; }
  if (!ti->done) {
    cudaSetDevice(ti->gpu);
    if (cudaEventSynchronize(ti->ev[3]) != cudaSuccess) { cudaGetLastError(); ti->err = TALSH_FAILURE; }
    if (!ti->err && tb_device_check(g_dev[ti->gpu].stream) != TB_SUCCESS) ti->err = TALSH_FAILURE;
    task_finish(t);
    t->task_error = ti->err ? 1 : 0;
    if (!ti->err) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ti->ev[0], ti->ev[3]);
      t->exec_time = ms * 1e-3;
    }
  }
  if (stats) *stats = ti->err ? TALSH_TASK_ERROR : TALSH_TASK_COMPLETED;
  return TALSH_SUCCESS;
}

extern "C" int talshTasksWait(int ntasks, talsh_task_t tasks[], int stats[]) {
  if (ntasks < 0 || (ntasks > 0 && (!tasks || !stats))) return TALSH_INVALID_ARGS;
  int err = TALSH_SUCCESS;
  for (int i = 0; i < ntasks; ++i) { int e = talshTaskWait(&tasks[i], &stats[i]); if (e) err = e; }
  return err;
}

extern "C" int talshTaskTime(talsh_task_t* t, double* total, double* comput, double* input, double* output,
                             double* mmul) {
  TaskImpl* ti = impl(t);
  if (!ti || !total) return TALSH_INVALID_ARGS;
  if (!ti->done) return TALSH_IN_PROGRESS;
  float a = 0, b = 0, c = 0, d = 0;
  cudaEventElapsedTime(&a, ti->ev[0], ti->ev[3]);
  cudaEventElapsedTime(&b, ti->ev[1], ti->ev[2]);
  cudaEventElapsedTime(&c, ti->ev[0], ti->ev[1]);
  cudaEventElapsedTime(&d, ti->ev[2], ti->ev[3]);
  *total = a * 1e-3;
  if (comput) *comput = b * 1e-3;
  if (input) *input = c * 1e-3;
  if (output) *output = d * 1e-3;
  if (mmul) *mmul = b * 1e-3;
  return TALSH_SUCCESS;
}

// =============================================================================
// Operation machinery: execution device, operand images, coherence
// =============================================================================
namespace {

// Resolves (dev_id, dev_kind) to a kind-specific GPU number, or a TALSH code.
int resolve_gpu(int dev_id, int dev_kind, int* gpu) {
  if (dev_kind == DEV_DEFAULT) {
    if (dev_id == DEV_DEFAULT) {
      for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) if (g_dev[g].on) { *gpu = g; return 0; }
      return TALSH_NOT_AVAILABLE;
    }
    int k;
    const int n = talshKindDevId(dev_id, &k);
    if (k == DEV_HOST) return TALSH_NOT_AVAILABLE;
    if (k != DEV_NVIDIA_GPU) return TALSH_INVALID_ARGS;
    dev_id = n;
  } else if (dev_kind == DEV_HOST) {
    return TALSH_NOT_AVAILABLE;
  } else if (dev_kind != DEV_NVIDIA_GPU) {
    return TALSH_NOT_AVAILABLE;
  } else if (dev_id == DEV_DEFAULT) {
    dev_id = 0;
    while (dev_id < MAX_GPUS_PER_NODE && !g_dev[dev_id].on) ++dev_id;
  }
  if (dev_id < 0 || dev_id >= MAX_GPUS_PER_NODE || !g_dev[dev_id].on) return TALSH_INVALID_ARGS;
  *gpu = dev_id;
  return 0;
}

// Copy-control value of argument arg_num among tot_args (D most senior).
int coh_of(int copy_ctrl, int tot_args, int arg_num) { return (copy_ctrl >> (2 * (tot_args - 1 - arg_num))) & 3; }

struct Operand {
  talsh_tens_t* t = nullptr;
  int src = -1;          // source image index
  bool moved = false;    // a new image was created on the execution GPU
  bool sliced = false;   // streamed to the GPU in slices by the computation itself
  void* dptr = nullptr;  // body on the execution GPU
  size_t bytes = 0;
};

// Prepares one operand on the execution GPU (H2D when its image is elsewhere).
// A sliced operand only gets its source: its host image.
int stage_operand(Operand& op, int gpu, int dtk, cudaStream_t s) {
  talsh_tens_t* t = op.t;
  const int flat = flat_gpu(gpu);
  op.bytes = volume_of(t) * elem_size(dtk);
  if (op.sliced) {
    for (int j = 0; j < t->ndev; ++j)
      if (t->avail[j] == YEP && t->data_kind[j] == dtk && t->dev_rsc[j].dev_id == 0) { op.src = j; return 0; }
    return TALSH_NOT_FOUND;
  }
  int i = find_image(t, flat);
  if (i >= 0 && t->data_kind[i] == dtk) { op.src = i; op.dptr = t->dev_rsc[i].gmem_p; return 0; }
  i = -1;
  for (int j = 0; j < t->ndev; ++j) if (t->avail[j] == YEP && t->data_kind[j] == dtk) { i = j; break; }
  if (i < 0) return TALSH_NOT_FOUND;
  op.src = i;
  if (int e = alloc_on(flat, op.bytes, &op.dptr, s)) return e;
  op.moved = true;
  const int src_flat = t->dev_rsc[i].dev_id;
  if (src_flat == 0) {
    if (cudaMemcpyAsync(op.dptr, t->dev_rsc[i].gmem_p, op.bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return TALSH_FAILURE;
  } else {
    if (cudaMemcpyPeerAsync(op.dptr, gpu, t->dev_rsc[i].gmem_p, gpu_of_flat(src_flat), op.bytes, s) != cudaSuccess)
      return TALSH_FAILURE;
  }
  return 0;
}

// Applies copy control to one operand once the computation is enqueued.
// is_out: the operand was written (its source image must see the result).
void settle_operand(Operand& op, int coh, bool is_out, int gpu, int dtk, cudaStream_t s, TaskImpl* ti) {
  talsh_tens_t* t = op.t;
  const int flat = flat_gpu(gpu);
  if (op.sliced) {  // an input read from its host image: only COPY_D has something to do
    if (coh == COPY_D) {
      void* p = t->dev_rsc[op.src].gmem_p;
      ti->finalize.push_back([t, p]() {
        for (int i = 0; i < t->ndev; ++i) if (t->dev_rsc[i].gmem_p == p) { remove_image(t, i); break; }
      });
    }
    return;
  }
  if (!op.moved) {
    if (coh == COPY_D) ti->finalize.push_back([t, flat]() { int i = find_image(t, flat); if (i >= 0) remove_image(t, i); });
    return;
  }
  const int src_flat = t->dev_rsc[op.src].dev_id;
  void* src_ptr = t->dev_rsc[op.src].gmem_p;
  if (is_out && (coh == COPY_T || coh == COPY_K)) {
    if (src_flat == 0) cudaMemcpyAsync(src_ptr, op.dptr, op.bytes, cudaMemcpyDeviceToHost, s);
    else cudaMemcpyPeerAsync(src_ptr, gpu_of_flat(src_flat), op.dptr, gpu, op.bytes, s);
  }
  if (coh == COPY_M || coh == COPY_K) {
    const int ni = add_image(t, flat, op.dptr, dtk, 0);
    if (ni < 0) { cudaFreeAsync(op.dptr, s); return; }
    if (coh == COPY_M) {
      void* p = src_ptr;
      ti->finalize.push_back([t, p]() {
        for (int i = 0; i < t->ndev; ++i) if (t->dev_rsc[i].gmem_p == p) { remove_image(t, i); break; }
      });
    }
  } else {
    cudaFreeAsync(op.dptr, s);  // stream-ordered: after the kernels that read it
    if (coh == COPY_D) {
      void* p = src_ptr;
      ti->finalize.push_back([t, p]() {
        for (int i = 0; i < t->ndev; ++i) if (t->dev_rsc[i].gmem_p == p) { remove_image(t, i); break; }
      });
    }
  }
}

using Compute = std::function<int(cudaStream_t, std::vector<Operand>&)>;

// Runs an operation on a GPU: stages operands, computes, settles coherence.
int run_op(std::vector<talsh_tens_t*> args, int copy_ctrl, int dev_id, int dev_kind, talsh_task_t* task,
           const Compute& compute, double flops, const std::vector<char>* sliced = nullptr) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g_on) return TALSH_NOT_INITIALIZED;
  for (auto* t : args) {
    if (!t) return TALSH_INVALID_ARGS;
    if (talshTensorIsEmpty(t) == YEP) return TALSH_OBJECT_IS_EMPTY;
  }
  if (task && talshTaskIsEmpty(task) != YEP) return TALSH_OBJECT_NOT_EMPTY;
  int gpu = -1;
  if (int e = resolve_gpu(dev_id, dev_kind, &gpu)) return e;
  // all images of an operation share one data kind
  int dtk = NO_TYPE;
  for (int j = 0; j < args[0]->ndev; ++j) if (args[0]->avail[j] == YEP) { dtk = args[0]->data_kind[j]; break; }
  if (dtk == NO_TYPE) return TALSH_NOT_FOUND;
  cudaSetDevice(gpu);
  cudaStream_t s = g_dev[gpu].stream;
  TaskImpl* ti = new TaskImpl();
  ti->gpu = gpu;
  for (auto& e : ti->ev) cudaEventCreate(&e);
  cudaEventRecord(ti->ev[0], s);
  std::vector<Operand> ops(args.size());
  int err = 0;
  for (size_t i = 0; i < args.size() && !err; ++i) {
    ops[i].t = args[i];
    ops[i].sliced = sliced && i < sliced->size() && (*sliced)[i];
    err = stage_operand(ops[i], gpu, dtk, s);
  }
  if (err) {
    for (auto& o : ops) if (o.moved) cudaFreeAsync(o.dptr, s);
    cudaStreamSynchronize(s);
    for (auto& e : ti->ev) cudaEventDestroy(e);
    delete ti;
    return err == TALSH_NOT_FOUND ? TALSH_INVALID_ARGS : err;
  }
  cudaEventRecord(ti->ev[1], s);
  err = compute(s, ops);
  cudaEventRecord(ti->ev[2], s);
  const int nargs = (int)args.size();
  for (int i = 0; i < nargs; ++i) settle_operand(ops[i], coh_of(copy_ctrl, nargs, i), i == 0 && !err, gpu, dtk, s, ti);
  cudaEventRecord(ti->ev[3], s);
  if (err) ti->err = TALSH_FAILURE;
  g_dev[gpu].flops += flops;
  talsh_task_t local;
  talsh_task_t* tk = task ? task : &local;
  if (!task) talshTaskClean(&local);
  tk->task_p = ti;
  tk->dev_kind = DEV_NVIDIA_GPU;
  tk->data_kind = dtk;
  tk->coherence = copy_ctrl;
  tk->num_args = nargs;
  for (int i = 0; i < nargs && i < MAX_TENSOR_OPERANDS; ++i) { tk->tens_args[i].tens_p = args[i]; tk->tens_args[i].source_image = ops[i].src; }
  tk->flops = flops;
  tk->data_vol = 0.0;
  for (auto& o : ops) tk->data_vol += (double)o.bytes;
  if (!task) {
    int st = 0;
    talshTaskWait(&local, &st);
    const int terr = local.task_error;
    talshTaskDestruct(&local);
    if (err) return err;
    return terr ? TALSH_TASK_ERROR : TALSH_SUCCESS;
  }
  return err;
}

int data_kind_of(const talsh_tens_t* t) {
  for (int j = 0; j < t->ndev; ++j) if (t->avail[j] == YEP) return t->data_kind[j];
  return NO_TYPE;
}

}  // namespace

// =============================================================================
// Operations (TALSH/talshc.cpp dispatchers: Init :3648, Scale :3869,
// Copy :4530, Add :4795, Contract :5073, ContractXL :5394)
// =============================================================================
extern "C" int talshTensorInit(talsh_tens_t* dtens, double vr, double vi, int dev_id, int dev_kind, int copy_ctrl,
                               talsh_task_t* task) {
  if (!dtens) return TALSH_INVALID_ARGS;
  const size_t vol = volume_of(dtens);
  return run_op({dtens}, copy_ctrl, dev_id, dev_kind, task,
                [&](cudaStream_t s, std::vector<Operand>& o) {
                  return map_tb(tb_tensor_init(data_kind_of(dtens), vol, o[0].dptr, vr, vi, s));
                }, 0.0);
}

extern "C" int talshTensorScale(talsh_tens_t* dtens, double sr, double si, int dev_id, int dev_kind, int copy_ctrl,
                                talsh_task_t* task) {
  if (!dtens) return TALSH_INVALID_ARGS;
  const size_t vol = volume_of(dtens);
  return run_op({dtens}, copy_ctrl, dev_id, dev_kind, task,
                [&](cudaStream_t s, std::vector<Operand>& o) {
                  return map_tb(tb_tensor_scale(data_kind_of(dtens), vol, o[0].dptr, sr, si, s));
                }, (double)vol);
}

namespace {

// Parses a unary pattern and checks it against D and L (talshc.cpp:4571).
int check_unary(const char* cptrn, const talsh_tens_t* d, const talsh_tens_t* l, tb::ParsedPattern* P) {
  if (!cptrn || !d || !l) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(d) == YEP || talshTensorIsEmpty(l) == YEP) return TALSH_OBJECT_IS_EMPTY;
  if (tb::parse_pattern(cptrn, P) || P->rrank != -1) return TALSH_INVALID_ARGS;
  if (P->drank != d->shape_p->num_dim || P->lrank != l->shape_p->num_dim || P->drank != P->lrank) return TALSH_INVALID_ARGS;
  for (int i = 0; i < P->lrank; ++i)
    if (d->shape_p->dims[P->cptrn[i] - 1] != l->shape_p->dims[i]) return TALSH_INVALID_ARGS;
  if (data_kind_of(d) != data_kind_of(l)) return TALSH_INVALID_ARGS;
  return 0;
}

}  // namespace

extern "C" int talshTensorCopy(const char* cptrn, talsh_tens_t* dtens, talsh_tens_t* ltens, int dev_id, int dev_kind,
                               int copy_ctrl, talsh_task_t* task) {
  tb::ParsedPattern P;
  if (int e = check_unary(cptrn, dtens, ltens, &P)) return e;
  const int dtk = data_kind_of(ltens);
  return run_op({dtens, ltens}, copy_ctrl, dev_id, dev_kind, task,
                [&](cudaStream_t s, std::vector<Operand>& o) {
                  return map_tb(tb_tensor_copy(dtk, P.lrank, ltens->shape_p->dims, P.cptrn, o[1].dptr, o[0].dptr,
                                               P.conj_bits, s));
                }, 0.0);
}

extern "C" int talshTensorAdd(const char* cptrn, talsh_tens_t* dtens, talsh_tens_t* ltens, double sr, double si,
                              int dev_id, int dev_kind, int copy_ctrl, talsh_task_t* task) {
  tb::ParsedPattern P;
  if (int e = check_unary(cptrn, dtens, ltens, &P)) return e;
  const int dtk = data_kind_of(ltens);
  const double flops = (double)volume_of(ltens) * ((dtk == C4 || dtk == C8) ? 8.0 : 2.0);
  return run_op({dtens, ltens}, copy_ctrl, dev_id, dev_kind, task,
                [&](cudaStream_t s, std::vector<Operand>& o) {
                  return map_tb(tb_tensor_add(dtk, P.lrank, ltens->shape_p->dims, P.cptrn, o[0].dptr, o[1].dptr, sr,
                                              si, P.conj_bits, s));
                }, flops);
}

namespace {

// ---- streamed contractions -------------------------------------------------
// TAL-SH splits an operation whose operands exceed the device buffer into
// sub-operations by halving dimensions (talshTensorOpDecompose2,
// talshc.cpp:3150) and runs them from the host (talshTensorOpProgress :2929,
// ContractXL :5394).  Here a contraction whose inputs L and R live only on
// the host (copy control COPY_T or COPY_D) and are large streams instead:
//   - it is split along the slowest index of L (or of R) when that index is
//     contracted, so that L's slices are contiguous host ranges; the other
//     operand's slices are one 2-D strided copy each;
//   - slices move host-to-device on a copy stream into a ring of three
//     buffers while the compute stream contracts the previous slices into D
//     (D += slice products; the first slice applies the caller's
//     accumulative flag), ordered by events;
//   - D is staged whole, as for any contraction.
// Transfers overlap the computation, and L and R need not fit in HBM.  Each
// slice is an ordinary contraction (same method choice), so results agree
// with the unsliced contraction within its error bound, not bit for bit
// (the sums are split along K).  TB_STREAM=0 turns it off;
// TB_STREAM_MIN_MB (default 1024) is the size of L plus R from which it runs.
struct SliceSpec {
  int big = 0;              // 1: slices of L are contiguous (its slowest index), 2: of R
  int bpos = -1, opos = -1; // position of the sliced index in that operand and in the other
  int64_t ext = 0, step = 0;
};

constexpr int kSliceRing = 3;
constexpr int64_t kSliceTargetBytes = (int64_t)512 << 20;

int64_t prod_dims(const int* d, int a, int b) {
  int64_t p = 1;
  for (int i = a; i < b; ++i) p *= d[i];
  return p;
}

bool host_only(const talsh_tens_t* t, int dtk, int gpu) {
  bool host = false;
  for (int j = 0; j < t->ndev; ++j) {
    if (t->avail[j] != YEP) continue;
    if (t->dev_rsc[j].dev_id == flat_gpu(gpu)) return false;
    if (t->dev_rsc[j].dev_id == 0 && t->data_kind[j] == dtk) host = true;
  }
  return host;
}

SliceSpec plan_slices(const tb::ParsedPattern& P, const talsh_tens_t* l, const talsh_tens_t* r, int dtk,
                      int copy_ctrl, int dev_id, int dev_kind) {
  SliceSpec sp;
  const char* on = std::getenv("TB_STREAM");
  if (on && on[0] == '0') return sp;
  const char* mb = std::getenv("TB_STREAM_MIN_MB");
  const int64_t min_bytes = (mb ? std::atoll(mb) : 1024) << 20;
  int gpu = -1;
  if (resolve_gpu(dev_id, dev_kind, &gpu) || P.hyper) return sp;
  for (int a = 1; a <= 2; ++a) {
    const int c = coh_of(copy_ctrl, 3, a);
    if (c != COPY_T && c != COPY_D) return sp;
  }
  if (!host_only(l, dtk, gpu) || !host_only(r, dtk, gpu)) return sp;
  const int64_t es = elem_size(dtk);
  const int64_t bytes = ((int64_t)volume_of(l) + (int64_t)volume_of(r)) * es;
  if (bytes < min_bytes || bytes == 0) return sp;
  const int* ld = l->shape_p->dims;
  const int* rd = r->shape_p->dims;
  if (P.lrank >= 1 && P.cptrn[P.lrank - 1] < 0) {
    sp.big = 1; sp.bpos = P.lrank - 1; sp.opos = -P.cptrn[P.lrank - 1] - 1; sp.ext = ld[sp.bpos];
  } else if (P.rrank >= 1 && P.cptrn[P.lrank + P.rrank - 1] < 0) {
    sp.big = 2; sp.bpos = P.rrank - 1; sp.opos = -P.cptrn[P.lrank + P.rrank - 1] - 1; sp.ext = rd[sp.bpos];
  } else {
    return SliceSpec();
  }
  if (sp.ext < 2) return SliceSpec();
  // the other operand's slices are 2-D copies: its row pitch must be legal
  const int* od = sp.big == 1 ? rd : ld;
  const int orank = sp.big == 1 ? P.rrank : P.lrank;
  const int64_t opitch = prod_dims(od, 0, sp.opos) * sp.ext * es;
  if (prod_dims(od, sp.opos + 1, orank) > 1 && opitch >= ((int64_t)1 << 31)) return SliceSpec();
  const int64_t bigbytes = (int64_t)volume_of(sp.big == 1 ? l : r) * es;
  int64_t nsl = std::max<int64_t>(kSliceRing, (bigbytes + kSliceTargetBytes - 1) / kSliceTargetBytes);
  nsl = std::min<int64_t>(nsl, sp.ext);
  sp.step = (sp.ext + nsl - 1) / nsl;
  return sp;
}

// The streamed computation (runs as run_op's compute step on stream s).
int contract_streamed(const tb::ParsedPattern& P, const SliceSpec& sp, int dtk, talsh_tens_t* dtens,
                      talsh_tens_t* ltens, talsh_tens_t* rtens, double sr, double si, int accumulative,
                      const tb_plan_t* plan, cudaStream_t s, std::vector<Operand>& o) {
  int g = 0;
  cudaGetDevice(&g);
  if (!g_dev[g].xstream && cudaStreamCreateWithFlags(&g_dev[g].xstream, cudaStreamNonBlocking) != cudaSuccess)
    return TALSH_FAILURE;
  cudaStream_t xs = g_dev[g].xstream;
  const int64_t es = elem_size(dtk);
  talsh_tens_t* big = sp.big == 1 ? ltens : rtens;
  talsh_tens_t* oth = sp.big == 1 ? rtens : ltens;
  const int brank = sp.big == 1 ? P.lrank : P.rrank, orank = sp.big == 1 ? P.rrank : P.lrank;
  const char* bh = (const char*)big->dev_rsc[o[sp.big].src].gmem_p;
  const char* oh = (const char*)oth->dev_rsc[o[3 - sp.big].src].gmem_p;
  int bd[MAX_TENSOR_RANK], od[MAX_TENSOR_RANK];
  std::memcpy(bd, big->shape_p->dims, sizeof(int) * brank);
  std::memcpy(od, oth->shape_p->dims, sizeof(int) * orank);
  const int64_t inner_b = prod_dims(bd, 0, sp.bpos);
  const int64_t inner_o = prod_dims(od, 0, sp.opos), outer_o = prod_dims(od, sp.opos + 1, orank);
  const size_t bslice = (size_t)(inner_b * sp.step * es), oslice = (size_t)(inner_o * sp.step * outer_o * es);
  void* bb[kSliceRing] = {nullptr, nullptr, nullptr};
  void* ob[kSliceRing] = {nullptr, nullptr, nullptr};
  cudaEvent_t ready[kSliceRing] = {nullptr, nullptr, nullptr}, freed[kSliceRing] = {nullptr, nullptr, nullptr};
  cudaEvent_t start = nullptr, copies_done = nullptr;
  int err = 0;
  for (int i = 0; i < kSliceRing && !err; ++i) {
    if ((err = alloc_on(flat_gpu(g), bslice, &bb[i], s))) break;
    if ((err = alloc_on(flat_gpu(g), oslice, &ob[i], s))) break;
  }
  for (int i = 0; i < kSliceRing && !err; ++i)
    if (cudaEventCreateWithFlags(&ready[i], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&freed[i], cudaEventDisableTiming) != cudaSuccess)
      err = TALSH_FAILURE;
  if (!err && (cudaEventCreateWithFlags(&start, cudaEventDisableTiming) != cudaSuccess ||
               cudaEventCreateWithFlags(&copies_done, cudaEventDisableTiming) != cudaSuccess))
    err = TALSH_FAILURE;
  if (!err) {
    cudaEventRecord(start, s);  // buffers allocated (stream-ordered on s)
    cudaStreamWaitEvent(xs, start, 0);
    const int64_t nsl = (sp.ext + sp.step - 1) / sp.step;
    for (int64_t k = 0; k < nsl && !err; ++k) {
      const int slot = (int)(k % kSliceRing);
      const int64_t x0 = k * sp.step, w = std::min(sp.step, sp.ext - x0);
      if (k >= kSliceRing) cudaStreamWaitEvent(xs, freed[slot], 0);
      if (cudaMemcpyAsync(bb[slot], bh + x0 * inner_b * es, (size_t)(w * inner_b * es), cudaMemcpyHostToDevice, xs) !=
          cudaSuccess) { err = TALSH_FAILURE; break; }
      const size_t width = (size_t)(inner_o * w * es);
      const cudaError_t ce =
          outer_o == 1 ? cudaMemcpyAsync(ob[slot], oh + x0 * inner_o * es, width, cudaMemcpyHostToDevice, xs)
                       : cudaMemcpy2DAsync(ob[slot], width, oh + x0 * inner_o * es, (size_t)(inner_o * sp.ext * es),
                                           width, (size_t)outer_o, cudaMemcpyHostToDevice, xs);
      if (ce != cudaSuccess) { err = TALSH_FAILURE; break; }
      cudaEventRecord(ready[slot], xs);
      cudaStreamWaitEvent(s, ready[slot], 0);
      bd[sp.bpos] = (int)w;
      od[sp.opos] = (int)w;
      const void* lp = sp.big == 1 ? bb[slot] : ob[slot];
      const void* rp = sp.big == 1 ? ob[slot] : bb[slot];
      const int* ldims = sp.big == 1 ? bd : od;
      const int* rdims = sp.big == 1 ? od : bd;
      err = map_tb(tb_tensor_contract(P.cptrn, dtk, P.drank, dtens->shape_p->dims, o[0].dptr, P.lrank, ldims, lp,
                                      P.rrank, rdims, rp, sr, si, P.conj_bits, k == 0 ? accumulative : YEP, plan, s));
      cudaEventRecord(freed[slot], s);
    }
    // every copy into the ring precedes s before the buffers are released
    cudaEventRecord(copies_done, xs);
    cudaStreamWaitEvent(s, copies_done, 0);
  }
  if (err) cudaGetLastError();
  for (int i = 0; i < kSliceRing; ++i) {
    if (bb[i]) cudaFreeAsync(bb[i], s);
    if (ob[i]) cudaFreeAsync(ob[i], s);
  }
  for (int i = 0; i < kSliceRing; ++i) {
    if (ready[i]) cudaEventDestroy(ready[i]);
    if (freed[i]) cudaEventDestroy(freed[i]);
  }
  if (start) cudaEventDestroy(start);
  if (copies_done) cudaEventDestroy(copies_done);
  return err;
}

// Output decomposition for talshTensorContractXL.  TAL-SH's XL contraction
// halves the largest dimension of the operation until its arguments fit the
// device buffer (talshTensorOpDecompose2, talshc.cpp:3150) and runs the parts
// one by one (ContractXL :5394-5642).  Here, when D, L and R live only on the
// host and the contraction with its scratch would not fit in the device
// budget, D is cut along its largest dimension (the slowest of equal ones):
//   - that index belongs to one input, X; the other input, Y, moves to the
//     GPU once and stays;
//   - each D slab and the matching X slab move in (D only when accumulating)
//     on the copy stream, are contracted on the compute stream, and D's slab
//     moves back on the copy stream, through two buffer sets, so that the
//     transfers of one slab overlap the contraction of the other;
//   - slabs are 2-D strided copies: inner dims x slab extent, times outer dims.
// Every D element is computed whole by one sub-contraction (its K sum is not
// split), with the same method choice as any contraction.  The budget is
// TB_XL_DEVICE_MB when set, else 80% of the GPU's free memory; the
// contraction's scratch is counted as twice its operands.
struct DSplit {
  int dpos = -1;           // sliced position of D
  int xop = 0, xpos = -1;  // input carrying it (1 = L, 2 = R) and its position there
  int64_t ext = 0, step = 0;
};

thread_local DSplit g_last_split;

bool slab_pitch_ok(const int* dims, int rank, int pos, int64_t es) {
  return prod_dims(dims, pos + 1, rank) == 1 || prod_dims(dims, 0, pos + 1) * es < ((int64_t)1 << 31);
}

DSplit plan_out_of_core(const tb::ParsedPattern& P, const talsh_tens_t* d, const talsh_tens_t* l,
                        const talsh_tens_t* r, int dtk, int gpu) {
  DSplit sp;
  if (P.hyper || P.drank < 1) return sp;
  if (!host_only(d, dtk, gpu) || !host_only(l, dtk, gpu) || !host_only(r, dtk, gpu)) return sp;
  int64_t budget = 0;
  if (const char* mb = std::getenv("TB_XL_DEVICE_MB")) {
    budget = (int64_t)std::atoll(mb) << 20;
  } else {
    size_t fr = 0, tot = 0;
    cudaSetDevice(gpu);
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { cudaGetLastError(); return sp; }
    budget = (int64_t)(0.8 * (double)fr);
  }
  const int64_t es = elem_size(dtk);
  const int64_t db = (int64_t)volume_of(d) * es, lb = (int64_t)volume_of(l) * es, rb = (int64_t)volume_of(r) * es;
  if (3 * (db + lb + rb) <= budget) return sp;  // fits whole
  const int* dd = d->shape_p->dims;
  for (int p = 0; p < P.drank; ++p)
    if (dd[p] >= 2 && (sp.dpos < 0 || dd[p] >= dd[sp.dpos])) sp.dpos = p;
  if (sp.dpos < 0) return DSplit();
  for (int i = 0; i < P.lrank; ++i)
    if (P.cptrn[i] == sp.dpos + 1) { sp.xop = 1; sp.xpos = i; }
  for (int j = 0; j < P.rrank; ++j)
    if (P.cptrn[P.lrank + j] == sp.dpos + 1) { sp.xop = 2; sp.xpos = j; }
  if (!sp.xop) return DSplit();
  const talsh_tens_t* x = sp.xop == 1 ? l : r;
  const int xrank = sp.xop == 1 ? P.lrank : P.rrank;
  if (!slab_pitch_ok(dd, P.drank, sp.dpos, es) || !slab_pitch_ok(x->shape_p->dims, xrank, sp.xpos, es))
    return DSplit();
  sp.ext = dd[sp.dpos];
  const int64_t yb = sp.xop == 1 ? rb : lb, xb = sp.xop == 1 ? lb : rb;
  const int64_t per = (db + xb) / sp.ext;  // D and X bytes per unit of the sliced extent
  // resident: Y + two slab sets; scratch of one sub-contraction: twice its operands
  const int64_t room = budget - 3 * yb;
  if (per <= 0 || room < 5 * per) return DSplit();
  sp.step = std::min<int64_t>(room / (5 * per), (sp.ext + 1) / 2);
  return sp;
}

cudaError_t copy_slab(void* dev, char* host, int64_t inner, int64_t ext, int64_t outer, int64_t x0, int64_t w,
                      int64_t es, bool to_dev, cudaStream_t st) {
  const size_t width = (size_t)(inner * w * es), pitch = (size_t)(inner * ext * es);
  char* h = host + x0 * inner * es;
  if (outer == 1)
    return to_dev ? cudaMemcpyAsync(dev, h, width, cudaMemcpyHostToDevice, st)
                  : cudaMemcpyAsync(h, dev, width, cudaMemcpyDeviceToHost, st);
  return to_dev ? cudaMemcpy2DAsync(dev, width, h, pitch, width, (size_t)outer, cudaMemcpyHostToDevice, st)
                : cudaMemcpy2DAsync(h, pitch, dev, width, width, (size_t)outer, cudaMemcpyDeviceToHost, st);
}

int contract_out_of_core(const tb::ParsedPattern& P, const DSplit& sp, int dtk, talsh_tens_t* dtens,
                         talsh_tens_t* ltens, talsh_tens_t* rtens, double sr, double si, int accumulative,
                         const tb_plan_t* plan, cudaStream_t s, std::vector<Operand>& o) {
  int g = 0;
  cudaGetDevice(&g);
  if (!g_dev[g].xstream && cudaStreamCreateWithFlags(&g_dev[g].xstream, cudaStreamNonBlocking) != cudaSuccess)
    return TALSH_FAILURE;
  cudaStream_t xs = g_dev[g].xstream;
  const int64_t es = elem_size(dtk);
  talsh_tens_t* xt = sp.xop == 1 ? ltens : rtens;
  talsh_tens_t* yt = sp.xop == 1 ? rtens : ltens;
  char* dh = (char*)dtens->dev_rsc[o[0].src].gmem_p;
  char* xh = (char*)xt->dev_rsc[o[sp.xop].src].gmem_p;
  const char* yh = (const char*)yt->dev_rsc[o[3 - sp.xop].src].gmem_p;
  const int xrank = sp.xop == 1 ? P.lrank : P.rrank;
  int dd[MAX_TENSOR_RANK], xd[MAX_TENSOR_RANK];
  std::memcpy(dd, dtens->shape_p->dims, sizeof(int) * P.drank);
  std::memcpy(xd, xt->shape_p->dims, sizeof(int) * xrank);
  const int64_t din = prod_dims(dd, 0, sp.dpos), dout = prod_dims(dd, sp.dpos + 1, P.drank);
  const int64_t xin = prod_dims(xd, 0, sp.xpos), xout = prod_dims(xd, sp.xpos + 1, xrank);
  const size_t dslab = (size_t)(din * sp.step * dout * es), xslab = (size_t)(xin * sp.step * xout * es);
  const size_t ybytes = volume_of(yt) * es;
  void* yb = nullptr;
  void* db[2] = {nullptr, nullptr};
  void* xb[2] = {nullptr, nullptr};
  cudaEvent_t ev[8] = {};  // ready[2], computed[2], freed[2], start, copies_done
  int err = alloc_on(flat_gpu(g), ybytes, &yb, s);
  for (int i = 0; i < 2 && !err; ++i) {
    if ((err = alloc_on(flat_gpu(g), dslab, &db[i], s))) break;
    err = alloc_on(flat_gpu(g), xslab, &xb[i], s);
  }
  for (int i = 0; i < 8 && !err; ++i)
    if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) err = TALSH_FAILURE;
  cudaEvent_t *ready = ev, *computed = ev + 2, *freed = ev + 4, start = ev[6], copies_done = ev[7];
  const int64_t nsl = (sp.ext + sp.step - 1) / sp.step;
  if (!err) {
    cudaEventRecord(start, s);  // buffers allocated (stream-ordered on s)
    cudaStreamWaitEvent(xs, start, 0);
    if (cudaMemcpyAsync(yb, yh, ybytes, cudaMemcpyHostToDevice, xs) != cudaSuccess) err = TALSH_FAILURE;
    for (int64_t k = 0; k < nsl && !err; ++k) {
      const int slot = (int)(k & 1);
      const int64_t x0 = k * sp.step, w = std::min(sp.step, sp.ext - x0);
      if (k >= 2) cudaStreamWaitEvent(xs, freed[slot], 0);
      if (copy_slab(xb[slot], xh, xin, sp.ext, xout, x0, w, es, true, xs) != cudaSuccess) { err = TALSH_FAILURE; break; }
      const cudaError_t ce = accumulative ? copy_slab(db[slot], dh, din, sp.ext, dout, x0, w, es, true, xs)
                                          : cudaMemsetAsync(db[slot], 0, (size_t)(din * w * dout * es), xs);
      if (ce != cudaSuccess) { err = TALSH_FAILURE; break; }
      cudaEventRecord(ready[slot], xs);
      cudaStreamWaitEvent(s, ready[slot], 0);
      dd[sp.dpos] = (int)w;
      xd[sp.xpos] = (int)w;
      const void* lp = sp.xop == 1 ? xb[slot] : yb;
      const void* rp = sp.xop == 1 ? yb : xb[slot];
      const int* ldims = sp.xop == 1 ? xd : ltens->shape_p->dims;
      const int* rdims = sp.xop == 1 ? rtens->shape_p->dims : xd;
      err = map_tb(tb_tensor_contract(P.cptrn, dtk, P.drank, dd, db[slot], P.lrank, ldims, lp, P.rrank, rdims, rp, sr,
                                      si, P.conj_bits, accumulative, plan, s));
      cudaEventRecord(computed[slot], s);
      cudaStreamWaitEvent(xs, computed[slot], 0);
      if (!err && copy_slab(db[slot], dh, din, sp.ext, dout, x0, w, es, false, xs) != cudaSuccess) err = TALSH_FAILURE;
      cudaEventRecord(freed[slot], xs);
    }
    cudaEventRecord(copies_done, xs);
    cudaStreamWaitEvent(s, copies_done, 0);
  }
  if (err) cudaGetLastError();
  if (yb) cudaFreeAsync(yb, s);
  for (int i = 0; i < 2; ++i) {
    if (db[i]) cudaFreeAsync(db[i], s);
    if (xb[i]) cudaFreeAsync(xb[i], s);
  }
  cudaStreamSynchronize(s);
  for (auto& e : ev) if (e) cudaEventDestroy(e);
  g_last_split = sp;
  if (!err) g_last_split.step = nsl;  // reported: the number of slabs
  return err;
}

}  // namespace

extern "C" int talshTensorContract(const char* cptrn, talsh_tens_t* dtens, talsh_tens_t* ltens, talsh_tens_t* rtens,
                                   double sr, double si, int dev_id, int dev_kind, int copy_ctrl, int accumulative,
                                   talsh_task_t* task) {
  if (!cptrn || !dtens || !ltens || !rtens) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(dtens) == YEP || talshTensorIsEmpty(ltens) == YEP || talshTensorIsEmpty(rtens) == YEP)
    return TALSH_OBJECT_IS_EMPTY;
  tb::ParsedPattern P;
  if (tb::parse_pattern(cptrn, &P) || P.rrank < 0) return TALSH_INVALID_ARGS;
  if (P.drank != dtens->shape_p->num_dim || P.lrank != ltens->shape_p->num_dim || P.rrank != rtens->shape_p->num_dim)
    return TALSH_INVALID_ARGS;
  if (P.hyper) return TALSH_NOT_IMPLEMENTED;  // the reference's GPU path rejects hyper-indices too
  const int dtk = data_kind_of(dtens);
  if (dtk != data_kind_of(ltens) || dtk != data_kind_of(rtens)) return TALSH_INVALID_ARGS;
  tb::Matricization Z;
  if (tb::matricize(P.cptrn, P.drank, dtens->shape_p->dims, P.lrank, ltens->shape_p->dims, P.rrank,
                    rtens->shape_p->dims, &Z))
    return TALSH_INVALID_ARGS;
  const double flops = ((dtk == C4 || dtk == C8) ? 8.0 : 2.0) * (double)Z.M * (double)Z.N * (double)Z.K;
  const SliceSpec sp = plan_slices(P, ltens, rtens, dtk, copy_ctrl, dev_id, dev_kind);
  if (sp.big) {
    const std::vector<char> sliced{0, 1, 1};
    return run_op({dtens, ltens, rtens}, copy_ctrl, dev_id, dev_kind, task,
                  [&](cudaStream_t s, std::vector<Operand>& o) {
                    int g = 0; cudaGetDevice(&g);
                    tb_plan_t plan; std::memset(&plan, 0, sizeof(plan));
                    plan.method = g_dev[g].fast_math ? TB_METHOD_AUTO : TB_METHOD_TTGT;
                    return contract_streamed(P, sp, dtk, dtens, ltens, rtens, sr, si, accumulative, &plan, s, o);
                  }, flops, &sliced);
  }
  return run_op({dtens, ltens, rtens}, copy_ctrl, dev_id, dev_kind, task,
                [&](cudaStream_t s, std::vector<Operand>& o) {
                  int g = 0; cudaGetDevice(&g);
                  tb_plan_t plan; std::memset(&plan, 0, sizeof(plan));
                  plan.method = g_dev[g].fast_math ? TB_METHOD_AUTO : TB_METHOD_TTGT;
                  return map_tb(tb_tensor_contract(P.cptrn, dtk, P.drank, dtens->shape_p->dims, o[0].dptr, P.lrank,
                                                   ltens->shape_p->dims, o[1].dptr, P.rrank, rtens->shape_p->dims,
                                                   o[2].dptr, sr, si, P.conj_bits, accumulative, &plan, s));
                }, flops);
}

extern "C" int talshTensorContractXL(const char* cptrn, talsh_tens_t* dtens, talsh_tens_t* ltens, talsh_tens_t* rtens,
                                     double sr, double si, int dev_id, int dev_kind, int accumulative) {
  // The XL form is a blocking contraction (talshc.cpp:5394).  When D, L and R
  // live on the host and would not fit in the device budget together, D is
  // decomposed into slabs (contract_out_of_core); otherwise host-resident
  // inputs of 1 GiB and more stream through the GPU in slices
  // (contract_streamed) and D is staged whole.
  g_last_split = DSplit();
  if (!cptrn || !dtens || !ltens || !rtens) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(dtens) == YEP || talshTensorIsEmpty(ltens) == YEP || talshTensorIsEmpty(rtens) == YEP)
    return TALSH_OBJECT_IS_EMPTY;
  tb::ParsedPattern P;
  if (tb::parse_pattern(cptrn, &P) || P.rrank < 0) return TALSH_INVALID_ARGS;
  if (P.drank != dtens->shape_p->num_dim || P.lrank != ltens->shape_p->num_dim || P.rrank != rtens->shape_p->num_dim)
    return TALSH_INVALID_ARGS;
  const int dtk = data_kind_of(dtens);
  int gpu = -1;
  DSplit sp;
  if (!P.hyper && dtk == data_kind_of(ltens) && dtk == data_kind_of(rtens) && !resolve_gpu(dev_id, dev_kind, &gpu)) {
    tb::Matricization Z;
    if (!tb::matricize(P.cptrn, P.drank, dtens->shape_p->dims, P.lrank, ltens->shape_p->dims, P.rrank,
                       rtens->shape_p->dims, &Z))
      sp = plan_out_of_core(P, dtens, ltens, rtens, dtk, gpu);
    if (sp.dpos >= 0) {
      const double flops = ((dtk == C4 || dtk == C8) ? 8.0 : 2.0) * (double)Z.M * (double)Z.N * (double)Z.K;
      const std::vector<char> sliced{1, 1, 1};
      return run_op({dtens, ltens, rtens}, COPY_MTT, dev_id, dev_kind, nullptr,
                    [&](cudaStream_t s, std::vector<Operand>& o) {
                      int g = 0; cudaGetDevice(&g);
                      tb_plan_t plan; std::memset(&plan, 0, sizeof(plan));
                      plan.method = g_dev[g].fast_math ? TB_METHOD_AUTO : TB_METHOD_TTGT;
                      return contract_out_of_core(P, sp, dtk, dtens, ltens, rtens, sr, si, accumulative, &plan, s, o);
                    }, flops, &sliced);
    }
  }
  return talshTensorContract(cptrn, dtens, ltens, rtens, sr, si, dev_id, dev_kind, COPY_MTT, accumulative, nullptr);
}

extern "C" int tb_xl_last_split(int* d_dim, int* slabs) {
  if (!d_dim || !slabs) return TB_ERR_INVALID_ARGS;
  *d_dim = g_last_split.dpos;
  *slabs = g_last_split.dpos >= 0 ? (int)g_last_split.step : 0;
  return 0;
}

extern "C" int talshTensorGetScalar(talsh_tens_t* t, double* sr, double* si) {
  if (!t || !sr || !si) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) == YEP) return TALSH_OBJECT_IS_EMPTY;
  if (t->shape_p->num_dim != 0) return TALSH_INVALID_REQUEST;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->avail[i] != YEP) continue;
    double buf[2] = {0.0, 0.0};
    const int es = elem_size(t->data_kind[i]);
    if (t->dev_rsc[i].dev_id == 0) {
      std::memcpy(buf, t->dev_rsc[i].gmem_p, es);
    } else {
      const int g = gpu_of_flat(t->dev_rsc[i].dev_id);
      cudaSetDevice(g);
      cudaStreamSynchronize(g_dev[g].stream);
      if (cudaMemcpy(buf, t->dev_rsc[i].gmem_p, es, cudaMemcpyDeviceToHost) != cudaSuccess) return TALSH_FAILURE;
    }
    switch (t->data_kind[i]) {
      case R4: *sr = ((float*)buf)[0]; *si = 0.0; break;
      case R8: *sr = buf[0]; *si = 0.0; break;
      case C4: *sr = ((float*)buf)[0]; *si = ((float*)buf)[1]; break;
      case C8: *sr = buf[0]; *si = buf[1]; break;
    }
    return TALSH_SUCCESS;
  }
  return TALSH_NOT_FOUND;
}

extern "C" int talshTensorPlace(talsh_tens_t* t, int dev_id, int dev_kind, void* dev_mem, int copy_ctrl,
                                talsh_task_t* task) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g_on) return TALSH_NOT_INITIALIZED;
  if (!t) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) == YEP) return TALSH_OBJECT_IS_EMPTY;
  const int flat = dev_kind == DEV_NULL ? dev_id : talshFlatDevId(dev_kind, dev_id);
  if (flat < 0 || flat > MAX_GPUS_PER_NODE || (flat > 0 && !g_dev[flat - 1].on)) return TALSH_INVALID_ARGS;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) if (g_dev[g].on) { cudaSetDevice(g); cudaStreamSynchronize(g_dev[g].stream); }
  int src = find_image(t, flat);
  if (src < 0) {
    src = -1;
    for (int j = 0; j < t->ndev; ++j) if (t->avail[j] == YEP) { src = j; break; }
    if (src < 0) return TALSH_NOT_FOUND;
    const int dtk = t->data_kind[src];
    const size_t bytes = volume_of(t) * elem_size(dtk);
    void* p = dev_mem;
    const int work_gpu = flat > 0 ? flat - 1 : gpu_of_flat(t->dev_rsc[src].dev_id);
    cudaSetDevice(work_gpu);
    cudaStream_t s = g_dev[work_gpu].stream;
    if (!p) { if (int e = alloc_on(flat, bytes, &p, s)) return e; }
    const int sflat = t->dev_rsc[src].dev_id;
    cudaError_t ce;
    if (flat == 0) ce = cudaMemcpyAsync(p, t->dev_rsc[src].gmem_p, bytes, cudaMemcpyDeviceToHost, s);
    else if (sflat == 0) ce = cudaMemcpyAsync(p, t->dev_rsc[src].gmem_p, bytes, cudaMemcpyHostToDevice, s);
    else ce = cudaMemcpyPeerAsync(p, flat - 1, t->dev_rsc[src].gmem_p, sflat - 1, bytes, s);
    if (ce != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return TALSH_FAILURE;
    const int ni = add_image(t, flat, p, dtk, dev_mem ? 1 : 0);
    if (ni < 0) return TALSH_LIMIT_EXCEEDED;
    if (coh_of(copy_ctrl, 1, 0) == COPY_M || coh_of(copy_ctrl, 1, 0) == COPY_D) {
      void* sp = t->dev_rsc[src].gmem_p;
      for (int i = 0; i < t->ndev; ++i) if (t->dev_rsc[i].gmem_p == sp) { remove_image(t, i); break; }
    }
  }
  if (task) {
    if (talshTaskIsEmpty(task) != YEP) return TALSH_OBJECT_NOT_EMPTY;
    TaskImpl* ti = new TaskImpl();
    int g = 0;
    while (g < MAX_GPUS_PER_NODE && !g_dev[g].on) ++g;
    ti->gpu = g < MAX_GPUS_PER_NODE ? g : 0;
    cudaSetDevice(ti->gpu);
    for (auto& e : ti->ev) { cudaEventCreate(&e); cudaEventRecord(e, g_dev[ti->gpu].stream); }
    task->task_p = ti;
    task->dev_kind = flat == 0 ? DEV_HOST : DEV_NVIDIA_GPU;
  }
  return TALSH_SUCCESS;
}

extern "C" int talshTensorDiscard(talsh_tens_t* t, int dev_id, int dev_kind) {
  if (!t) return TALSH_INVALID_ARGS;
  const int flat = dev_kind == DEV_NULL ? dev_id : talshFlatDevId(dev_kind, dev_id);
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) if (g_dev[g].on) { cudaSetDevice(g); cudaStreamSynchronize(g_dev[g].stream); }
  for (int i = t->ndev - 1; i >= 0; --i) if (t->dev_rsc[i].dev_id == flat) remove_image(t, i);
  return TALSH_SUCCESS;
}

extern "C" int talshTensorDiscardOther(talsh_tens_t* t, int dev_id, int dev_kind) {
  if (!t) return TALSH_INVALID_ARGS;
  const int flat = dev_kind == DEV_NULL ? dev_id : talshFlatDevId(dev_kind, dev_id);
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) if (g_dev[g].on) { cudaSetDevice(g); cudaStreamSynchronize(g_dev[g].stream); }
  for (int i = t->ndev - 1; i >= 0; --i) if (t->dev_rsc[i].dev_id != flat) remove_image(t, i);
  return TALSH_SUCCESS;
}
