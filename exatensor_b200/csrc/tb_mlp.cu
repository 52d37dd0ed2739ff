// tb_mlp.cu -- the plan selector's network: a 3-layer MLP (in -> H -> H -> out,
// ReLU hidden layers, FP32) with hand-written forward, backward and Adam
// kernels.  Used to predict the log-runtime of every candidate contraction
// plan from a contraction descriptor; trained on autotuner timings.
//
// Layout: row-major activations [batch][features]; W_l is [in_l][out_l].
// All reductions run in a fixed order (one thread per output, sequential sum
// over the batch), so results are deterministic.
#include <cmath>
#include <cstring>
#include <vector>

#include "tb_common.cuh"

struct tb_mlp_s {
  int nin = 0, nh = 0, nout = 0, cap = 0;  // cap: allocated batch
  float* params = nullptr;                 // W1 b1 W2 b2 W3 b3
  float* grads = nullptr;
  float* m = nullptr;                      // Adam moments
  float* v = nullptr;
  float* act = nullptr;                    // z1 h1 z2 h2 y (cap rows each)
  float* dact = nullptr;                   // gradient buffers (cap x max(nh, nout)) x 2
  float* loss = nullptr;                   // device scalar
  size_t nparams = 0;
  int step = 0;
};

namespace tb {
namespace {

constexpr int kMlpT = 128;

struct Offs { size_t w1, b1, w2, b2, w3, b3, n; };
Offs offs(int nin, int nh, int nout) {
  Offs o;
  o.w1 = 0; o.b1 = o.w1 + (size_t)nin * nh;
  o.w2 = o.b1 + nh; o.b2 = o.w2 + (size_t)nh * nh;
  o.w3 = o.b2 + nh; o.b3 = o.w3 + (size_t)nh * nout;
  o.n = o.b3 + nout;
  return o;
}

// Y[b][o] = act(sum_i X[b][i] W[i][o] + bias[o]); Z keeps the pre-activation.
// One thread per output element; the weights of a column are read by all
// threads of the column (cached), X rows are broadcast within a block.
__global__ void mlp_dense_fwd(const float* __restrict__ X, const float* __restrict__ W, const float* __restrict__ bias,
                              float* __restrict__ Z, float* __restrict__ Y, int B, int I, int O, int relu) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (o >= O || b >= B) return;
  const float* x = X + (size_t)b * I;
  float acc = bias[o];
  for (int i = 0; i < I; ++i) acc = fmaf(x[i], W[(size_t)i * O + o], acc);
  if (Z) Z[(size_t)b * O + o] = acc;
  Y[(size_t)b * O + o] = relu ? fmaxf(acc, 0.f) : acc;
}

// dY = (Y - T) * mask * 2 / count, where mask = T is finite (missing labels
// are NaN).  The loss (mean squared error over the labelled entries) is
// reduced by one block in a fixed order.
__global__ void mlp_mse(const float* __restrict__ Y, const float* __restrict__ T, float* __restrict__ dY,
                        float* __restrict__ loss, int n) {
  __shared__ float sl[kMlpT];
  __shared__ float sc[kMlpT];
  float l = 0.f, c = 0.f;
  for (int i = threadIdx.x; i < n; i += kMlpT) {
    const float t = T[i];
    if (isfinite(t)) { const float d = Y[i] - t; l += d * d; c += 1.f; }
  }
  sl[threadIdx.x] = l;
  sc[threadIdx.x] = c;
  __syncthreads();
  for (int w = kMlpT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { sl[threadIdx.x] += sl[threadIdx.x + w]; sc[threadIdx.x] += sc[threadIdx.x + w]; }
    __syncthreads();
  }
  const float cnt = fmaxf(sc[0], 1.f);
  for (int i = threadIdx.x; i < n; i += kMlpT) {
    const float t = T[i];
    dY[i] = isfinite(t) ? 2.f * (Y[i] - t) / cnt : 0.f;
  }
  if (threadIdx.x == 0) *loss = sl[0] / cnt;
}

// dW[i][o] = sum_b X[b][i] dY[b][o];  db[o] = sum_b dY[b][o]  (sequential over b)
__global__ void mlp_dense_wgrad(const float* __restrict__ X, const float* __restrict__ dY, float* __restrict__ dW,
                                float* __restrict__ db, int B, int I, int O) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < I * O) {
    const int i = idx / O, o = idx % O;
    float acc = 0.f;
    for (int b = 0; b < B; ++b) acc = fmaf(X[(size_t)b * I + i], dY[(size_t)b * O + o], acc);
    dW[idx] = acc;
  } else if (idx < I * O + O) {
    const int o = idx - I * O;
    float acc = 0.f;
    for (int b = 0; b < B; ++b) acc += dY[(size_t)b * O + o];
    db[o] = acc;
  }
}

// dX[b][i] = (sum_o dY[b][o] W[i][o]) * (Z[b][i] > 0)   (ReLU of the layer below)
__global__ void mlp_dense_xgrad(const float* __restrict__ dY, const float* __restrict__ W,
                                const float* __restrict__ Zin, float* __restrict__ dX, int B, int I, int O) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (i >= I || b >= B) return;
  float acc = 0.f;
  for (int o = 0; o < O; ++o) acc = fmaf(dY[(size_t)b * O + o], W[(size_t)i * O + o], acc);
  dX[(size_t)b * I + i] = Zin[(size_t)b * I + i] > 0.f ? acc : 0.f;
}

__global__ void mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                         float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

float* dmalloc(size_t n, int* err) {
  void* p = nullptr;
  if (*err) return nullptr;
  if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    *err = TB_ERR_NO_MEMORY;
    return nullptr;
  }
  cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(float));
  return (float*)p;
}

// Forward pass for `batch` rows (batch <= cap) into the activation buffers.
int forward(tb_mlp_s* N, const float* X, int batch, cudaStream_t s) {
  const Offs o = offs(N->nin, N->nh, N->nout);
  float* z1 = N->act;
  float* h1 = z1 + (size_t)N->cap * N->nh;
  float* z2 = h1 + (size_t)N->cap * N->nh;
  float* h2 = z2 + (size_t)N->cap * N->nh;
  float* y = h2 + (size_t)N->cap * N->nh;
  const dim3 gh((N->nh + kMlpT - 1) / kMlpT, batch), go((N->nout + kMlpT - 1) / kMlpT, batch);
  mlp_dense_fwd<<<gh, kMlpT, 0, s>>>(X, N->params + o.w1, N->params + o.b1, z1, h1, batch, N->nin, N->nh, 1);
  TB_CHECK_LAUNCH();
  mlp_dense_fwd<<<gh, kMlpT, 0, s>>>(h1, N->params + o.w2, N->params + o.b2, z2, h2, batch, N->nh, N->nh, 1);
  TB_CHECK_LAUNCH();
  mlp_dense_fwd<<<go, kMlpT, 0, s>>>(h2, N->params + o.w3, N->params + o.b3, nullptr, y, batch, N->nh, N->nout, 0);
  TB_CHECK_LAUNCH();
  return 0;
}

}  // namespace
}  // namespace tb

using namespace tb;

extern "C" int tb_mlp_create(int nin, int nhidden, int nout, int max_batch, uint64_t seed, tb_mlp_t** out) {
  if (!out || nin < 1 || nhidden < 1 || nout < 1 || max_batch < 1) { set_error("tb_mlp_create: bad sizes"); return TB_ERR_INVALID_ARGS; }
  auto* N = new tb_mlp_s();
  N->nin = nin; N->nh = nhidden; N->nout = nout; N->cap = max_batch;
  const Offs o = offs(nin, nhidden, nout);
  N->nparams = o.n;
  int err = 0;
  N->params = dmalloc(o.n, &err);
  N->grads = dmalloc(o.n, &err);
  N->m = dmalloc(o.n, &err);
  N->v = dmalloc(o.n, &err);
  N->act = dmalloc((size_t)max_batch * (4 * (size_t)nhidden + nout), &err);
  N->dact = dmalloc((size_t)max_batch * 2 * std::max(nhidden, nout), &err);
  N->loss = dmalloc(1, &err);
  if (err) { set_error("tb_mlp_create: out of device memory"); tb_mlp_destroy(N); return err; }
  // He-style uniform initialisation from a splitmix64 stream (biases zero)
  std::vector<float> h(o.n, 0.f);
  uint64_t st = seed;
  auto u01 = [&st]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](size_t off, int fan_in, size_t n) {
    const double a = std::sqrt(6.0 / fan_in);
    for (size_t i = 0; i < n; ++i) h[off + i] = (float)((2.0 * u01() - 1.0) * a);
  };
  fill(o.w1, nin, (size_t)nin * nhidden);
  fill(o.w2, nhidden, (size_t)nhidden * nhidden);
  fill(o.w3, nhidden, (size_t)nhidden * nout);
  if (cudaMemcpy(N->params, h.data(), o.n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    tb_mlp_destroy(N);
    return TB_ERR_CUDA;
  }
  *out = N;
  return 0;
}

extern "C" int tb_mlp_destroy(tb_mlp_t* N) {
  if (!N) return 0;
  for (float* p : {N->params, N->grads, N->m, N->v, N->act, N->dact, N->loss})
    if (p) cudaFree(p);
  delete N;
  return 0;
}

extern "C" long long tb_mlp_num_params(const tb_mlp_t* N) { return N ? (long long)N->nparams : 0; }

extern "C" int tb_mlp_get_params(const tb_mlp_t* N, float* host, int grads) {
  if (!N || !host) return TB_ERR_INVALID_ARGS;
  if (cudaMemcpy(host, grads ? N->grads : N->params, N->nparams * sizeof(float), cudaMemcpyDeviceToHost) !=
      cudaSuccess) {
    cudaGetLastError();
    return TB_ERR_CUDA;
  }
  return 0;
}

extern "C" int tb_mlp_set_params(tb_mlp_t* N, const float* host) {
  if (!N || !host) return TB_ERR_INVALID_ARGS;
  if (cudaMemcpy(N->params, host, N->nparams * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    return TB_ERR_CUDA;
  }
  cudaMemset(N->m, 0, N->nparams * sizeof(float));
  cudaMemset(N->v, 0, N->nparams * sizeof(float));
  N->step = 0;
  return 0;
}

// Inference: Y[batch][nout] (device) from X[batch][nin] (device), in chunks of the capacity.
extern "C" int tb_mlp_forward(tb_mlp_t* N, const float* X, int batch, float* Y, void* stream) {
  if (!N || !X || !Y || batch < 0) return TB_ERR_INVALID_ARGS;
  cudaStream_t s = (cudaStream_t)stream;
  for (int b0 = 0; b0 < batch; b0 += N->cap) {
    const int nb = std::min(N->cap, batch - b0);
    if (int e = forward(N, X + (size_t)b0 * N->nin, nb, s)) return e;
    float* y = N->act + (size_t)N->cap * 4 * N->nh;
    if (cudaMemcpyAsync(Y + (size_t)b0 * N->nout, y, (size_t)nb * N->nout * sizeof(float), cudaMemcpyDeviceToDevice,
                        s) != cudaSuccess)
      return TB_ERR_CUDA;
  }
  return 0;
}

// Loss and gradients of the batch (batch <= capacity); targets T[batch][nout]
// (NaN = no label).  Gradients stay on the device (tb_mlp_get_params(.., 1)).
extern "C" int tb_mlp_backward(tb_mlp_t* N, const float* X, const float* T, int batch, float* loss_host,
                               void* stream) {
  if (!N || !X || !T || batch < 1 || batch > N->cap) return TB_ERR_INVALID_ARGS;
  cudaStream_t s = (cudaStream_t)stream;
  if (int e = forward(N, X, batch, s)) return e;
  const Offs o = offs(N->nin, N->nh, N->nout);
  const size_t H = (size_t)N->cap * N->nh;
  float* z1 = N->act;
  float* h1 = z1 + H;
  float* z2 = h1 + H;
  float* h2 = z2 + H;
  float* y = h2 + H;
  const size_t D = (size_t)N->cap * std::max(N->nh, N->nout);
  float* dy = N->dact;       // [batch][nout], then reused
  float* dh = N->dact + D;   // [batch][nh]
  mlp_mse<<<1, kMlpT, 0, s>>>(y, T, dy, N->loss, batch * N->nout);
  TB_CHECK_LAUNCH();
  auto wgrad = [&](const float* X_, const float* dY_, size_t wo, size_t bo, int I, int O) {
    const int n = I * O + O;
    mlp_dense_wgrad<<<(n + kMlpT - 1) / kMlpT, kMlpT, 0, s>>>(X_, dY_, N->grads + wo, N->grads + bo, batch, I, O);
  };
  wgrad(h2, dy, o.w3, o.b3, N->nh, N->nout);
  TB_CHECK_LAUNCH();
  mlp_dense_xgrad<<<dim3((N->nh + kMlpT - 1) / kMlpT, batch), kMlpT, 0, s>>>(dy, N->params + o.w3, z2, dh, batch, N->nh,
                                                                          N->nout);
  TB_CHECK_LAUNCH();
  wgrad(h1, dh, o.w2, o.b2, N->nh, N->nh);
  TB_CHECK_LAUNCH();
  mlp_dense_xgrad<<<dim3((N->nh + kMlpT - 1) / kMlpT, batch), kMlpT, 0, s>>>(dh, N->params + o.w2, z1, dy, batch, N->nh,
                                                                          N->nh);
  TB_CHECK_LAUNCH();
  wgrad(X, dy, o.w1, o.b1, N->nin, N->nh);
  TB_CHECK_LAUNCH();
  if (loss_host) {
    if (cudaMemcpyAsync(loss_host, N->loss, sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return TB_ERR_CUDA;
  }
  return 0;
}

extern "C" int tb_mlp_adam_step(tb_mlp_t* N, float lr, float beta1, float beta2, float eps, void* stream) {
  if (!N) return TB_ERR_INVALID_ARGS;
  ++N->step;
  const float c1 = 1.f - std::pow(beta1, (float)N->step), c2 = 1.f - std::pow(beta2, (float)N->step);
  const int grid = (int)std::min<size_t>((N->nparams + 255) / 256, 1024);
  mlp_adam<<<grid, 256, 0, (cudaStream_t)stream>>>(N->params, N->grads, N->m, N->v, N->nparams, lr, beta1, beta2, eps,
                                                     c1, c2);
  TB_CHECK_LAUNCH();
  return 0;
}
