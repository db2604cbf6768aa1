// lp_mlp.cu - training of the Herschel-Bulkley warm-start network on the device
// (forward, backward, Adam), no reference counterpart.
//
// Minibatch step, batch B:
//   k_mlp_sample : per sample, forward pass and back-propagation of the squared error to the
//                  hidden pre-activations (dZ1, dZ2), stored with the activations (H1, H2);
//   k_mlp_wgrad  : weight gradients as fixed-order sums over the batch, split in S slices whose
//                  partials are summed in slice order (deterministic);
//   k_mlp_adam   : Adam update.
// Loss = mean over the batch of (out - y)^2, with y = logit of the root fraction.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lp_mpm.h"
#include "lp_kernels.h"
#include "lp_mlp.cuh"

namespace lp {

constexpr int MLP_SPLIT = 16;

__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// per sample forward + backward to the pre-activations
__global__ void k_mlp_sample(const float* __restrict__ W, const float* __restrict__ X, const float* __restrict__ Y,
                             int64_t n, float* __restrict__ H1, float* __restrict__ H2, float* __restrict__ dZ1,
                             float* __restrict__ dZ2, float* __restrict__ G3, float* __restrict__ loss_part) {
  __shared__ float sw[MLP_NW];
  __shared__ float sl[256];
  for (int j = threadIdx.x; j < MLP_NW; j += blockDim.x) sw[j] = W[j];
  __syncthreads();
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (s < n) {
    float x[MLP_IN];
    for (int i = 0; i < MLP_IN; ++i) x[i] = X[s * MLP_IN + i];
    float z1[MLP_H], h1[MLP_H];
    for (int j = 0; j < MLP_H; ++j) {
      float a = sw[MLP_B1 + j];
      for (int i = 0; i < MLP_IN; ++i) a += sw[MLP_W1 + j * MLP_IN + i] * x[i];
      z1[j] = a;
      h1[j] = silu(a);
      H1[s * MLP_H + j] = h1[j];
    }
    float out = sw[MLP_B3];
    float z2[MLP_H];
    for (int j = 0; j < MLP_H; ++j) {
      float a = sw[MLP_B2 + j];
      for (int i = 0; i < MLP_H; ++i) a += sw[MLP_W2 + j * MLP_H + i] * h1[i];
      z2[j] = a;
      const float h = silu(a);
      H2[s * MLP_H + j] = h;
      out += sw[MLP_W3 + j] * h;
    }
    const float e = out - Y[s];
    l = e * e;
    const float g3 = 2.0f * e / (float)n;
    G3[s] = g3;
    float dz2[MLP_H];
    for (int j = 0; j < MLP_H; ++j) {
      dz2[j] = g3 * sw[MLP_W3 + j] * silu_grad(z2[j]);
      dZ2[s * MLP_H + j] = dz2[j];
    }
    for (int i = 0; i < MLP_H; ++i) {
      float a = 0.0f;
      for (int j = 0; j < MLP_H; ++j) a += sw[MLP_W2 + j * MLP_H + i] * dz2[j];
      dZ1[s * MLP_H + i] = a * silu_grad(z1[i]);
    }
  }
  sl[threadIdx.x] = l;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sl[threadIdx.x] += sl[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = sl[0];
}

// weight gradients: partial sums over batch slice `blockIdx.y`, one thread per weight
__global__ void k_mlp_wgrad(const float* __restrict__ X, const float* __restrict__ H1, const float* __restrict__ H2,
                            const float* __restrict__ dZ1, const float* __restrict__ dZ2, const float* __restrict__ G3,
                            int64_t n, float* __restrict__ part) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= MLP_NW) return;
  const int slice = blockIdx.y;
  const int64_t per = (n + MLP_SPLIT - 1) / MLP_SPLIT;
  const int64_t s0 = slice * per, s1 = s0 + per < n ? s0 + per : n;
  float acc = 0.0f;
  if (w < MLP_B1) {
    const int j = (w - MLP_W1) / MLP_IN, i = (w - MLP_W1) % MLP_IN;
    for (int64_t s = s0; s < s1; ++s) acc += dZ1[s * MLP_H + j] * X[s * MLP_IN + i];
  } else if (w < MLP_W2) {
    const int j = w - MLP_B1;
    for (int64_t s = s0; s < s1; ++s) acc += dZ1[s * MLP_H + j];
  } else if (w < MLP_B2) {
    const int j = (w - MLP_W2) / MLP_H, i = (w - MLP_W2) % MLP_H;
    for (int64_t s = s0; s < s1; ++s) acc += dZ2[s * MLP_H + j] * H1[s * MLP_H + i];
  } else if (w < MLP_W3) {
    const int j = w - MLP_B2;
    for (int64_t s = s0; s < s1; ++s) acc += dZ2[s * MLP_H + j];
  } else if (w < MLP_B3) {
    const int j = w - MLP_W3;
    for (int64_t s = s0; s < s1; ++s) acc += G3[s] * H2[s * MLP_H + j];
  } else {
    for (int64_t s = s0; s < s1; ++s) acc += G3[s];
  }
  part[(int64_t)slice * MLP_NW + w] = acc;
}

__global__ void k_mlp_gsum(const float* __restrict__ part, float* __restrict__ grad) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= MLP_NW) return;
  float g = 0.0f;
  for (int s = 0; s < MLP_SPLIT; ++s) g += part[(int64_t)s * MLP_NW + w];
  grad[w] = g;
}

__global__ void k_mlp_adam(float* __restrict__ W, const float* __restrict__ grad, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float b1t, float b2t) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= MLP_NW) return;
  const float g = grad[w];
  const float a = 0.9f * m1[w] + 0.1f * g;
  const float b = 0.999f * m2[w] + 0.001f * g * g;
  m1[w] = a;
  m2[w] = b;
  const float ah = a / (1.0f - b1t), bh = b / (1.0f - b2t);
  W[w] -= lr * ah / (sqrtf(bh) + 1e-8f);
}

__global__ void k_mlp_loss_final(const float* __restrict__ part, int nparts, int64_t n, float* __restrict__ loss) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < nparts; ++i) s += part[i];
  loss[0] = (float)(s / (double)n);
}

__global__ void k_mlp_infer(const float* __restrict__ W, const float* __restrict__ X, int64_t n, float* __restrict__ Y) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float f[MLP_IN];
  for (int i = 0; i < MLP_IN; ++i) f[i] = X[s * MLP_IN + i];
  Y[s] = mlp_forward(W, f);
}

__global__ void k_mlp_pack(const float* __restrict__ W, MlpPacked* __restrict__ P) {
  mlp_pack_words(W, *P, (int)(blockIdx.x * blockDim.x + threadIdx.x), (int)(gridDim.x * blockDim.x));
}

void launch_mlp_pack(const float* W, MlpPacked* P, cudaStream_t s) {
  k_mlp_pack<<<8, 256, 0, s>>>(W, P);
  add_kernel_launches(1);
}

// tensor-core inference of the network (the path the solver uses), on feature rows
__global__ void __launch_bounds__(128) k_mlp_infer_mma(const MlpPacked* __restrict__ P, const float* __restrict__ X,
                                                       int64_t n, float* __restrict__ Y) {
  __shared__ MlpPacked S;
  __shared__ uint32_t xs[4 * MLP_XS_WORDS];
  mlp_stage(P, S);
  __syncthreads();
  if ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u) >= n) return;  // warp-uniform
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = i0 < n ? i0 : n - 1;
  float f[MLP_IN];
#pragma unroll
  for (int j = 0; j < MLP_IN; ++j) f[j] = X[i * MLP_IN + j];
  const float y = warp_mlp_logit(S, xs + (threadIdx.x >> 5) * MLP_XS_WORDS, f);
  if (i0 < n) Y[i0] = y;
}

}  // namespace lp

namespace {
thread_local std::string g_mlp_err;
lp_status mlp_fail(lp_status s, const std::string& m) {
  g_mlp_err = m;
  lp::set_last_error(m.c_str());
  return s;
}
#define MCK(expr)                                                                                 \
  do {                                                                                            \
    cudaError_t _e = (expr);                                                                      \
    if (_e != cudaSuccess) return mlp_fail(LP_DEVICE, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

struct MlpBuffers {
  float *W = nullptr, *X = nullptr, *Y = nullptr, *H1 = nullptr, *H2 = nullptr, *dZ1 = nullptr, *dZ2 = nullptr,
        *G3 = nullptr, *loss = nullptr, *part = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  int64_t batch = 0;
  ~MlpBuffers() {
    float* ps[] = {W, X, Y, H1, H2, dZ1, dZ2, G3, loss, part, grad, m1, m2};
    for (float* p : ps)
      if (p) cudaFree(p);
  }
  lp_status alloc(int64_t b) {
    batch = b;
    MCK(cudaMalloc(&W, sizeof(float) * lp::MLP_NW));
    MCK(cudaMalloc(&H1, sizeof(float) * b * lp::MLP_H));
    MCK(cudaMalloc(&H2, sizeof(float) * b * lp::MLP_H));
    MCK(cudaMalloc(&dZ1, sizeof(float) * b * lp::MLP_H));
    MCK(cudaMalloc(&dZ2, sizeof(float) * b * lp::MLP_H));
    MCK(cudaMalloc(&G3, sizeof(float) * b));
    MCK(cudaMalloc(&loss, sizeof(float) * ((b + 255) / 256)));
    MCK(cudaMalloc(&part, sizeof(float) * lp::MLP_SPLIT * lp::MLP_NW));
    MCK(cudaMalloc(&grad, sizeof(float) * lp::MLP_NW));
    MCK(cudaMalloc(&m1, sizeof(float) * lp::MLP_NW));
    MCK(cudaMalloc(&m2, sizeof(float) * lp::MLP_NW));
    MCK(cudaMemset(m1, 0, sizeof(float) * lp::MLP_NW));
    MCK(cudaMemset(m2, 0, sizeof(float) * lp::MLP_NW));
    return LP_OK;
  }
};

// loss and gradient of one batch (X, Y device pointers) into B.grad; returns mean loss
lp_status batch_grad(MlpBuffers& B, const float* X, const float* Y, int64_t n, float* loss_out) {
  const unsigned nb = (unsigned)((n + 255) / 256);
  lp::k_mlp_sample<<<nb, 256>>>(B.W, X, Y, n, B.H1, B.H2, B.dZ1, B.dZ2, B.G3, B.loss);
  dim3 g((lp::MLP_NW + 255) / 256, lp::MLP_SPLIT);
  lp::k_mlp_wgrad<<<g, 256>>>(X, B.H1, B.H2, B.dZ1, B.dZ2, B.G3, n, B.part);
  lp::k_mlp_gsum<<<(lp::MLP_NW + 255) / 256, 256>>>(B.part, B.grad);
  lp::add_kernel_launches(3);
  MCK(cudaGetLastError());
  if (loss_out) {
    std::vector<float> lp_(nb);
    MCK(cudaMemcpy(lp_.data(), B.loss, sizeof(float) * nb, cudaMemcpyDeviceToHost));
    double s = 0.0;
    for (float v : lp_) s += v;
    *loss_out = (float)(s / (double)n);
  }
  return LP_OK;
}

uint64_t splitmix(uint64_t& s) {
  s += 0x9E3779B97F4A7C15ull;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
}  // namespace

// Work space of lp_mlp_loss_grad_noalloc: a fixed static device array, so that callers who
// cannot allocate device memory can still evaluate the loss and gradient.  Layout (floats):
// H1, H2, dZ1, dZ2 [NOALLOC_MAX * 64 each], G3 [NOALLOC_MAX], loss partials, gradient partials.
namespace {
constexpr int64_t NOALLOC_MAX = LP_MLP_NOALLOC_MAX_SAMPLES;
constexpr int64_t NA_H1 = 0;
constexpr int64_t NA_H2 = NA_H1 + NOALLOC_MAX * lp::MLP_H;
constexpr int64_t NA_DZ1 = NA_H2 + NOALLOC_MAX * lp::MLP_H;
constexpr int64_t NA_DZ2 = NA_DZ1 + NOALLOC_MAX * lp::MLP_H;
constexpr int64_t NA_G3 = NA_DZ2 + NOALLOC_MAX * lp::MLP_H;
constexpr int64_t NA_LOSS = NA_G3 + NOALLOC_MAX;
constexpr int64_t NA_PART = NA_LOSS + (NOALLOC_MAX + 255) / 256;
constexpr int64_t NA_TOTAL = NA_PART + (int64_t)lp::MLP_SPLIT * lp::MLP_NW;
constexpr int kMaxDevices = 64;
// Device address of g_noalloc_scratch per device, looked up once.  Atomic so that host threads
// making their first call at the same time both store the same address without a data race.
std::atomic<float*> g_noalloc_ptr[kMaxDevices];

// Device buffers of one allocating call, freed on every return path.
struct DevBufs {
  std::vector<void*> ptrs;
  ~DevBufs() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  cudaError_t alloc(T** p, size_t bytes) {
    *p = nullptr;
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, bytes);
    if (e == cudaSuccess) {
      ptrs.push_back(q);
      *p = static_cast<T*>(q);
    }
    return e;
  }
};
}  // namespace

static __device__ __align__(256) float g_noalloc_scratch[NA_TOTAL];

extern "C" {

int32_t lp_mlp_weight_count(void) { return lp::MLP_NW; }

lp_status lp_mlp_loss_grad_noalloc(const float* w, const float* x, const float* y, int64_t n, float* loss,
                                   float* grad, void* stream) {
  if (!w || !x || !y || !loss || !grad) return mlp_fail(LP_INVALID, "null argument");
  if (n <= 0 || n > NOALLOC_MAX)
    return mlp_fail(LP_INVALID, "n=" + std::to_string(n) + " is outside 1.." + std::to_string(NOALLOC_MAX) +
                                    " (the fixed work space of lp_mlp_loss_grad_noalloc)");
  int dev = 0;
  MCK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return mlp_fail(LP_DEVICE, "device index out of range");
  float* S = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (S == nullptr) {
    // one-time set-up on this device: the host-side name is not a device address
    void* ptr = nullptr;
    MCK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    S = static_cast<float*>(ptr);
    g_noalloc_ptr[dev].store(S, std::memory_order_release);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned nb = (unsigned)((n + 255) / 256);
  lp::k_mlp_sample<<<nb, 256, 0, st>>>(w, x, y, n, S + NA_H1, S + NA_H2, S + NA_DZ1, S + NA_DZ2, S + NA_G3,
                                       S + NA_LOSS);
  dim3 g((lp::MLP_NW + 255) / 256, lp::MLP_SPLIT);
  lp::k_mlp_wgrad<<<g, 256, 0, st>>>(x, S + NA_H1, S + NA_H2, S + NA_DZ1, S + NA_DZ2, S + NA_G3, n, S + NA_PART);
  lp::k_mlp_gsum<<<(lp::MLP_NW + 255) / 256, 256, 0, st>>>(S + NA_PART, grad);
  lp::k_mlp_loss_final<<<1, 1, 0, st>>>(S + NA_LOSS, (int)nb, n, loss);
  lp::add_kernel_launches(4);
  MCK(cudaGetLastError());
  return LP_OK;
}

lp_status lp_mlp_init(float* w, int32_t nw, uint64_t seed) {
  if (!w || nw != lp::MLP_NW) return mlp_fail(LP_INVALID, "weight count mismatch");
  uint64_t s = seed;
  auto uni = [&]() { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); };
  const double a1 = std::sqrt(6.0 / (lp::MLP_IN + lp::MLP_H)), a2 = std::sqrt(6.0 / (2 * lp::MLP_H)),
               a3 = std::sqrt(6.0 / (lp::MLP_H + 1));
  for (int k = 0; k < lp::MLP_NW; ++k) {
    double a = 0.0;
    if (k < lp::MLP_B1) a = a1;
    else if (k >= lp::MLP_W2 && k < lp::MLP_B2) a = a2;
    else if (k >= lp::MLP_W3 && k < lp::MLP_B3) a = a3;
    w[k] = (float)((2.0 * uni() - 1.0) * a);
  }
  return LP_OK;
}

lp_status lp_mlp_loss_grad(const float* w, int32_t nw, const float* x, const float* y, int64_t n, float* loss,
                           float* grad) {
  if (!w || nw != lp::MLP_NW || n <= 0) return mlp_fail(LP_INVALID, "bad arguments");
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) return mlp_fail(LP_DEVICE, "no CUDA device");
  MlpBuffers B;
  lp_status st = B.alloc(n);
  if (st != LP_OK) return st;
  MCK(cudaMalloc(&B.X, sizeof(float) * n * lp::MLP_IN));  // owned by B from here on
  MCK(cudaMalloc(&B.Y, sizeof(float) * n));
  float *X = B.X, *Y = B.Y;
  MCK(cudaMemcpy(B.W, w, sizeof(float) * lp::MLP_NW, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(X, x, sizeof(float) * n * lp::MLP_IN, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(Y, y, sizeof(float) * n, cudaMemcpyHostToDevice));
  st = batch_grad(B, X, Y, n, loss);
  if (st != LP_OK) return st;
  MCK(cudaMemcpy(grad, B.grad, sizeof(float) * lp::MLP_NW, cudaMemcpyDeviceToHost));
  return LP_OK;
}

lp_status lp_mlp_train(float* w, int32_t nw, const float* x, const float* y, int64_t n, int32_t epochs, int32_t batch,
                       float lr, float* final_loss) {
  if (!w || nw != lp::MLP_NW || n <= 0 || batch <= 0 || epochs <= 0) return mlp_fail(LP_INVALID, "bad arguments");
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) return mlp_fail(LP_DEVICE, "no CUDA device");
  const int64_t b = std::min<int64_t>(batch, n);
  MlpBuffers B;
  lp_status st = B.alloc(b);
  if (st != LP_OK) return st;
  MCK(cudaMalloc(&B.X, sizeof(float) * n * lp::MLP_IN));  // owned by B from here on
  MCK(cudaMalloc(&B.Y, sizeof(float) * n));
  float *X = B.X, *Y = B.Y;
  MCK(cudaMemcpy(B.W, w, sizeof(float) * lp::MLP_NW, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(X, x, sizeof(float) * n * lp::MLP_IN, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(Y, y, sizeof(float) * n, cudaMemcpyHostToDevice));
  double b1t = 1.0, b2t = 1.0;
  float last = 0.0f;
  const int64_t steps_per_epoch = n / b;
  for (int e = 0; e < epochs; ++e) {
    // the host shuffles sample order by choosing contiguous batches of a pre-shuffled set;
    // callers pass shuffled data, batches cycle through it in order
    double eloss = 0.0;
    for (int64_t k = 0; k < steps_per_epoch; ++k) {
      const float* xb = X + k * b * lp::MLP_IN;
      const float* yb = Y + k * b;
      float l = 0.0f;
      const bool want = (k == steps_per_epoch - 1);
      st = batch_grad(B, xb, yb, b, want ? &l : nullptr);
      if (st != LP_OK) return st;
      b1t *= 0.9;
      b2t *= 0.999;
      lp::k_mlp_adam<<<(lp::MLP_NW + 255) / 256, 256>>>(B.W, B.grad, B.m1, B.m2, lr, (float)b1t, (float)b2t);
      lp::add_kernel_launches(1);
      if (want) eloss = l;
    }
    last = (float)eloss;
  }
  MCK(cudaDeviceSynchronize());
  MCK(cudaMemcpy(w, B.W, sizeof(float) * lp::MLP_NW, cudaMemcpyDeviceToHost));
  if (final_loss) *final_loss = last;
  return LP_OK;
}

lp_status lp_mlp_forward(const float* w, int32_t nw, const float* x, int64_t n, float* y) {
  if (!w || nw != lp::MLP_NW || n <= 0) return mlp_fail(LP_INVALID, "bad arguments");
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) return mlp_fail(LP_DEVICE, "no CUDA device");
  DevBufs bufs;  // freed on every return path
  float *W = nullptr, *X = nullptr, *Y = nullptr;
  MCK(bufs.alloc(&W, sizeof(float) * lp::MLP_NW));
  MCK(bufs.alloc(&X, sizeof(float) * n * lp::MLP_IN));
  MCK(bufs.alloc(&Y, sizeof(float) * n));
  MCK(cudaMemcpy(W, w, sizeof(float) * lp::MLP_NW, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(X, x, sizeof(float) * n * lp::MLP_IN, cudaMemcpyHostToDevice));
  lp::k_mlp_infer<<<(unsigned)((n + 255) / 256), 256>>>(W, X, n, Y);
  lp::add_kernel_launches(1);
  MCK(cudaGetLastError());
  MCK(cudaMemcpy(y, Y, sizeof(float) * n, cudaMemcpyDeviceToHost));
  return LP_OK;
}

lp_status lp_mlp_forward_mma(const float* w, int32_t nw, const float* x, int64_t n, float* y) {
  if (!w || nw != lp::MLP_NW || n <= 0) return mlp_fail(LP_INVALID, "bad arguments");
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) return mlp_fail(LP_DEVICE, "no CUDA device");
  DevBufs bufs;  // freed on every return path
  float *W = nullptr, *X = nullptr, *Y = nullptr;
  lp::MlpPacked* P = nullptr;
  MCK(bufs.alloc(&W, sizeof(float) * lp::MLP_NW));
  MCK(bufs.alloc(&P, sizeof(lp::MlpPacked)));
  MCK(bufs.alloc(&X, sizeof(float) * n * lp::MLP_IN));
  MCK(bufs.alloc(&Y, sizeof(float) * n));
  MCK(cudaMemcpy(W, w, sizeof(float) * lp::MLP_NW, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(X, x, sizeof(float) * n * lp::MLP_IN, cudaMemcpyHostToDevice));
  lp::launch_mlp_pack(W, P, 0);
  lp::k_mlp_infer_mma<<<(unsigned)((n + 127) / 128), 128>>>(P, X, n, Y);
  lp::add_kernel_launches(1);
  MCK(cudaGetLastError());
  MCK(cudaMemcpy(y, Y, sizeof(float) * n, cudaMemcpyDeviceToHost));
  return LP_OK;
}

}  // extern "C"
