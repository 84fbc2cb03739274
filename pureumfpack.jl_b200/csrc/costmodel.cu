// costmodel.cu -- the learned part of the autotuner: a small MLP trained on
// the GPU by this library's own kernels.
//
// The network maps the features of one batched GEMM launch (its flops,
// bytes, task and tile counts, mean shapes, kind, precision and the kernel
// variant) to the log of its device time; the autotuner asks it for every
// variant of every tunable launch and picks the fastest.  The network only
// schedules: every variant computes the same update.  No counterpart in the
// reference, which runs on the CPU with one code path.
//
// Layers: nin -> H -> H -> 1, tanh hidden activations, mean-squared error on
// the (already standardised) targets, Adam.  Parameters are FP32 and laid out
// as W1 (H x nin, row-major), b1 (H), W2 (H x H), b2 (H), w3 (H), b3 (1).
// Training is deterministic: per-sample deltas, then one thread per parameter
// sums its gradient over the samples in a fixed order.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/mfgpu.h"

namespace {

constexpr int kMaxHidden = 64;
constexpr int kMaxIn = 32;

struct Layout {
  int nin, h;
  int w1, b1, w2, b2, w3, b3, total;
  __host__ __device__ Layout(int nin_, int h_) : nin(nin_), h(h_) {
    w1 = 0;
    b1 = w1 + h * nin;
    w2 = b1 + h;
    b2 = w2 + h * h;
    w3 = b2 + h;
    b3 = w3 + h;
    total = b3 + 1;
  }
};

// Forward pass, one thread per sample; keeps both hidden activations.
__global__ void k_mlp_forward(const float* __restrict__ p, int nin, int h, const float* __restrict__ X, int64_t n,
                              float* __restrict__ a1, float* __restrict__ a2, float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Layout L(nin, h);
  float x[kMaxIn], z1[kMaxHidden], z2[kMaxHidden];
  for (int k = 0; k < nin; ++k) x[k] = X[i * nin + k];
  for (int j = 0; j < h; ++j) {
    float s = p[L.b1 + j];
    for (int k = 0; k < nin; ++k) s += p[L.w1 + j * nin + k] * x[k];
    z1[j] = tanhf(s);
    a1[i * h + j] = z1[j];
  }
  for (int j = 0; j < h; ++j) {
    float s = p[L.b2 + j];
    for (int k = 0; k < h; ++k) s += p[L.w2 + j * h + k] * z1[k];
    z2[j] = tanhf(s);
    a2[i * h + j] = z2[j];
  }
  float s = p[L.b3];
  for (int k = 0; k < h; ++k) s += p[L.w3 + k] * z2[k];
  out[i] = s;
}

// Per-sample deltas of the loss (1/n) sum (out - y)^2 at every layer's
// pre-activation: d3 (n), d2 (n x h), d1 (n x h).
__global__ void k_mlp_deltas(const float* __restrict__ p, int nin, int h, const float* __restrict__ Y, int64_t n,
                             const float* __restrict__ a1, const float* __restrict__ a2,
                             const float* __restrict__ out, float* __restrict__ d1, float* __restrict__ d2,
                             float* __restrict__ d3) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Layout L(nin, h);
  const float g3 = 2.0f * (out[i] - Y[i]) / (float)n;
  d3[i] = g3;
  float g2[kMaxHidden];
  for (int j = 0; j < h; ++j) {
    const float a = a2[i * h + j];
    g2[j] = g3 * p[L.w3 + j] * (1.0f - a * a);
    d2[i * h + j] = g2[j];
  }
  for (int k = 0; k < h; ++k) {
    float s = 0.0f;
    for (int j = 0; j < h; ++j) s += p[L.w2 + j * h + k] * g2[j];
    const float a = a1[i * h + k];
    d1[i * h + k] = s * (1.0f - a * a);
  }
}

// One thread per parameter: its gradient summed over the samples in order.
__global__ void k_mlp_param_grads(int nin, int h, const float* __restrict__ X, int64_t n,
                                  const float* __restrict__ a1, const float* __restrict__ a2,
                                  const float* __restrict__ d1, const float* __restrict__ d2,
                                  const float* __restrict__ d3, float* __restrict__ grad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const Layout L(nin, h);
  if (q >= L.total) return;
  float s = 0.0f;
  if (q < L.b1) {                       // W1[j][k]
    const int j = q / nin, k = q % nin;
    for (int64_t i = 0; i < n; ++i) s += d1[i * h + j] * X[i * nin + k];
  } else if (q < L.w2) {                // b1[j]
    const int j = q - L.b1;
    for (int64_t i = 0; i < n; ++i) s += d1[i * h + j];
  } else if (q < L.b2) {                // W2[j][k]
    const int j = (q - L.w2) / h, k = (q - L.w2) % h;
    for (int64_t i = 0; i < n; ++i) s += d2[i * h + j] * a1[i * h + k];
  } else if (q < L.w3) {                // b2[j]
    const int j = q - L.b2;
    for (int64_t i = 0; i < n; ++i) s += d2[i * h + j];
  } else if (q < L.b3) {                // w3[k]
    const int k = q - L.w3;
    for (int64_t i = 0; i < n; ++i) s += d3[i] * a2[i * h + k];
  } else {                              // b3
    for (int64_t i = 0; i < n; ++i) s += d3[i];
  }
  grad[q] = s;
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int np, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  m[q] = b1 * m[q] + (1.0f - b1) * g[q];
  v[q] = b2 * v[q] + (1.0f - b2) * g[q] * g[q];
  p[q] -= lr * (m[q] / c1) / (sqrtf(v[q] / c2) + eps);
}

__global__ void k_sq_loss(const float* __restrict__ out, const float* __restrict__ Y, int64_t n,
                          float* __restrict__ loss) {
  // one CTA, fixed-order reduction
  __shared__ float red[256];
  float s = 0.0f;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const float d = out[i] - Y[i];
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0] / (float)n;
}

struct DBuf {
  void* p = nullptr;
  size_t cap = 0;
  bool ensure(size_t bytes) {
    if (bytes <= cap) return true;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return false;
    cap = bytes;
    return true;
  }
  float* f() const { return static_cast<float*>(p); }
  ~DBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

struct mfgpu_mlp {
  int device = 0, nin = 0, h = 0;
  Layout L{1, 1};
  DBuf params, grad, m, v, X, Y, a1, a2, d1, d2, d3, out, loss;
  int64_t step = 0;
  std::string err;
  mfgpu_mlp(int nin_, int h_) : nin(nin_), h(h_), L(nin_, h_) {}
};

namespace {

int mlp_fail(mfgpu_mlp* m, const std::string& msg, int code = MFGPU_ERR_CUDA) {
  if (m) m->err = msg;
  return code;
}

#define MLP_CK(x)                                                          \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess) return mlp_fail(m, cudaGetErrorString(e_));     \
  } while (0)

int mlp_upload(mfgpu_mlp* m, const float* X, const float* Y, int64_t n) {
  if (!m->X.ensure(std::max<size_t>(n * m->nin, 1) * 4) || !m->a1.ensure(std::max<size_t>(n * m->h, 1) * 4) ||
      !m->a2.ensure(std::max<size_t>(n * m->h, 1) * 4) || !m->d1.ensure(std::max<size_t>(n * m->h, 1) * 4) ||
      !m->d2.ensure(std::max<size_t>(n * m->h, 1) * 4) || !m->d3.ensure(std::max<size_t>(n, 1) * 4) ||
      !m->out.ensure(std::max<size_t>(n, 1) * 4) || !m->loss.ensure(4))
    return mlp_fail(m, "device allocation failed", MFGPU_ERR_NOMEM);
  MLP_CK(cudaMemcpy(m->X.p, X, n * m->nin * 4, cudaMemcpyHostToDevice));
  if (Y) {
    if (!m->Y.ensure(std::max<size_t>(n, 1) * 4)) return mlp_fail(m, "device allocation failed", MFGPU_ERR_NOMEM);
    MLP_CK(cudaMemcpy(m->Y.p, Y, n * 4, cudaMemcpyHostToDevice));
  }
  return MFGPU_OK;
}

// forward + deltas + parameter gradients on the uploaded samples
int mlp_grad_pass(mfgpu_mlp* m, int64_t n) {
  const unsigned gs = (unsigned)((n + 127) / 128);
  k_mlp_forward<<<gs, 128>>>(m->params.f(), m->nin, m->h, m->X.f(), n, m->a1.f(), m->a2.f(), m->out.f());
  k_mlp_deltas<<<gs, 128>>>(m->params.f(), m->nin, m->h, m->Y.f(), n, m->a1.f(), m->a2.f(), m->out.f(), m->d1.f(),
                            m->d2.f(), m->d3.f());
  k_mlp_param_grads<<<(unsigned)((m->L.total + 127) / 128), 128>>>(m->nin, m->h, m->X.f(), n, m->a1.f(), m->a2.f(),
                                                                    m->d1.f(), m->d2.f(), m->d3.f(), m->grad.f());
  MLP_CK(cudaGetLastError());
  return MFGPU_OK;
}

}  // namespace

extern "C" {

int mfgpu_mlp_create(int32_t device, int32_t nin, int32_t hidden, uint64_t seed, mfgpu_mlp** out) {
  if (!out || nin < 1 || nin > kMaxIn || hidden < 1 || hidden > kMaxHidden) return MFGPU_ERR_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return MFGPU_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return MFGPU_ERR_CUDA;
  auto* m = new mfgpu_mlp(nin, hidden);
  m->device = device;
  const int P = m->L.total;
  if (!m->params.ensure(P * 4) || !m->grad.ensure(P * 4) || !m->m.ensure(P * 4) || !m->v.ensure(P * 4)) {
    delete m;
    return MFGPU_ERR_NOMEM;
  }
  // Glorot-uniform weights, zero biases
  std::vector<float> p(P, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int fan_in, int fan_out, int count) {
    const float a = std::sqrt(6.0f / (float)(fan_in + fan_out));
    std::uniform_real_distribution<float> u(-a, a);
    for (int i = 0; i < count; ++i) p[off + i] = u(rng);
  };
  fill(m->L.w1, nin, hidden, hidden * nin);
  fill(m->L.w2, hidden, hidden, hidden * hidden);
  fill(m->L.w3, hidden, 1, hidden);
  if (cudaMemcpy(m->params.p, p.data(), P * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(m->m.p, 0, P * 4) != cudaSuccess || cudaMemset(m->v.p, 0, P * 4) != cudaSuccess) {
    delete m;
    return MFGPU_ERR_CUDA;
  }
  *out = m;
  return MFGPU_OK;
}

void mfgpu_mlp_destroy(mfgpu_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  delete m;
}

const char* mfgpu_mlp_last_error(const mfgpu_mlp* m) { return m ? m->err.c_str() : "null model"; }

int32_t mfgpu_mlp_nparams(const mfgpu_mlp* m) { return m ? m->L.total : 0; }

int mfgpu_mlp_get_params(mfgpu_mlp* m, float* out) {
  if (!m || !out) return MFGPU_ERR_ARGUMENT;
  MLP_CK(cudaSetDevice(m->device));
  MLP_CK(cudaMemcpy(out, m->params.p, m->L.total * 4, cudaMemcpyDeviceToHost));
  return MFGPU_OK;
}

int mfgpu_mlp_set_params(mfgpu_mlp* m, const float* in) {
  if (!m || !in) return MFGPU_ERR_ARGUMENT;
  MLP_CK(cudaSetDevice(m->device));
  MLP_CK(cudaMemcpy(m->params.p, in, m->L.total * 4, cudaMemcpyHostToDevice));
  MLP_CK(cudaMemset(m->m.p, 0, m->L.total * 4));
  MLP_CK(cudaMemset(m->v.p, 0, m->L.total * 4));
  m->step = 0;
  return MFGPU_OK;
}

int mfgpu_mlp_predict(mfgpu_mlp* m, const float* X, int64_t n, float* out) {
  if (!m || (n > 0 && (!X || !out)) || n < 0) return MFGPU_ERR_ARGUMENT;
  if (n == 0) return MFGPU_OK;
  MLP_CK(cudaSetDevice(m->device));
  int rc = mlp_upload(m, X, nullptr, n);
  if (rc) return rc;
  k_mlp_forward<<<(unsigned)((n + 127) / 128), 128>>>(m->params.f(), m->nin, m->h, m->X.f(), n, m->a1.f(),
                                                       m->a2.f(), m->out.f());
  MLP_CK(cudaGetLastError());
  MLP_CK(cudaMemcpy(out, m->out.p, n * 4, cudaMemcpyDeviceToHost));
  return MFGPU_OK;
}

int mfgpu_mlp_loss_grad(mfgpu_mlp* m, const float* X, const float* Y, int64_t n, float* loss, float* grad) {
  if (!m || n < 1 || !X || !Y) return MFGPU_ERR_ARGUMENT;
  MLP_CK(cudaSetDevice(m->device));
  int rc = mlp_upload(m, X, Y, n);
  if (rc) return rc;
  rc = mlp_grad_pass(m, n);
  if (rc) return rc;
  k_sq_loss<<<1, 256>>>(m->out.f(), m->Y.f(), n, m->loss.f());
  MLP_CK(cudaGetLastError());
  if (loss) MLP_CK(cudaMemcpy(loss, m->loss.p, 4, cudaMemcpyDeviceToHost));
  if (grad) MLP_CK(cudaMemcpy(grad, m->grad.p, m->L.total * 4, cudaMemcpyDeviceToHost));
  return MFGPU_OK;
}

int mfgpu_mlp_train(mfgpu_mlp* m, const float* X, const float* Y, int64_t n, int32_t iters, float lr,
                    float* final_loss) {
  if (!m || n < 1 || !X || !Y || iters < 0 || !(lr > 0)) return MFGPU_ERR_ARGUMENT;
  MLP_CK(cudaSetDevice(m->device));
  int rc = mlp_upload(m, X, Y, n);
  if (rc) return rc;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const unsigned pg = (unsigned)((m->L.total + 127) / 128);
  for (int it = 0; it < iters; ++it) {
    rc = mlp_grad_pass(m, n);
    if (rc) return rc;
    ++m->step;
    const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
    k_adam<<<pg, 128>>>(m->params.f(), m->grad.f(), m->m.f(), m->v.f(), m->L.total, lr, b1, b2, eps, c1, c2);
  }
  k_mlp_forward<<<(unsigned)((n + 127) / 128), 128>>>(m->params.f(), m->nin, m->h, m->X.f(), n, m->a1.f(),
                                                       m->a2.f(), m->out.f());
  k_sq_loss<<<1, 256>>>(m->out.f(), m->Y.f(), n, m->loss.f());
  MLP_CK(cudaGetLastError());
  if (final_loss) MLP_CK(cudaMemcpy(final_loss, m->loss.p, 4, cudaMemcpyDeviceToHost));
  MLP_CK(cudaDeviceSynchronize());
  return MFGPU_OK;
}

}  // extern "C"
