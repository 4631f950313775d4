// The learned per-front precision selector's network: a one-hidden-layer
// MLP (D features -> H ReLU units -> one logit) trained with a weighted
// binary cross-entropy, with hand-written forward, backward and Adam
// kernels (FP32). Parameters, packed: W1 (H x D, row-major), b1 (H), w2
// (H), b2 (1). Gradients are summed per block, then the block partials in
// block order (deterministic).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include "../../include/smfg.h"

namespace {

constexpr int kMaxD = 32, kMaxH = 64, kThreads = 128;

__host__ __device__ inline int nparams(int d, int h) { return h * d + 2 * h + 1; }

__global__ void k_mlp_forward(const float *__restrict__ X, int n, int d, const float *__restrict__ P, int h,
                              float *__restrict__ out) {
  const float *W1 = P, *b1 = P + h * d, *w2 = b1 + h, *b2 = w2 + h;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float *x = X + (int64_t)s * d;
    float z2 = b2[0];
    for (int j = 0; j < h; ++j) {
      float z = b1[j];
      for (int c = 0; c < d; ++c) z = fmaf(W1[j * d + c], x[c], z);
      z2 = fmaf(w2[j], fmaxf(z, 0.0f), z2);
    }
    out[s] = 1.0f / (1.0f + expf(-z2));
  }
}

// Per-block partial gradients of sum_s w_s BCE(p_s, y_s) / n and the loss.
__global__ void __launch_bounds__(kThreads) k_mlp_backward(const float *__restrict__ X, const float *__restrict__ y,
                                                           const float *__restrict__ wt, int n, int d,
                                                           const float *__restrict__ P, int h,
                                                           float *__restrict__ part) {
  const int np = nparams(d, h);
  extern __shared__ float acc[];  // np + 1 (loss)
  for (int t = threadIdx.x; t <= np; t += blockDim.x) acc[t] = 0.0f;
  __syncthreads();
  const float *W1 = P, *b1 = P + h * d, *w2 = b1 + h, *b2 = w2 + h;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = s < n;
  const float *x = X + (int64_t)(valid ? s : 0) * d;
  float z1[kMaxH];
  float dz2 = 0.0f, loss = 0.0f;
  if (valid) {
    float z2 = b2[0];
    for (int j = 0; j < h; ++j) {
      float z = b1[j];
      for (int c = 0; c < d; ++c) z = fmaf(W1[j * d + c], x[c], z);
      z1[j] = z;
      z2 = fmaf(w2[j], fmaxf(z, 0.0f), z2);
    }
    const float p = 1.0f / (1.0f + expf(-z2));
    const float ws = wt ? wt[s] : 1.0f;
    const float yy = y[s];
    const float pc = fminf(fmaxf(p, 1e-7f), 1.0f - 1e-7f);
    loss = -ws * (yy * logf(pc) + (1.0f - yy) * logf(1.0f - pc)) / (float)n;
    dz2 = ws * (p - yy) / (float)n;
  }
  // the block's samples added in thread order (a fixed order: the gradient
  // does not depend on scheduling)
  for (int t = 0; t < (int)blockDim.x; ++t) {
    if ((int)threadIdx.x == t && valid) {
      for (int j = 0; j < h; ++j) {
        const float a = fmaxf(z1[j], 0.0f);
        const float dz1 = (z1[j] > 0.0f) ? dz2 * w2[j] : 0.0f;
        for (int c = 0; c < d; ++c) acc[j * d + c] += dz1 * x[c];
        acc[h * d + j] += dz1;
        acc[h * d + h + j] += dz2 * a;
      }
      acc[h * d + 2 * h] += dz2;
      acc[np] += loss;
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t <= np; t += blockDim.x) part[(int64_t)blockIdx.x * (np + 1) + t] = acc[t];
}

__global__ void k_mlp_reduce(const float *__restrict__ part, int nblocks, int np1, float *__restrict__ grad) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < np1; t += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int b = 0; b < nblocks; ++b) s += part[(int64_t)b * np1 + t];
    grad[t] = s;
  }
}

__global__ void k_adam(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ M,
                       float *__restrict__ V, int np, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x) {
    const float g = G[t];
    const float m = b1 * M[t] + (1.0f - b1) * g;
    const float v = b2 * V[t] + (1.0f - b2) * g * g;
    M[t] = m;
    V[t] = v;
    P[t] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
  }
}

}  // namespace

extern "C" {

SMFG_API int smfg_mlp_params(int d, int h) { return nparams(d, h); }

SMFG_API int smfg_mlp_forward(const float *d_X, int n, int d, const float *d_params, int h, float *d_out) {
  if (n < 0 || d < 1 || d > kMaxD || h < 1 || h > kMaxH || (n > 0 && (!d_X || !d_params || !d_out)))
    return SMFG_ERR_INVALID_ARG;
  if (n == 0) return SMFG_OK;
  const int g = std::max(1, std::min(1024, (n + kThreads - 1) / kThreads));
  k_mlp_forward<<<g, kThreads>>>(d_X, n, d, d_params, h, d_out);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return SMFG_ERR_CUDA;
  return SMFG_OK;
}

SMFG_API int smfg_mlp_backward(const float *d_X, const float *d_y, const float *d_w, int n, int d,
                               const float *d_params, int h, float *d_scratch, float *d_grad) {
  if (n < 1 || d < 1 || d > kMaxD || h < 1 || h > kMaxH || !d_X || !d_y || !d_params || !d_scratch || !d_grad)
    return SMFG_ERR_INVALID_ARG;
  const int np = nparams(d, h);
  const int nb = (n + kThreads - 1) / kThreads;
  k_mlp_backward<<<nb, kThreads, sizeof(float) * (np + 1)>>>(d_X, d_y, d_w, n, d, d_params, h, d_scratch);
  k_mlp_reduce<<<(np + 1 + 127) / 128, 128>>>(d_scratch, nb, np + 1, d_grad);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return SMFG_ERR_CUDA;
  return SMFG_OK;
}

SMFG_API int smfg_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, int np, float lr,
                           float beta1, float beta2, float eps, int step) {
  if (np < 1 || step < 1 || !d_params || !d_grad || !d_m || !d_v) return SMFG_ERR_INVALID_ARG;
  const float c1 = 1.0f - std::pow(beta1, (float)step), c2 = 1.0f - std::pow(beta2, (float)step);
  k_adam<<<(np + 255) / 256, 256>>>(d_params, d_grad, d_m, d_v, np, lr, beta1, beta2, eps, c1, c2);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return SMFG_ERR_CUDA;
  return SMFG_OK;
}

}  // extern "C"
