// mlp.cu -- the learned configuration picker's network: a 3-layer MLP
// (kMlpIn -> 64 -> 64 -> kMlpOut, ReLU, FP32) with hand-written CUDA training kernels.
//
// It plays the role of Eigen's computeProductBlockingSizes
// (Eigen/src/Core/products/GeneralBlockPanelKernel.h:202-452), which maps (m, n, k) and
// the cache model to blocking sizes; here the inputs are shape and data features and
// the outputs are (a) scores of the kernel configurations and (b) scores of the digit
// slice counts of the emulated DGEMM.  Training data come from the exhaustive autotuner.
//
// Parameter layout (one flat float array, kMlpParams entries):
//   W1[64][kMlpIn] b1[64] W2[64][64] b2[64] W3[kMlpOut][64] b3[kMlpOut]
// Loss per sample: cross-entropy over the config logits [0, kMlpConfigs) plus, when the
// sample has a slice label (>= 0), cross-entropy over the slice logits.
#include <cuda_runtime.h>

#include "mlp.h"

namespace eb2 {

namespace {

constexpr int H = kMlpHidden;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + H * kMlpIn;
constexpr int kOffW2 = kOffB1 + H;
constexpr int kOffB2 = kOffW2 + H * H;
constexpr int kOffW3 = kOffB2 + H;
constexpr int kOffB3 = kOffW3 + kMlpOut * H;
static_assert(kOffB3 + kMlpOut == kMlpParams, "parameter layout");

constexpr int kSamplesPerBlock = 64;

// Forward of one sample; keeps the activations the backward pass needs.
__device__ void forward_one(const float* __restrict__ w, const float* x, float* h1, float* h2, float* out) {
  for (int j = 0; j < H; ++j) {
    float s = w[kOffB1 + j];
    for (int i = 0; i < kMlpIn; ++i) s = fmaf(w[kOffW1 + j * kMlpIn + i], x[i], s);
    h1[j] = s > 0.f ? s : 0.f;
  }
  for (int j = 0; j < H; ++j) {
    float s = w[kOffB2 + j];
    for (int i = 0; i < H; ++i) s = fmaf(w[kOffW2 + j * H + i], h1[i], s);
    h2[j] = s > 0.f ? s : 0.f;
  }
  for (int j = 0; j < kMlpOut; ++j) {
    float s = w[kOffB3 + j];
    for (int i = 0; i < H; ++i) s = fmaf(w[kOffW3 + j * H + i], h2[i], s);
    out[j] = s;
  }
}

__global__ void mlp_forward_kernel(const float* __restrict__ w, const float* __restrict__ X, int batch,
                                   float* __restrict__ logits) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= batch) return;
  float h1[H], h2[H], out[kMlpOut];
  forward_one(w, X + size_t(s) * kMlpIn, h1, h2, out);
  for (int j = 0; j < kMlpOut; ++j) logits[size_t(s) * kMlpOut + j] = out[j];
}

// softmax cross-entropy over logits[lo, hi) with target t; writes dL/dlogit into g
__device__ float xent(const float* logits, int lo, int hi, int t, float* g) {
  float mx = logits[lo];
  for (int j = lo + 1; j < hi; ++j) mx = fmaxf(mx, logits[j]);
  float z = 0.f;
  for (int j = lo; j < hi; ++j) z += __expf(logits[j] - mx);
  for (int j = lo; j < hi; ++j) g[j] = __expf(logits[j] - mx) / z - (j - lo == t ? 1.f : 0.f);
  return __logf(z) + mx - logits[lo + t];
}

// grads (kMlpParams) and loss (1 float) are accumulated (+=) with atomics; the mean over
// the batch is taken by the caller's scale factor `inv_batch`.
__global__ void __launch_bounds__(kSamplesPerBlock) mlp_backward_kernel(const float* __restrict__ w,
                                                                        const float* __restrict__ X,
                                                                        const int* __restrict__ cfg_label,
                                                                        const int* __restrict__ slice_label,
                                                                        int batch, float inv_batch,
                                                                        float* __restrict__ grads, float* loss) {
  __shared__ float sg[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) sg[i] = 0.f;
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < batch) {
    const float* x = X + size_t(s) * kMlpIn;
    float h1[H], h2[H], out[kMlpOut], g3[kMlpOut];
    forward_one(w, x, h1, h2, out);
    float l = xent(out, 0, kMlpConfigs, cfg_label[s], g3);
    const int sl = slice_label[s];
    if (sl >= 0) {
      l += xent(out, kMlpConfigs, kMlpOut, sl, g3);
    } else {
      for (int j = kMlpConfigs; j < kMlpOut; ++j) g3[j] = 0.f;
    }
    atomicAdd(loss, l * inv_batch);
    for (int j = 0; j < kMlpOut; ++j) g3[j] *= inv_batch;
    // layer 3
    float g2[H];
    for (int i = 0; i < H; ++i) g2[i] = 0.f;
    for (int j = 0; j < kMlpOut; ++j) {
      if (g3[j] == 0.f) continue;
      atomicAdd(&sg[kOffB3 + j], g3[j]);
      for (int i = 0; i < H; ++i) {
        atomicAdd(&sg[kOffW3 + j * H + i], g3[j] * h2[i]);
        g2[i] = fmaf(w[kOffW3 + j * H + i], g3[j], g2[i]);
      }
    }
    // layer 2 (ReLU mask)
    float g1[H];
    for (int i = 0; i < H; ++i) g1[i] = 0.f;
    for (int j = 0; j < H; ++j) {
      const float gj = h2[j] > 0.f ? g2[j] : 0.f;
      if (gj == 0.f) continue;
      atomicAdd(&sg[kOffB2 + j], gj);
      for (int i = 0; i < H; ++i) {
        atomicAdd(&sg[kOffW2 + j * H + i], gj * h1[i]);
        g1[i] = fmaf(w[kOffW2 + j * H + i], gj, g1[i]);
      }
    }
    // layer 1
    for (int j = 0; j < H; ++j) {
      const float gj = h1[j] > 0.f ? g1[j] : 0.f;
      if (gj == 0.f) continue;
      atomicAdd(&sg[kOffB1 + j], gj);
      for (int i = 0; i < kMlpIn; ++i) atomicAdd(&sg[kOffW1 + j * kMlpIn + i], gj * x[i]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x)
    if (sg[i] != 0.f) atomicAdd(&grads[i], sg[i]);
}

// Adam (Kingma & Ba 2015) with bias correction; step t >= 1.
__global__ void mlp_adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                                float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace

cudaError_t launch_mlp_forward(const float* w, const float* X, int batch, float* logits, cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  mlp_forward_kernel<<<(batch + 127) / 128, 128, 0, st>>>(w, X, batch, logits);
  return cudaGetLastError();
}

cudaError_t launch_mlp_backward(const float* w, const float* X, const int* cfg_label, const int* slice_label,
                                int batch, float* grads, float* loss, cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(grads, 0, sizeof(float) * kMlpParams, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(loss, 0, sizeof(float), st);
  if (e != cudaSuccess) return e;
  mlp_backward_kernel<<<(batch + kSamplesPerBlock - 1) / kSamplesPerBlock, kSamplesPerBlock, 0, st>>>(
      w, X, cfg_label, slice_label, batch, 1.f / float(batch), grads, loss);
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* w, const float* g, float* m, float* v, int step, float lr, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
  mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(w, g, m, v, kMlpParams, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

}  // namespace eb2
