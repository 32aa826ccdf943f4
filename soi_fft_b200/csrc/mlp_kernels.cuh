// mlp_kernels.cuh -- the learned-window surrogate: a 4-64-64-1 GELU MLP with
// hand-written forward, backward and Adam kernels (FP32).
//
// The network maps a window description (oversampling mu, taps B, tau, sigma;
// normalised on the host) to the predicted log10 relative L2 error of the SOI
// transform with that window.  It has no counterpart in the reference, whose
// windows come from the analytic family and the Pareto table of
// pfft.c:111-137.
//
// Parameter vector layout (kMlpParams floats):
//   W1[64][4] b1[64] W2[64][64] b2[64] W3[64] b3[1]
#pragma once

#include <cuda_runtime.h>

namespace soi {

constexpr int kMlpIn = 4, kMlpH = 64;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpH * kMlpIn, kOffW2 = kOffB1 + kMlpH,
              kOffB2 = kOffW2 + kMlpH * kMlpH, kOffW3 = kOffB2 + kMlpH, kOffB3 = kOffW3 + kMlpH,
              kMlpParams = kOffB3 + 1;
constexpr int kMlpBlock = 32;    // samples per block in the gradient kernel (one warp)

// GELU with the tanh approximation: 0.5 x (1 + tanh(c (x + 0.044715 x^3)))
__device__ __forceinline__ float gelu_f(float x, float *dgelu)
{
  const float c = 0.7978845608028654f;   // sqrt(2/pi)
  const float u = c * (x + 0.044715f * x * x * x);
  const float t = tanhf(u);
  if (dgelu) *dgelu = 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * c * (1.f + 3.f * 0.044715f * x * x);
  return 0.5f * x * (1.f + t);
}

__device__ __forceinline__ void mlp_forward_one(const float *p, const float *x, float *z1, float *h1,
                                                float *z2, float *h2, float &out)
{
  for (int j = 0; j < kMlpH; ++j) {
    float s = p[kOffB1 + j];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) s = fmaf(p[kOffW1 + j * kMlpIn + i], x[i], s);
    z1[j] = s;
    h1[j] = gelu_f(s, nullptr);
  }
  for (int j = 0; j < kMlpH; ++j) {
    float s = p[kOffB2 + j];
    for (int i = 0; i < kMlpH; ++i) s = fmaf(p[kOffW2 + j * kMlpH + i], h1[i], s);
    z2[j] = s;
    h2[j] = gelu_f(s, nullptr);
  }
  float o = p[kOffB3];
  for (int i = 0; i < kMlpH; ++i) o = fmaf(p[kOffW3 + i], h2[i], o);
  out = o;
}

// y[n] = MLP(x[n][4])
__global__ void mlp_forward_kernel(const float *params, const float *x, float *y, int n)
{
  __shared__ float p[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    float z1[kMlpH], h1[kMlpH], z2[kMlpH], h2[kMlpH], o;
    mlp_forward_one(p, x + (size_t)s * kMlpIn, z1, h1, z2, h2, o);
    y[s] = o;
  }
}

// Mean-squared-error gradient over n samples, accumulated into grad (zeroed
// by the caller) and loss (sum of squared errors / n).  One block handles
// kMlpBlock samples: forward and backward per thread, then the weight
// gradients are reduced over the block's samples through shared memory.
__global__ void __launch_bounds__(kMlpBlock) mlp_grad_kernel(const float *params, const float *x,
                                                             const float *y, int n, float *grad, float *loss)
{
  __shared__ float p[kMlpParams];
  __shared__ float s_h1[kMlpBlock][kMlpH + 1];   // h1, later reused
  __shared__ float s_d2[kMlpBlock][kMlpH + 1];   // delta2 = dL/dz2
  __shared__ float s_x[kMlpBlock][kMlpIn];
  __shared__ float s_d1[kMlpBlock][kMlpH + 1];   // delta1 = dL/dz1
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  const int s = blockIdx.x * kMlpBlock + threadIdx.x;
  const bool valid = s < n;
  const float inv_n = 1.f / (float)n;
  float d3 = 0.f;
  {
    float xin[kMlpIn] = { 0, 0, 0, 0 };
    if (valid)
      for (int i = 0; i < kMlpIn; ++i) xin[i] = x[(size_t)s * kMlpIn + i];
    for (int i = 0; i < kMlpIn; ++i) s_x[threadIdx.x][i] = xin[i];
    float z1[kMlpH], h1[kMlpH], z2[kMlpH], h2[kMlpH], o;
    mlp_forward_one(p, xin, z1, h1, z2, h2, o);
    if (valid) {
      const float e = o - y[s];
      d3 = 2.f * e * inv_n;
      atomicAdd(loss, e * e * inv_n);
    }
    for (int j = 0; j < kMlpH; ++j) {
      s_h1[threadIdx.x][j] = valid ? h1[j] : 0.f;
      float g2;
      gelu_f(z2[j], &g2);
      s_d2[threadIdx.x][j] = valid ? d3 * p[kOffW3 + j] * g2 : 0.f;
    }
    // delta1 = (W2^T delta2) * gelu'(z1)
    for (int i = 0; i < kMlpH; ++i) {
      float acc = 0.f;
      for (int j = 0; j < kMlpH; ++j) acc = fmaf(p[kOffW2 + j * kMlpH + i], s_d2[threadIdx.x][j], acc);
      float g1;
      gelu_f(z1[i], &g1);
      s_d1[threadIdx.x][i] = valid ? acc * g1 : 0.f;
    }
    // layer-3 gradients need h2: reuse s_d1's row? keep in registers below
    // dW3[j] = sum d3*h2[j], db3 = sum d3 (reduced with warp shuffles)
    for (int j = 0; j < kMlpH; ++j) {
      float v = valid ? d3 * h2[j] : 0.f;
      for (int o2 = 16; o2; o2 >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o2);
      if ((threadIdx.x & 31) == 0) atomicAdd(grad + kOffW3 + j, v);
    }
    float v = valid ? d3 : 0.f;
    for (int o2 = 16; o2; o2 >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o2);
    if ((threadIdx.x & 31) == 0) atomicAdd(grad + kOffB3, v);
  }
  __syncthreads();
  // dW2[j][i] = sum_s d2[s][j] h1[s][i]; db2[j] = sum_s d2[s][j]
  for (int e = threadIdx.x; e < kMlpH * kMlpH; e += blockDim.x) {
    const int j = e / kMlpH, i = e % kMlpH;
    float acc = 0.f;
    for (int q = 0; q < kMlpBlock; ++q) acc = fmaf(s_d2[q][j], s_h1[q][i], acc);
    atomicAdd(grad + kOffW2 + e, acc);
  }
  for (int j = threadIdx.x; j < kMlpH; j += blockDim.x) {
    float a2 = 0.f, a1 = 0.f;
    for (int q = 0; q < kMlpBlock; ++q) { a2 += s_d2[q][j]; a1 += s_d1[q][j]; }
    atomicAdd(grad + kOffB2 + j, a2);
    atomicAdd(grad + kOffB1 + j, a1);
  }
  // dW1[j][i] = sum_s d1[s][j] x[s][i]
  for (int e = threadIdx.x; e < kMlpH * kMlpIn; e += blockDim.x) {
    const int j = e / kMlpIn, i = e % kMlpIn;
    float acc = 0.f;
    for (int q = 0; q < kMlpBlock; ++q) acc = fmaf(s_d1[q][j], s_x[q][i], acc);
    atomicAdd(grad + kOffW1 + e, acc);
  }
}

// Adam (Kingma & Ba 2015) on the parameter vector.
__global__ void mlp_adam_kernel(float *params, float *m, float *v, const float *grad, int n, float lr, float beta1,
                                float beta2, float eps, int step)
{
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = grad[i];
    m[i] = beta1 * m[i] + (1.f - beta1) * g;
    v[i] = beta2 * v[i] + (1.f - beta2) * g * g;
    params[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
  }
}

// ---- the window proposer: an IN-64-64-OUT GELU MLP ------------------------
//
// Maps (oversampling mu, log10 of the target error; normalised on the host)
// to OUT = 32 Chebyshev coefficients of a window's frequency-response profile
// (soi_fft_b200/window_cheb.py).  Same GELU, layer width and Adam as the
// surrogate above; the loss is the mean squared error over samples and
// outputs.  Parameter layout: W1[64][IN] b1[64] W2[64][64] b2[64] W3[OUT][64]
// b3[OUT].  No counterpart in the reference.
namespace wmlp {

constexpr int H = 64;
template <int IN, int OUT> struct Dims {
  static constexpr int W1 = 0, B1 = W1 + H * IN, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H, B3 = W3 + OUT * H,
                       P = B3 + OUT;
};
constexpr int kIn = 2, kOut = 32;
constexpr int kParams = Dims<kIn, kOut>::P;
constexpr int kBlock = 32;           // samples per block of the gradient kernel (one warp)

template <int IN, int OUT>
__device__ __forceinline__ void forward_one(const float *__restrict__ p, const float *x, float *z1, float *h1,
                                            float *z2, float *h2, float *out)
{
  using G = Dims<IN, OUT>;
  for (int j = 0; j < H; ++j) {
    float s = __ldg(p + G::B1 + j);
#pragma unroll
    for (int i = 0; i < IN; ++i) s = fmaf(__ldg(p + G::W1 + j * IN + i), x[i], s);
    z1[j] = s;
    h1[j] = gelu_f(s, nullptr);
  }
  for (int j = 0; j < H; ++j) {
    float s = __ldg(p + G::B2 + j);
    for (int i = 0; i < H; ++i) s = fmaf(__ldg(p + G::W2 + j * H + i), h1[i], s);
    z2[j] = s;
    h2[j] = gelu_f(s, nullptr);
  }
  for (int o = 0; o < OUT; ++o) {
    float s = __ldg(p + G::B3 + o);
    for (int i = 0; i < H; ++i) s = fmaf(__ldg(p + G::W3 + o * H + i), h2[i], s);
    out[o] = s;
  }
}

// y[n][OUT] = MLP(x[n][IN])
template <int IN, int OUT>
__global__ void forward_kernel(const float *params, const float *x, float *y, int n)
{
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    float z1[H], h1[H], z2[H], h2[H], o[OUT];
    forward_one<IN, OUT>(params, x + (size_t)s * IN, z1, h1, z2, h2, o);
    for (int k = 0; k < OUT; ++k) y[(size_t)s * OUT + k] = o[k];
  }
}

// Gradient of mean((MLP(x) - y)^2) over n samples and OUT outputs,
// accumulated into grad and loss (both zeroed by the caller).  One block of
// kBlock samples: forward and backward per thread, weight gradients reduced
// over the block's samples through shared memory.
template <int IN, int OUT>
__global__ void __launch_bounds__(kBlock) grad_kernel(const float *params, const float *x, const float *y, int n,
                                                      float *grad, float *loss)
{
  using G = Dims<IN, OUT>;
  __shared__ float s_x[kBlock][IN];
  __shared__ float s_h1[kBlock][H + 1];
  __shared__ float s_h2[kBlock][H + 1];
  __shared__ float s_d1[kBlock][H + 1];
  __shared__ float s_d2[kBlock][H + 1];
  __shared__ float s_d3[kBlock][OUT + 1];
  const int t = threadIdx.x;
  const int s = blockIdx.x * kBlock + t;
  const bool valid = s < n;
  const float scale = 2.f / ((float)n * (float)OUT);
  {
    float xin[IN];
    for (int i = 0; i < IN; ++i) xin[i] = valid ? x[(size_t)s * IN + i] : 0.f;
    for (int i = 0; i < IN; ++i) s_x[t][i] = xin[i];
    float z1[H], h1[H], z2[H], h2[H], o[OUT];
    forward_one<IN, OUT>(params, xin, z1, h1, z2, h2, o);
    float l = 0.f;
    for (int k = 0; k < OUT; ++k) {
      const float e = valid ? o[k] - y[(size_t)s * OUT + k] : 0.f;
      l += e * e;
      s_d3[t][k] = e * scale;
    }
    if (valid) atomicAdd(loss, l / ((float)n * (float)OUT));
    for (int j = 0; j < H; ++j) {
      s_h1[t][j] = valid ? h1[j] : 0.f;
      s_h2[t][j] = valid ? h2[j] : 0.f;
    }
    // delta2 = (W3^T delta3) * gelu'(z2)
    for (int j = 0; j < H; ++j) {
      float acc = 0.f;
      for (int k = 0; k < OUT; ++k) acc = fmaf(__ldg(params + G::W3 + k * H + j), s_d3[t][k], acc);
      float g2;
      gelu_f(z2[j], &g2);
      s_d2[t][j] = valid ? acc * g2 : 0.f;
    }
    // delta1 = (W2^T delta2) * gelu'(z1)
    for (int i = 0; i < H; ++i) {
      float acc = 0.f;
      for (int j = 0; j < H; ++j) acc = fmaf(__ldg(params + G::W2 + j * H + i), s_d2[t][j], acc);
      float g1;
      gelu_f(z1[i], &g1);
      s_d1[t][i] = valid ? acc * g1 : 0.f;
    }
  }
  __syncwarp();
  // dW3[k][j] = sum_q d3[q][k] h2[q][j]; db3[k] = sum_q d3[q][k]
  for (int e = t; e < OUT * H; e += kBlock) {
    const int k = e / H, j = e % H;
    float acc = 0.f;
    for (int q = 0; q < kBlock; ++q) acc = fmaf(s_d3[q][k], s_h2[q][j], acc);
    atomicAdd(grad + G::W3 + e, acc);
  }
  for (int k = t; k < OUT; k += kBlock) {
    float acc = 0.f;
    for (int q = 0; q < kBlock; ++q) acc += s_d3[q][k];
    atomicAdd(grad + G::B3 + k, acc);
  }
  // dW2[j][i] = sum_q d2[q][j] h1[q][i]; db2, db1
  for (int e = t; e < H * H; e += kBlock) {
    const int j = e / H, i = e % H;
    float acc = 0.f;
    for (int q = 0; q < kBlock; ++q) acc = fmaf(s_d2[q][j], s_h1[q][i], acc);
    atomicAdd(grad + G::W2 + e, acc);
  }
  for (int j = t; j < H; j += kBlock) {
    float a2 = 0.f, a1 = 0.f;
    for (int q = 0; q < kBlock; ++q) { a2 += s_d2[q][j]; a1 += s_d1[q][j]; }
    atomicAdd(grad + G::B2 + j, a2);
    atomicAdd(grad + G::B1 + j, a1);
  }
  // dW1[j][i] = sum_q d1[q][j] x[q][i]
  for (int e = t; e < H * IN; e += kBlock) {
    const int j = e / IN, i = e % IN;
    float acc = 0.f;
    for (int q = 0; q < kBlock; ++q) acc = fmaf(s_d1[q][j], s_x[q][i], acc);
    atomicAdd(grad + G::W1 + e, acc);
  }
}

}  // namespace wmlp
}  // namespace soi
