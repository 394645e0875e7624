// Learned closure, training side: the network's forward and backward passes
// and an Adam update, as the project's own kernels. Parameters are FP32
// (master copy); the inference layout (MlpNet) rounds the weights to BF16.
//
// Parameter vector (MLP_P floats): W1[64][9], b1[64], W2[64][64], b2[64],
// w3[64], b3. The model is
//   x' = (x - shift) * scale,  h1 = relu(W1 x' + b1),  h2 = relu(W2 h1 + b2),
//   y = w3 . h2 + b3,  Cs^2 = out_scale * softplus(y),
// and the loss the mean squared error of Cs^2 against the targets.
//
// k_mlp_grad: a fixed grid of blocks; each block takes chunks of 128 samples
// (one per thread), keeps the chunk's activations in shared memory, and turns
// the backward pass into block-wide outer products, accumulating the
// gradient in shared memory. Each block writes one row of partial sums;
// k_mlp_reduce adds the rows in a fixed order, so gradients are deterministic.
#include <cuda_bf16.h>
#include <cstring>
#include <string>
#include <vector>
#include "aslb.h"
#include "kernels.h"
#include "mlp.cuh"

namespace aslb {

constexpr int kIn = kMlpIn, kH = kMlpHidden;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH;
constexpr int kParams = oB3 + 1;
constexpr int kChunk = 128;
constexpr int kPad = kH + 1;  // row stride of the activation tiles (no bank conflicts)

__device__ __forceinline__ float softplus_f(float y) { return y > 20.f ? y : log1pf(expf(y)); }
__device__ __forceinline__ float sigmoid_f(float y) { return 1.f / (1.f + expf(-y)); }

__global__ void __launch_bounds__(kChunk)
    k_mlp_grad(const float* __restrict__ params, const float* __restrict__ X, const float* __restrict__ T,
               long long n, const float* __restrict__ norm, float out_scale, float inv_count,
               float* __restrict__ partials) {
  extern __shared__ float sm[];
  float* W = sm;                  // kParams
  float* G = W + kParams;         // kParams (gradient accumulator; last slot: loss)
  float* H1 = G + kParams + 1;    // kChunk x kPad
  float* H2 = H1 + kChunk * kPad; // kChunk x kPad
  float* XS = H2 + kChunk * kPad; // kChunk x kIn
  float* DY = XS + kChunk * kIn;  // kChunk
  const int t = threadIdx.x;
  for (int i = t; i < kParams; i += kChunk) {
    W[i] = params[i];
    G[i] = 0.f;
  }
  if (t == 0) G[kParams] = 0.f;
  __syncthreads();
  const long long nchunks = (n + kChunk - 1) / kChunk;
  for (long long c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const long long i = c * kChunk + t;
    const bool valid = i < n;
    // forward
    float x[kIn];
#pragma unroll
    for (int j = 0; j < kIn; ++j) {
      x[j] = valid ? (X[(long long)j * n + i] - norm[j]) * norm[kIn + j] : 0.f;
      XS[t * kIn + j] = x[j];
    }
    for (int k = 0; k < kH; ++k) {
      float a = W[oB1 + k];
#pragma unroll
      for (int j = 0; j < kIn; ++j) a = fmaf(W[oW1 + k * kIn + j], x[j], a);
      H1[t * kPad + k] = fmaxf(a, 0.f);
    }
    float y = W[oB3];
    for (int k = 0; k < kH; ++k) {
      float a = W[oB2 + k];
      for (int j = 0; j < kH; ++j) a = fmaf(W[oW2 + k * kH + j], H1[t * kPad + j], a);
      a = fmaxf(a, 0.f);
      H2[t * kPad + k] = a;
      y = fmaf(W[oW3 + k], a, y);
    }
    float dy = 0.f;
    if (valid) {
      const float e = out_scale * softplus_f(y) - T[i];
      dy = 2.f * e * out_scale * sigmoid_f(y) * inv_count;
      DY[t] = dy;
      H1[t * kPad + kH] = e * e;  // the padding column carries the squared error
    } else {
      DY[t] = 0.f;
      H1[t * kPad + kH] = 0.f;
    }
    __syncthreads();
    // output layer: gw3[k] = sum_s dy_s h2[s][k]; gb3 = sum_s dy_s; loss
    if (t < kH) {
      float a = 0.f;
      for (int s = 0; s < kChunk; ++s) a = fmaf(DY[s], H2[s * kPad + t], a);
      G[oW3 + t] += a;
    } else if (t == kH) {
      float a = 0.f, l = 0.f;
      for (int s = 0; s < kChunk; ++s) {
        a += DY[s];
        l += H1[s * kPad + kH];
      }
      G[oB3] += a;
      G[kParams] += l;
    }
    __syncthreads();
    // dh2 = dy w3 [h2 > 0], in place
    for (int k = 0; k < kH; ++k) {
      const float h = H2[t * kPad + k];
      H2[t * kPad + k] = h > 0.f ? dy * W[oW3 + k] : 0.f;
    }
    __syncthreads();
    // gW2[m][j] = sum_s dh2[s][m] h1[s][j]; gb2[m] = sum_s dh2[s][m]
    {
      const int m = t >> 1, j0 = (t & 1) * (kH / 2);
      float acc[kH / 2];
#pragma unroll
      for (int q = 0; q < kH / 2; ++q) acc[q] = 0.f;
      float bsum = 0.f;
      for (int s = 0; s < kChunk; ++s) {
        const float d = H2[s * kPad + m];
        bsum += d;
#pragma unroll
        for (int q = 0; q < kH / 2; ++q) acc[q] = fmaf(d, H1[s * kPad + j0 + q], acc[q]);
      }
#pragma unroll
      for (int q = 0; q < kH / 2; ++q) G[oW2 + m * kH + j0 + q] += acc[q];
      if ((t & 1) == 0) G[oB2 + m] += bsum;
    }
    __syncthreads();
    // dh1[s][j] = [h1 > 0] sum_m dh2[s][m] W2[m][j], in place (own row)
    {
      float d1[kH];
#pragma unroll
      for (int j = 0; j < kH; ++j) d1[j] = 0.f;
      for (int m = 0; m < kH; ++m) {
        const float d = H2[t * kPad + m];
#pragma unroll
        for (int j = 0; j < kH; ++j) d1[j] = fmaf(d, W[oW2 + m * kH + j], d1[j]);
      }
#pragma unroll
      for (int j = 0; j < kH; ++j) H1[t * kPad + j] = H1[t * kPad + j] > 0.f ? d1[j] : 0.f;
    }
    __syncthreads();
    // gW1[m][j] = sum_s dh1[s][m] x[s][j]; gb1[m] = sum_s dh1[s][m]
    for (int e = t; e < kH * (kIn + 1); e += kChunk) {
      const int m = e / (kIn + 1), j = e % (kIn + 1);
      float a = 0.f;
      if (j < kIn) {
        for (int s = 0; s < kChunk; ++s) a = fmaf(H1[s * kPad + m], XS[s * kIn + j], a);
        G[oW1 + m * kIn + j] += a;
      } else {
        for (int s = 0; s < kChunk; ++s) a += H1[s * kPad + m];
        G[oB1 + m] += a;
      }
    }
    __syncthreads();
  }
  for (int i = t; i <= kParams; i += kChunk) partials[(long long)blockIdx.x * (kParams + 1) + i] = G[i];
}

__global__ void k_mlp_reduce(const float* __restrict__ partials, int rows, float* __restrict__ grad_loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kParams) return;
  float a = 0.f;
  for (int r = 0; r < rows; ++r) a += partials[(long long)r * (kParams + 1) + i];
  grad_loss[i] = a;
}

__global__ void k_mlp_adam(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace aslb

using namespace aslb;

namespace {
constexpr int kGradBlocks = 148;
size_t grad_smem() { return (size_t)(2 * kParams + 1 + 2 * kChunk * kPad + kChunk * kIn + kChunk) * sizeof(float); }
int err(const char* what, cudaError_t e) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return ASLB_ERR_CUDA;
}
int arg_err(const char* what) {
  set_last_error(std::string(what) + ": bad arguments");
  return ASLB_ERR_ARG;
}
}  // namespace

extern "C" {

int aslb_mlp_param_count(void) { return kParams; }

size_t aslb_mlp_grad_scratch_floats(void) { return (size_t)kGradBlocks * (kParams + 1); }

int aslb_mlp_grad(const float* params, const float* x, const float* t, long long n, const float* norm,
                  float out_scale, float* scratch, float* grad_loss, void* stream) {
  if (!params || !x || !t || !norm || !scratch || !grad_loss || n <= 0) return arg_err("aslb_mlp_grad");
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem());
    if (e != cudaSuccess) return err("aslb_mlp_grad", e);
    configured = true;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long long chunks = (n + kChunk - 1) / kChunk;
  const int blocks = (int)(chunks < kGradBlocks ? chunks : kGradBlocks);
  k_mlp_grad<<<blocks, kChunk, grad_smem(), st>>>(params, x, t, n, norm, out_scale, 1.f / (float)n, scratch);
  k_mlp_reduce<<<(kParams + 1 + 255) / 256, 256, 0, st>>>(scratch, blocks, grad_loss);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ASLB_OK : err("aslb_mlp_grad", e);
}

int aslb_mlp_adam(float* params, const float* grad, float* m, float* v, int step, float lr, float beta1,
                  float beta2, float eps, void* stream) {
  if (!params || !grad || !m || !v || step < 1) return arg_err("aslb_mlp_adam");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_mlp_adam<<<(kParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, lr, beta1, beta2, eps,
                                                                       c1, c2);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ASLB_OK : err("aslb_mlp_adam", e);
}

int aslb_mlp_pack(const float* params_host, const float* norm_host, float out_scale, void* net_host) {
  if (!params_host || !norm_host || !net_host) return arg_err("aslb_mlp_pack");
  MlpNet net;
  std::memset(&net, 0, sizeof(net));
  for (int j = 0; j < kMlpInPad; ++j) {
    net.in_shift[j] = j < kIn ? norm_host[j] : 0.f;
    net.in_scale[j] = j < kIn ? norm_host[kIn + j] : 0.f;
  }
  for (int k = 0; k < kH; ++k) {
    for (int j = 0; j < kMlpInPad; ++j)
      net.w1[k][j] = __float2bfloat16_rn(j < kIn ? params_host[oW1 + k * kIn + j] : 0.f);
    net.b1[k] = params_host[oB1 + k];
    for (int j = 0; j < kH; ++j) net.w2[k][j] = __float2bfloat16_rn(params_host[oW2 + k * kH + j]);
    net.b2[k] = params_host[oB2 + k];
    net.w3[k] = __float2bfloat16_rn(params_host[oW3 + k]);
  }
  net.b3 = params_host[oB3];
  net.out_scale = out_scale;
  std::memcpy(net_host, &net, sizeof(net));
  return ASLB_OK;
}

}  // extern "C"
