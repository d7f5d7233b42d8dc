// Training and standalone inference kernels of the closure MLP
// (36 -> 32 -> 32 -> 1, ReLU, output clamped to [0, 1]; see av_closure.cuh).
//
// Training: minibatch Adam on float32 master weights.  Each step rounds the
// weights to bfloat16 for the forward pass (the precision the closure runs
// in), runs forward + backward with one thread per sample, reduces the
// per-sample gradients across each warp with shuffles, accumulates warp sums
// in shared memory and adds each block's sums to the global gradient once.
// Samples are drawn with replacement by a counter-based hash of
// (seed, step, lane), so a run is reproducible for a given seed.
//
// Loss: (clamp(z) - y)^2 with the gradient passed straight through the clamp
// when z lies on the wrong side of it (z < 0 < y or z > 1 > y); a clamped
// output on the target's side of the clamp has zero gradient.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "av_closure.cuh"
#include "selfgpu_internal.h"

using namespace selfgpu;

namespace {

constexpr int IN = kMlpIn, H = kMlpHidden;
constexpr int oW1 = 0, oB1 = oW1 + H * IN, oW2 = oB1 + H, oB2 = oW2 + H * H, oW3 = oB2 + H, oB3 = oW3 + H;
constexpr int NP = oB3 + 1;  // 2273 master parameters
static_assert(NP == SELFGPU_MLP_MASTER, "master parameter count");
static_assert(kMlpWeights == SELFGPU_MLP_WEIGHTS && kMlpFloats == SELFGPU_MLP_PARAMS, "closure weight layout");

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ bool is_weight(int k) {
  return (k >= oW1 && k < oB1) || (k >= oW2 && k < oB2) || (k >= oW3 && k < oB3);
}

__global__ void k_round_weights(const float* __restrict__ master, float* __restrict__ fw) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NP; k += gridDim.x * blockDim.x)
    fw[k] = is_weight(k) ? __bfloat162float(__float2bfloat16_rn(master[k])) : master[k];
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// accumulate one parameter's per-sample gradient: warp sum, then lane 0 adds to shared
__device__ __forceinline__ void acc_grad(float* sg, int k, float v, int lane) {
  v = warp_sum(v);
  if (lane == 0) atomicAdd(&sg[k], v);
}

__global__ void __launch_bounds__(256) k_grad(const float* __restrict__ feat, const float* __restrict__ label,
                                              int n, const float* __restrict__ fw, float* __restrict__ grad,
                                              float* __restrict__ loss, unsigned long long seed, long long step,
                                              int batch) {
  __shared__ float sw[NP], sg[NP];
  __shared__ float sloss;
  for (int k = threadIdx.x; k < NP; k += blockDim.x) {
    sw[k] = fw[k];
    sg[k] = 0.f;
  }
  if (threadIdx.x == 0) sloss = 0.f;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = b < batch;  // dead lanes contribute zero gradients (warp sums stay uniform)
  long long idx = 0;
  if (live) idx = (long long)(mix64(seed ^ mix64((unsigned long long)step * 0x100000001ull + (unsigned long long)b)) %
                              (unsigned long long)n);
  float f[IN], h1[H], h2[H];
#pragma unroll
  for (int k = 0; k < IN; ++k) f[k] = live ? feat[k + (long long)IN * idx] : 0.f;
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < IN; ++k) acc = fmaf(sw[oW1 + j * IN + k], f[k], acc);
    acc = acc + sw[oB1 + j];
    h1[j] = acc > 0.f ? acc : 0.f;
  }
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < H; ++k) acc = fmaf(sw[oW2 + j * H + k], h1[k], acc);
    acc = acc + sw[oB2 + j];
    h2[j] = acc > 0.f ? acc : 0.f;
  }
  float z = 0.f;
#pragma unroll
  for (int k = 0; k < H; ++k) z = fmaf(sw[oW3 + k], h2[k], z);
  z = z + sw[oB3];
  const float y = live ? label[idx] : 0.f;
  const float a = z < 0.f ? 0.f : (z > 1.f ? 1.f : z);
  float d = a - y;
  if ((z < 0.f && y > 0.f) || (z > 1.f && y < 1.f)) d = z - y;  // straight through the clamp
  if (!live) d = 0.f;
  const float l = live ? (a - y) * (a - y) : 0.f;
  const float ls = warp_sum(l);
  if (lane == 0) atomicAdd(&sloss, ls);
  const float g = 2.f * d / (float)batch;
  // output layer
  float dh2[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    acc_grad(sg, oW3 + j, g * h2[j], lane);
    dh2[j] = h2[j] > 0.f ? g * sw[oW3 + j] : 0.f;
  }
  acc_grad(sg, oB3, g, lane);
  // hidden layer 2
  float dh1[H];
#pragma unroll
  for (int k = 0; k < H; ++k) dh1[k] = 0.f;
#pragma unroll
  for (int j = 0; j < H; ++j) {
    acc_grad(sg, oB2 + j, dh2[j], lane);
#pragma unroll
    for (int k = 0; k < H; ++k) {
      acc_grad(sg, oW2 + j * H + k, dh2[j] * h1[k], lane);
      dh1[k] = fmaf(sw[oW2 + j * H + k], dh2[j], dh1[k]);
    }
  }
  // hidden layer 1
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const float dj = h1[j] > 0.f ? dh1[j] : 0.f;
    acc_grad(sg, oB1 + j, dj, lane);
#pragma unroll
    for (int k = 0; k < IN; ++k) acc_grad(sg, oW1 + j * IN + k, dj * f[k], lane);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < NP; k += blockDim.x) atomicAdd(&grad[k], sg[k]);
  if (threadIdx.x == 0) atomicAdd(loss, sloss);
}

__global__ void k_adam(float* __restrict__ master, float* __restrict__ grad, float* __restrict__ m1,
                       float* __restrict__ m2, float lr, float c1, float c2) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NP; k += gridDim.x * blockDim.x) {
    const float gk = grad[k];
    m1[k] = b1 * m1[k] + (1.f - b1) * gk;
    m2[k] = b2 * m2[k] + (1.f - b2) * gk * gk;
    const float mh = m1[k] / c1, vh = m2[k] / c2;
    master[k] -= lr * mh / (sqrtf(vh) + eps);
    grad[k] = 0.f;
  }
}

// One thread per sample; the arithmetic of the in-stage MLP (av_closure.cuh).
__global__ void __launch_bounds__(256) k_infer(const float* __restrict__ feat, int n,
                                               const __nv_bfloat16* __restrict__ w, const float* __restrict__ p,
                                               float* __restrict__ out) {
  __shared__ float sW1[H * IN], sW2[H * H], sw3[H], sB[kMlpFloats];
  for (int k = threadIdx.x; k < H * IN; k += blockDim.x) sW1[k] = __bfloat162float(w[k]);
  for (int k = threadIdx.x; k < H * H; k += blockDim.x) sW2[k] = __bfloat162float(w[H * IN + k]);
  for (int k = threadIdx.x; k < H; k += blockDim.x) sw3[k] = __bfloat162float(w[H * IN + H * H + k]);
  for (int k = threadIdx.x; k < kMlpFloats; k += blockDim.x) sB[k] = p[k];
  __syncthreads();
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) return;
  float f[IN], h1[H];
#pragma unroll
  for (int k = 0; k < IN; ++k) f[k] = feat[k + (long long)IN * s];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float acc = 0.f;
#pragma unroll 4
    for (int k = 0; k < IN; ++k) acc = fmaf(sW1[j * IN + k], f[k], acc);
    acc = acc + sB[j];
    h1[j] = acc > 0.f ? acc : 0.f;
  }
  float z = 0.f;
  for (int j = 0; j < H; ++j) {
    float acc = 0.f;
#pragma unroll 4
    for (int k = 0; k < H; ++k) acc = fmaf(sW2[j * H + k], h1[k], acc);
    acc = acc + sB[H + j];
    z = fmaf(sw3[j], acc > 0.f ? acc : 0.f, z);
  }
  z = z + sB[2 * H];
  out[s] = z < 0.f ? 0.f : (z > 1.f ? 1.f : z);
}

int fail(const char* where, cudaError_t e) {
  return set_error(SELFGPU_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int selfgpu_mlp_train(const float* features, const float* labels, int n, int epochs, int batch, float lr,
                      unsigned long long seed, float* params, float* lossPerEpoch, void* stream) {
  if (!features || !labels || n < 1 || epochs < 0 || batch < 1 || batch > (1 << 22) || !(lr > 0.f) || !params)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_mlp_train: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  float* buf = nullptr;  // master, forward, grad, m1, m2, loss
  cudaError_t e = cudaMalloc(&buf, (5 * NP + 1) * sizeof(float));
  if (e != cudaSuccess) return fail("selfgpu_mlp_train", e);
  float *master = buf, *fw = buf + NP, *grad = buf + 2 * NP, *m1 = buf + 3 * NP, *m2 = buf + 4 * NP,
        *loss = buf + 5 * NP;
  e = cudaMemsetAsync(buf, 0, (5 * NP + 1) * sizeof(float), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(master, params, NP * sizeof(float), cudaMemcpyHostToDevice, st);
  const long long stepsPerEpoch = ((long long)n + batch - 1) / batch;
  long long t = 0;
  float c1 = 1.f, c2 = 1.f;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    e = cudaMemsetAsync(loss, 0, sizeof(float), st);
    for (long long s = 0; s < stepsPerEpoch && e == cudaSuccess; ++s, ++t) {
      k_round_weights<<<(NP + 255) / 256, 256, 0, st>>>(master, fw);
      k_grad<<<(batch + 255) / 256, 256, 0, st>>>(features, labels, n, fw, grad, loss, seed, t, batch);
      c1 *= 0.9f;
      c2 *= 0.999f;
      k_adam<<<(NP + 255) / 256, 256, 0, st>>>(master, grad, m1, m2, lr, 1.f - c1, 1.f - c2);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && lossPerEpoch) {
      float h = 0.f;
      e = cudaMemcpyAsync(&h, loss, sizeof(float), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      lossPerEpoch[ep] = h / (float)(stepsPerEpoch * batch);
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(params, master, NP * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(buf);
  if (e != cudaSuccess) return fail("selfgpu_mlp_train", e);
  return SELFGPU_OK;
}

int selfgpu_mlp_infer(const float* features, int n, const uint16_t* weights, const float* params, float* out,
                      void* stream) {
  if (!features || n < 1 || !weights || !params || !out)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_mlp_infer: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  void* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, kMlpWeights * sizeof(uint16_t) + kMlpFloats * sizeof(float) + 16);
  if (e != cudaSuccess) return fail("selfgpu_mlp_infer", e);
  __nv_bfloat16* w = reinterpret_cast<__nv_bfloat16*>(buf);
  float* p = reinterpret_cast<float*>(reinterpret_cast<char*>(buf) + ((kMlpWeights * sizeof(uint16_t) + 15) / 16 * 16));
  e = cudaMemcpyAsync(w, weights, kMlpWeights * sizeof(uint16_t), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p, params, kMlpFloats * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_infer<<<(n + 255) / 256, 256, 0, st>>>(features, n, w, p, out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(buf);
  if (e != cudaSuccess) return fail("selfgpu_mlp_infer", e);
  return SELFGPU_OK;
}

}  // extern "C"
