// The planner network: a 3-layer perceptron  inputs -> 64 -> 64 -> 2  (ReLU
// between layers) that predicts the next layer's log growth and duplicate
// ratio of a BFS from its recent layer sizes and generator features.  It is
// trained and evaluated only by the kernels in this file.
//
// Parameters are one flat fp32 buffer:
//     W1[64][in] | b1[64] | W2[64][64] | b2[64] | W3[2][64] | b3[2]
// Training: mlp_loss_grad (forward + backward of a weighted squared error,
// per-block gradient reduction in shared memory, one global atomicAdd per
// parameter per block) and mlp_adam.  Inference: mlp_infer_bf16 reads bf16
// parameters and keeps activations in bf16, accumulating in fp32.
// No reference counterpart: the reference sizes its buffers by worst-case
// bounds and timed pilot runs (crates/mgbfs-runtime/src/generic_memory.rs:36-49,
// multigpubfs/autotune.py:276).
#include <cuda_bf16.h>

#include <algorithm>

#include "../../include/mgbfs2.h"
#include "engine.h"

namespace mgbfs2 {
namespace {

constexpr uint32_t kHidden = 64, kOut = 2, kMaxIn = 32, kMlpBlock = 128;

struct Offsets {
  uint32_t w1, b1, w2, b2, w3, b3, total;
};

__host__ __device__ __forceinline__ Offsets offsets(uint32_t in) {
  Offsets o;
  o.w1 = 0;
  o.b1 = o.w1 + kHidden * in;
  o.w2 = o.b1 + kHidden;
  o.b2 = o.w2 + kHidden * kHidden;
  o.w3 = o.b2 + kHidden;
  o.b3 = o.w3 + kOut * kHidden;
  o.total = o.b3 + kOut;
  return o;
}

// h1 = relu(W1 x + b1); returns y = W3 relu(W2 h1 + b2) + b3, keeping h1/h2.
__device__ __forceinline__ void forward_one(const float* P, const Offsets& o, uint32_t in, const float* x, float* h1,
                                            float* h2, float* y) {
  for (uint32_t k = 0; k < kHidden; ++k) {
    float a = P[o.b1 + k];
    for (uint32_t i = 0; i < in; ++i) a = fmaf(P[o.w1 + k * in + i], x[i], a);
    h1[k] = fmaxf(a, 0.f);
  }
  y[0] = P[o.b3];
  y[1] = P[o.b3 + 1];
  for (uint32_t j = 0; j < kHidden; ++j) {
    float a = P[o.b2 + j];
    for (uint32_t k = 0; k < kHidden; ++k) a = fmaf(P[o.w2 + j * kHidden + k], h1[k], a);
    a = fmaxf(a, 0.f);
    h2[j] = a;
    y[0] = fmaf(P[o.w3 + j], a, y[0]);
    y[1] = fmaf(P[o.w3 + kHidden + j], a, y[1]);
  }
}

__global__ void __launch_bounds__(kMlpBlock) mlp_forward_kernel(uint32_t in, const float* params, const float* x,
                                                                unsigned long long batch, float* y) {
  extern __shared__ float P[];
  const Offsets o = offsets(in);
  for (uint32_t i = threadIdx.x; i < o.total; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  for (unsigned long long s = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; s < batch;
       s += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    float xs[kMaxIn], h1[kHidden], h2[kHidden], out[kOut];
    for (uint32_t i = 0; i < in; ++i) xs[i] = x[s * in + i];
    forward_one(P, o, in, xs, h1, h2, out);
    y[s * kOut] = out[0];
    y[s * kOut + 1] = out[1];
  }
}

// loss = sum_s sum_o w_o (y_so - t_so)^2 / batch; grad += d loss / d params.
__global__ void __launch_bounds__(kMlpBlock) mlp_loss_grad_kernel(uint32_t in, const float* params, const float* x,
                                                                  const float* target, float w0, float w1,
                                                                  unsigned long long batch, float* grad,
                                                                  float* loss) {
  extern __shared__ float smem[];
  const Offsets o = offsets(in);
  float* P = smem;
  float* G = smem + o.total;
  for (uint32_t i = threadIdx.x; i < o.total; i += blockDim.x) {
    P[i] = params[i];
    G[i] = 0.f;
  }
  __syncthreads();
  const float scale = 2.f / static_cast<float>(batch);
  float local_loss = 0.f;
  for (unsigned long long s = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; s < batch;
       s += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    float xs[kMaxIn], h1[kHidden], h2[kHidden], y[kOut], dh1[kHidden];
    for (uint32_t i = 0; i < in; ++i) xs[i] = x[s * in + i];
    forward_one(P, o, in, xs, h1, h2, y);
    const float e0 = y[0] - target[s * kOut], e1 = y[1] - target[s * kOut + 1];
    local_loss += (w0 * e0 * e0 + w1 * e1 * e1) / static_cast<float>(batch);
    const float dy0 = scale * w0 * e0, dy1 = scale * w1 * e1;
    atomicAdd(&G[o.b3], dy0);
    atomicAdd(&G[o.b3 + 1], dy1);
    for (uint32_t k = 0; k < kHidden; ++k) dh1[k] = 0.f;
    for (uint32_t j = 0; j < kHidden; ++j) {
      atomicAdd(&G[o.w3 + j], dy0 * h2[j]);
      atomicAdd(&G[o.w3 + kHidden + j], dy1 * h2[j]);
      const float dh2 = h2[j] > 0.f ? fmaf(P[o.w3 + j], dy0, P[o.w3 + kHidden + j] * dy1) : 0.f;
      if (dh2 == 0.f) continue;
      atomicAdd(&G[o.b2 + j], dh2);
      for (uint32_t k = 0; k < kHidden; ++k) {
        if (h1[k] > 0.f) atomicAdd(&G[o.w2 + j * kHidden + k], dh2 * h1[k]);
        dh1[k] = fmaf(P[o.w2 + j * kHidden + k], dh2, dh1[k]);
      }
    }
    for (uint32_t k = 0; k < kHidden; ++k) {
      if (h1[k] <= 0.f || dh1[k] == 0.f) continue;
      atomicAdd(&G[o.b1 + k], dh1[k]);
      for (uint32_t i = 0; i < in; ++i) atomicAdd(&G[o.w1 + k * in + i], dh1[k] * xs[i]);
    }
  }
  // Block reduction of the loss, then one global add per parameter.
  for (int off = 16; off > 0; off >>= 1) local_loss += __shfl_xor_sync(kFullMask, local_loss, off);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, local_loss);
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < o.total; i += blockDim.x)
    if (G[i] != 0.f) atomicAdd(&grad[i], G[i]);
}

__global__ void mlp_adam_kernel(uint32_t count, float* params, const float* grad, float* m, float* v, float lr,
                                float beta1, float beta2, float eps, float c1, float c2) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const float g = grad[i];
    m[i] = beta1 * m[i] + (1.f - beta1) * g;
    v[i] = beta2 * v[i] + (1.f - beta2) * g * g;
    params[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
  }
}

__global__ void mlp_to_bf16_kernel(uint32_t count, const float* params, __nv_bfloat16* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(params[i]);
}

// bf16 parameters and activations, fp32 accumulation; two hidden units per
// step through bf16x2 pairs.
__global__ void __launch_bounds__(kMlpBlock) mlp_infer_bf16_kernel(uint32_t in, const __nv_bfloat16* params,
                                                                   const float* x, unsigned long long batch,
                                                                   float* y) {
  extern __shared__ __nv_bfloat16 Q[];
  const Offsets o = offsets(in);
  for (uint32_t i = threadIdx.x; i < o.total; i += blockDim.x) Q[i] = params[i];
  __syncthreads();
  for (unsigned long long s = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; s < batch;
       s += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    __nv_bfloat16 xs[kMaxIn], h1[kHidden];
    for (uint32_t i = 0; i < in; ++i) xs[i] = __float2bfloat16(x[s * in + i]);
    for (uint32_t k = 0; k < kHidden; ++k) {
      float a = __bfloat162float(Q[o.b1 + k]);
      for (uint32_t i = 0; i < in; ++i) a = fmaf(__bfloat162float(Q[o.w1 + k * in + i]), __bfloat162float(xs[i]), a);
      h1[k] = __float2bfloat16(fmaxf(a, 0.f));
    }
    float y0 = __bfloat162float(Q[o.b3]), y1 = __bfloat162float(Q[o.b3 + 1]);
    for (uint32_t j = 0; j < kHidden; ++j) {
      float a = __bfloat162float(Q[o.b2 + j]);
      const __nv_bfloat162* row = reinterpret_cast<const __nv_bfloat162*>(Q + o.w2 + j * kHidden);
      for (uint32_t k = 0; k < kHidden; k += 2) {
        const float2 w = __bfloat1622float2(row[k / 2]);
        a = fmaf(w.x, __bfloat162float(h1[k]), a);
        a = fmaf(w.y, __bfloat162float(h1[k + 1]), a);
      }
      const float h2 = __bfloat162float(__float2bfloat16(fmaxf(a, 0.f)));
      y0 = fmaf(__bfloat162float(Q[o.w3 + j]), h2, y0);
      y1 = fmaf(__bfloat162float(Q[o.w3 + kHidden + j]), h2, y1);
    }
    y[s * kOut] = y0;
    y[s * kOut + 1] = y1;
  }
}

// Whole-profile rollout on the device, one thread per instance: the 16
// planner features of depth d are formed from the last four predicted layers
// (bookkeeping in fp64), run through the same bf16 network as
// mlp_infer_bf16_kernel (bf16 inputs and hidden activations, fp32
// accumulation), and the predicted next layer
//     |L_{d+1}| = min(expm1(y0 + log1p |L_d|), orbit - visited, g |L_d|)
// is appended until it drops below one half.  statics[8 m + k] holds
// log orbit, n/16, g/8, inverse-closed, mean and max log generator order,
// fixed-point fraction and cycle fraction; gens[m] the generator counts.
constexpr uint32_t kRolloutInputs = 16;

__global__ void __launch_bounds__(kMlpBlock) mlp_rollout_kernel(const __nv_bfloat16* params, const float* x_mean,
                                                                const float* x_scale, const float* statics,
                                                                const float* gens, uint32_t count, uint32_t max_depth,
                                                                double* peak, double* total, uint32_t* depth) {
  extern __shared__ __nv_bfloat16 Q[];
  const Offsets o = offsets(kRolloutInputs);
  for (uint32_t i = threadIdx.x; i < o.total; i += blockDim.x) Q[i] = params[i];
  __syncthreads();
  const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= count) return;
  const float* st = statics + 8ull * m;
  const double g = gens[m], log_orbit = st[0], orbit = exp(log_orbit);
  double last[4] = {1.0, 0.0, 0.0, 0.0}, visited = 1.0, best = 1.0, sum = 1.0;
  uint32_t d = 0;
  for (; d < max_depth; ++d) {
    float x[kRolloutInputs];
    for (int k = 0; k < 4; ++k) x[k] = static_cast<float>(log1p(last[k]));
    x[4] = static_cast<float>(log1p(visited));
    for (int k = 0; k < 8; ++k) x[5 + k] = st[k];
    x[13] = static_cast<float>(d) / 64.0f;
    x[14] = static_cast<float>(visited / orbit);
    x[15] = static_cast<float>(log1p(g * last[0]));
    __nv_bfloat16 xs[kRolloutInputs], h1[kHidden];
    for (uint32_t i = 0; i < kRolloutInputs; ++i) xs[i] = __float2bfloat16((x[i] - x_mean[i]) / x_scale[i]);
    for (uint32_t k = 0; k < kHidden; ++k) {
      float a = __bfloat162float(Q[o.b1 + k]);
      for (uint32_t i = 0; i < kRolloutInputs; ++i)
        a = fmaf(__bfloat162float(Q[o.w1 + k * kRolloutInputs + i]), __bfloat162float(xs[i]), a);
      h1[k] = __float2bfloat16(fmaxf(a, 0.f));
    }
    float y0 = __bfloat162float(Q[o.b3]);
    for (uint32_t j = 0; j < kHidden; ++j) {
      float a = __bfloat162float(Q[o.b2 + j]);
      const __nv_bfloat162* row = reinterpret_cast<const __nv_bfloat162*>(Q + o.w2 + j * kHidden);
      for (uint32_t k = 0; k < kHidden; k += 2) {
        const float2 w = __bfloat1622float2(row[k / 2]);
        a = fmaf(w.x, __bfloat162float(h1[k]), a);
        a = fmaf(w.y, __bfloat162float(h1[k + 1]), a);
      }
      y0 = fmaf(__bfloat162float(Q[o.w3 + j]), __bfloat162float(__float2bfloat16(fmaxf(a, 0.f))), y0);
    }
    double nxt = expm1(static_cast<double>(y0) + log1p(last[0]));
    nxt = fmin(nxt, fmin(orbit - visited, g * last[0]));
    if (!(nxt >= 0.5)) break;
    last[3] = last[2];
    last[2] = last[1];
    last[1] = last[0];
    last[0] = nxt;
    visited += nxt;
    sum += nxt;
    best = fmax(best, nxt);
  }
  peak[m] = best;
  total[m] = sum;
  depth[m] = d + 1;
}

uint32_t mlp_grid(unsigned long long batch) {
  return static_cast<uint32_t>(std::max<unsigned long long>(1, std::min<unsigned long long>((batch + kMlpBlock - 1) / kMlpBlock, 148ull * 4)));
}

}  // namespace
}  // namespace mgbfs2

using namespace mgbfs2;

extern "C" {

uint32_t mgbfs2_mlp_param_count(uint32_t inputs) { return offsets(inputs).total; }

int mgbfs2_mlp_forward(uint32_t inputs, const float* params, const float* x, uint64_t batch, float* y, void* stream) {
  if (!inputs || inputs > kMaxIn || !params || (batch && (!x || !y))) return MGBFS2_INVALID_ARGUMENT;
  if (!batch) return MGBFS2_OK;
  const size_t smem = offsets(inputs).total * sizeof(float);
  mlp_forward_kernel<<<mlp_grid(batch), kMlpBlock, smem, static_cast<cudaStream_t>(stream)>>>(inputs, params, x, batch,
                                                                                               y);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_mlp_loss_grad(uint32_t inputs, const float* params, const float* x, const float* target, float weight0,
                         float weight1, uint64_t batch, float* grad, float* loss, void* stream) {
  if (!inputs || inputs > kMaxIn || !params || !grad || (batch && (!x || !target))) return MGBFS2_INVALID_ARGUMENT;
  if (!batch) return MGBFS2_OK;
  mgbfs2::TraceRange range("planner.loss_grad");
  const size_t smem = 2 * offsets(inputs).total * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(mlp_loss_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return cuda_status(e);
  mlp_loss_grad_kernel<<<mlp_grid(batch), kMlpBlock, smem, static_cast<cudaStream_t>(stream)>>>(
      inputs, params, x, target, weight0, weight1, batch, grad, loss);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_mlp_adam(uint32_t count, float* params, const float* grad, float* m, float* v, float lr, float beta1,
                    float beta2, float eps, uint32_t step, void* stream) {
  if (!count || !params || !grad || !m || !v || !step) return MGBFS2_INVALID_ARGUMENT;
  const float c1 = 1.f - powf(beta1, static_cast<float>(step)), c2 = 1.f - powf(beta2, static_cast<float>(step));
  mlp_adam_kernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(count, params, grad, m, v, lr,
                                                                                       beta1, beta2, eps, c1, c2);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_mlp_to_bf16(uint32_t count, const float* params, void* params_bf16, void* stream) {
  if (!count || !params || !params_bf16) return MGBFS2_INVALID_ARGUMENT;
  mlp_to_bf16_kernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      count, params, static_cast<__nv_bfloat16*>(params_bf16));
  return cuda_status(cudaGetLastError());
}

int mgbfs2_mlp_infer_bf16(uint32_t inputs, const void* params_bf16, const float* x, uint64_t batch, float* y,
                          void* stream) {
  if (!inputs || inputs > kMaxIn || !params_bf16 || (batch && (!x || !y))) return MGBFS2_INVALID_ARGUMENT;
  if (!batch) return MGBFS2_OK;
  const size_t smem = offsets(inputs).total * sizeof(__nv_bfloat16);
  mlp_infer_bf16_kernel<<<mlp_grid(batch), kMlpBlock, smem, static_cast<cudaStream_t>(stream)>>>(
      inputs, static_cast<const __nv_bfloat16*>(params_bf16), x, batch, y);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_mlp_rollout_bf16(const void* params_bf16, const float* x_mean, const float* x_scale, const float* statics,
                            const float* gens, uint32_t count, uint32_t max_depth, double* peak, double* total,
                            uint32_t* depth, void* stream) {
  mgbfs2::TraceRange range("planner.rollout");
  if (!params_bf16 || !x_mean || !x_scale || (count && (!statics || !gens || !peak || !total || !depth)))
    return MGBFS2_INVALID_ARGUMENT;
  if (!count) return MGBFS2_OK;
  const size_t smem = offsets(kRolloutInputs).total * sizeof(__nv_bfloat16);
  mlp_rollout_kernel<<<(count + kMlpBlock - 1) / kMlpBlock, kMlpBlock, smem, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(params_bf16), x_mean, x_scale, statics, gens, count, max_depth, peak, total,
      depth);
  return cuda_status(cudaGetLastError());
}

}  // extern "C"
