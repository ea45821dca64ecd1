// libaq.so: the sensitivity surrogate's MLP (in -> h -> h -> out, GELU on the
// hidden layers), bf16 weights with fp32 accumulation, training kernels
// (forward, backward, Adam).  No reference counterpart: the reference derives
// every scheme from a full autodiff run (mpm_solver.py:1093-1302).
//
// Parameter vector layout (float32 master, bf16 working copy, same order):
//   W1[h][in], b1[h], W2[h][h], b2[h], W3[out][h], b3[out]
// Biases are applied in fp32 from the master copy; weights are read as bf16
// and every dot product accumulates in fp32.
// Activations saved by the forward pass for the backward pass (fp32):
//   z1[B][h], a1[B][h], z2[B][h], a2[B][h]
// The layers are small (4 MFLOP per pass at batch 512): one thread per
// output element with the operand rows read through L1, no tensor cores.
#include <cuda_bf16.h>
#include <math.h>

#include "aq_common.cuh"

namespace aq {

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Y[b][n] = act(sum_k X[b][k] W[n][k] + bias[n]); Z (pre-activation) optional
__global__ void k_dense_fwd(const float* __restrict__ X, const __nv_bfloat16* __restrict__ W,
                            const float* __restrict__ bias, float* __restrict__ Z, float* __restrict__ Y, int B, int K,
                            int N, int act) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * N) return;
  const int b = i / N, n = i - b * N;
  const float* x = X + (size_t)b * K;
  const __nv_bfloat16* w = W + (size_t)n * K;
  float acc = bias[n];
  for (int k = 0; k < K; ++k) acc = fmaf(x[k], __bfloat162float(w[k]), acc);
  if (Z) Z[i] = acc;
  Y[i] = act ? gelu(acc) : acc;
}

// dW[n][k] = sum_b dZ[b][n] X[b][k];  db[n] = sum_b dZ[b][n]
__global__ void k_dense_wgrad(const float* __restrict__ dZ, const float* __restrict__ X, float* __restrict__ dW,
                              float* __restrict__ db, int B, int K, int N) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * (K + 1)) return;
  const int n = i / (K + 1), k = i - n * (K + 1);
  float acc = 0.f;
  if (k < K) {
    for (int b = 0; b < B; ++b) acc = fmaf(dZ[(size_t)b * N + n], X[(size_t)b * K + k], acc);
    dW[(size_t)n * K + k] = acc;
  } else {
    for (int b = 0; b < B; ++b) acc += dZ[(size_t)b * N + n];
    db[n] = acc;
  }
}

// dX[b][k] = (sum_n dZ[b][n] W[n][k]) * (gelu'(Zprev[b][k]) if act)
__global__ void k_dense_xgrad(const float* __restrict__ dZ, const __nv_bfloat16* __restrict__ W,
                              const float* __restrict__ Zprev, float* __restrict__ dX, int B, int K, int N, int act) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * K) return;
  const int b = i / K, k = i - b * K;
  float acc = 0.f;
  for (int n = 0; n < N; ++n) acc = fmaf(dZ[(size_t)b * N + n], __bfloat162float(W[(size_t)n * K + k]), acc);
  dX[i] = act ? acc * gelu_grad(Zprev[i]) : acc;
}

// Adam (Kingma & Ba 2015) on the fp32 master parameters, then the bf16 copy
__global__ void k_adam(float* __restrict__ p, __nv_bfloat16* __restrict__ pb, float* __restrict__ m,
                       float* __restrict__ v, const float* __restrict__ g, int64_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  pb[i] = __float2bfloat16_rn(pi);
}

__global__ void k_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ pb, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pb[i] = __float2bfloat16_rn(p[i]);
}

// dY = 2 (Y - T) M / max(1, sum M);  *loss += sum M (Y - T)^2 / max(1, sum M)
__global__ void k_mse_grad(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ M,
                           float* __restrict__ dY, int64_t n, float inv_count, float* __restrict__ loss) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < n) {
    const float r = (Y[i] - T[i]) * M[i];
    dY[i] = 2.f * r * inv_count;
    l = r * r * inv_count;
  }
#pragma unroll
  for (int k = 16; k; k >>= 1) l += __shfl_xor_sync(0xffffffffu, l, k);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, l);
}

struct MlpOffsets {
  int64_t w1, b1, w2, b2, w3, b3, total;
};

static MlpOffsets offsets(int in, int h, int out) {
  MlpOffsets o;
  o.w1 = 0;
  o.b1 = o.w1 + (int64_t)h * in;
  o.w2 = o.b1 + h;
  o.b2 = o.w2 + (int64_t)h * h;
  o.w3 = o.b2 + h;
  o.b3 = o.w3 + (int64_t)out * h;
  o.total = o.b3 + out;
  return o;
}

}  // namespace aq

using namespace aq;

extern "C" {

int64_t aq_mlp_param_count(int32_t in, int32_t h, int32_t out) {
  if (in < 1 || h < 1 || out < 1) return AQ_E_ARG;
  return offsets(in, h, out).total;
}

int aq_mlp_to_bf16(const float* d_params, uint16_t* d_params_bf16, int64_t n, void* stream) {
  if (!d_params || !d_params_bf16 || n < 0) return AQ_E_ARG;
  if (n == 0) return AQ_OK;
  k_to_bf16<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(d_params, (__nv_bfloat16*)d_params_bf16, n);
  AQ_CUDA_TRY(cudaGetLastError());
  return AQ_OK;
}

int aq_mlp_forward(int32_t in, int32_t h, int32_t out, const float* d_params, const uint16_t* d_params_bf16,
                   const float* d_x, int32_t B, float* d_y, float* d_act, void* stream) {
  if (!d_params || !d_params_bf16 || !d_x || !d_y || B < 1 || in < 1 || h < 1 || out < 1) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  const MlpOffsets o = offsets(in, h, out);
  const __nv_bfloat16* wb = (const __nv_bfloat16*)d_params_bf16;
  float *z1 = nullptr, *a1 = nullptr, *z2 = nullptr, *a2 = nullptr;
  float* tmp = nullptr;
  if (d_act) {
    z1 = d_act;
    a1 = z1 + (size_t)B * h;
    z2 = a1 + (size_t)B * h;
    a2 = z2 + (size_t)B * h;
  } else {
    AQ_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(float) * 2 * (size_t)B * h, st));
    a1 = tmp;
    a2 = tmp + (size_t)B * h;
  }
  k_dense_fwd<<<grid_for((int64_t)B * h, 128), 128, 0, st>>>(d_x, wb + o.w1, d_params + o.b1, z1, a1, B, in, h, 1);
  k_dense_fwd<<<grid_for((int64_t)B * h, 128), 128, 0, st>>>(a1, wb + o.w2, d_params + o.b2, z2, a2, B, h, h, 1);
  k_dense_fwd<<<grid_for((int64_t)B * out, 128), 128, 0, st>>>(a2, wb + o.w3, d_params + o.b3, nullptr, d_y, B, h,
                                                                out, 0);
  AQ_CUDA_TRY(cudaGetLastError());
  if (tmp) AQ_CUDA_TRY(cudaFreeAsync(tmp, st));
  return AQ_OK;
}

int aq_mlp_backward(int32_t in, int32_t h, int32_t out, const uint16_t* d_params_bf16, const float* d_x, int32_t B,
                    const float* d_act, const float* d_dy, float* d_grad, void* stream) {
  if (!d_params_bf16 || !d_x || !d_act || !d_dy || !d_grad || B < 1) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  const MlpOffsets o = offsets(in, h, out);
  const __nv_bfloat16* wb = (const __nv_bfloat16*)d_params_bf16;
  const float* z1 = d_act;
  const float* a1 = z1 + (size_t)B * h;
  const float* z2 = a1 + (size_t)B * h;
  const float* a2 = z2 + (size_t)B * h;
  float* dz = nullptr;
  AQ_CUDA_TRY(cudaMallocAsync((void**)&dz, sizeof(float) * 2 * (size_t)B * h, st));
  float* dz2 = dz;
  float* dz1 = dz + (size_t)B * h;
  k_dense_wgrad<<<grid_for((int64_t)out * (h + 1), 128), 128, 0, st>>>(d_dy, a2, d_grad + o.w3, d_grad + o.b3, B, h,
                                                                        out);
  k_dense_xgrad<<<grid_for((int64_t)B * h, 128), 128, 0, st>>>(d_dy, wb + o.w3, z2, dz2, B, h, out, 1);
  k_dense_wgrad<<<grid_for((int64_t)h * (h + 1), 128), 128, 0, st>>>(dz2, a1, d_grad + o.w2, d_grad + o.b2, B, h, h);
  k_dense_xgrad<<<grid_for((int64_t)B * h, 128), 128, 0, st>>>(dz2, wb + o.w2, z1, dz1, B, h, h, 1);
  k_dense_wgrad<<<grid_for((int64_t)h * (in + 1), 128), 128, 0, st>>>(dz1, d_x, d_grad + o.w1, d_grad + o.b1, B, in,
                                                                       h);
  AQ_CUDA_TRY(cudaGetLastError());
  AQ_CUDA_TRY(cudaFreeAsync(dz, st));
  return AQ_OK;
}

int aq_mlp_mse_grad(const float* d_y, const float* d_target, const float* d_mask, float* d_dy, int64_t n,
                    float count, float* d_loss, void* stream) {
  if (!d_y || !d_target || !d_mask || !d_dy || n < 1) return AQ_E_ARG;
  const float inv = 1.f / (count > 1.f ? count : 1.f);
  k_mse_grad<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(d_y, d_target, d_mask, d_dy, n, inv, d_loss);
  AQ_CUDA_TRY(cudaGetLastError());
  return AQ_OK;
}

int aq_mlp_adam(float* d_params, uint16_t* d_params_bf16, float* d_m, float* d_v, const float* d_grad, int64_t n,
                float lr, float beta1, float beta2, float eps, int32_t t, void* stream) {
  if (!d_params || !d_params_bf16 || !d_m || !d_v || !d_grad || n < 1 || t < 1) return AQ_E_ARG;
  const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
  k_adam<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(d_params, (__nv_bfloat16*)d_params_bf16, d_m, d_v, d_grad,
                                                          n, lr, beta1, beta2, eps, c1, c2);
  AQ_CUDA_TRY(cudaGetLastError());
  return AQ_OK;
}

}  // extern "C"
