// libaq.so: the sensitivity surrogate's MLP (in -> h -> h -> out, GELU on the
// hidden layers), bf16 weights with fp32 accumulation, training kernels
// (forward, backward, Adam).  No reference counterpart: the reference derives
// every scheme from a full autodiff run (mpm_solver.py:1093-1302).
//
// Parameter vector layout (float32 master, bf16 working copy, same order):
//   W1[h][in], b1[h], W2[h][h], b2[h], W3[out][h], b3[out]
// Biases are applied in fp32 from the master copy; weights are read as bf16.
// Activations saved by the forward pass for the backward pass (fp32):
//   z1[B][h], a1[B][h], z2[B][h], a2[B][h]
// Every contraction (forward, input gradient, weight gradient) runs on the
// bf16 tensor cores with fp32 accumulation: the operands, weights and
// activations alike, enter the products rounded to bf16 (round to nearest
// even); biases, pre-activations, GELU and its derivative stay fp32.
#include <cuda_bf16.h>
#include <math.h>

#include "aq_common.cuh"

namespace aq {

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ------------------------------------------------------ tensor-core GEMM
//
// C[m][n] = sum_k A(m, k) B(n, k) on bf16 tensor cores (mma.sync m16n8k16,
// fp32 accumulation) with a fused epilogue.  Operands are read from global
// memory in either major order and staged in shared memory as bf16 rows of
// k (fp32 sources are rounded to nearest even on the way in):
//   forward   Y = X W^T          A = X [M][K] (K-major), B = W [N][K] (K-major)
//   x-grad    dX = dZ W          A = dZ [M][K] (K-major), B(n, k) = W[k][n] (MN-major)
//   w-grad    dW = dZ^T X        A(m, k) = dZ[k][m] (MN-major), B(n, k) = X[k][n] (MN-major)
// A CTA of 4 warps computes a 64 x 64 tile of C in k chunks of 64; each
// warp a 32 x 32 quarter as 2 x 4 mma tiles of 16 x 8.

constexpr int GT = 64;       // CTA tile edge (m and n)
constexpr int GK = 64;       // k chunk
constexpr int GKP = GK + 8;  // padded row of the staged chunk (bf16): conflict-free 32-bit fragment loads

enum { EPI_FWD = 0, EPI_XGRAD = 1, EPI_STORE = 2 };

template <class T>
__device__ __forceinline__ float ld_f(const T* p, int64_t i);
template <>
__device__ __forceinline__ float ld_f<float>(const float* p, int64_t i) {
  return p[i];
}
template <>
__device__ __forceinline__ float ld_f<__nv_bfloat16>(const __nv_bfloat16* p, int64_t i) {
  return __bfloat162float(p[i]);
}

// A chunk of an operand (rows [r0, r0 + GT) x k [k0, k0 + GK)) is moved in
// two steps: stage_load reads the thread's GPT element pairs into registers
// (all loads issued together, zeros outside [R, K)), stage_store writes them
// to s[GT][GKP] as bf16.  The next chunk's loads are issued before the
// current chunk's products, so their latency overlaps the tensor-core work.
// kmajor: element (r, k) at src[r * ld + k], else at src[k * ld + r].
constexpr int GTHREADS = 128;                   // threads per GEMM CTA
constexpr int GPT = GT * GK / 2 / GTHREADS;     // element pairs per thread and operand

__device__ __forceinline__ void pair_pos(int i, bool kmajor, int& r, int& kk) {
  if (kmajor) {  // consecutive threads along k
    r = i / (GK / 2);
    kk = 2 * (i - r * (GK / 2));
  } else {  // consecutive threads along r
    kk = 2 * (i / GT);
    r = i - (kk / 2) * GT;
  }
}

template <class T>
__device__ __forceinline__ void stage_load(float (&v)[GPT][2], const T* src, int64_t ld, bool kmajor, int r0, int R,
                                           int k0, int K) {
#pragma unroll
  for (int q = 0; q < GPT; ++q) {
    int r, kk;
    pair_pos(threadIdx.x + q * GTHREADS, kmajor, r, kk);
    const int gr = r0 + r, gk = k0 + kk;
    v[q][0] = v[q][1] = 0.f;
    if (gr < R) {
      if (gk < K) v[q][0] = ld_f(src, kmajor ? (int64_t)gr * ld + gk : (int64_t)gk * ld + gr);
      if (gk + 1 < K) v[q][1] = ld_f(src, kmajor ? (int64_t)gr * ld + gk + 1 : (int64_t)(gk + 1) * ld + gr);
    }
  }
}

__device__ __forceinline__ void stage_store(__nv_bfloat16 (*s)[GKP], const float (&v)[GPT][2], bool kmajor) {
#pragma unroll
  for (int q = 0; q < GPT; ++q) {
    int r, kk;
    pair_pos(threadIdx.x + q * GTHREADS, kmajor, r, kk);
    *reinterpret_cast<__nv_bfloat162*>(&s[r][kk]) = __floats2bfloat162_rn(v[q][0], v[q][1]);
  }
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// epi: EPI_FWD   Z = acc + bias[n] (stored when Z), out = act ? gelu(Z) : Z
//      EPI_XGRAD out = act ? acc * gelu'(aux[m][n]) : acc
//      EPI_STORE out = acc
template <class TA, class TB, int EPI>
__global__ void __launch_bounds__(GTHREADS) k_gemm_bf16(const TA* __restrict__ A, int64_t lda, int a_kmajor,
                                                   const TB* __restrict__ B, int64_t ldb, int b_kmajor, int M, int N,
                                                   int K, const float* __restrict__ bias, const float* __restrict__ aux,
                                                   float* __restrict__ Z, float* __restrict__ out, int act) {
  __shared__ __align__(16) __nv_bfloat16 sA[GT][GKP];
  __shared__ __align__(16) __nv_bfloat16 sB[GT][GKP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.x * GT, n0 = blockIdx.y * GT;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
  float va[GPT][2], vb[GPT][2];
  stage_load(va, A, lda, a_kmajor != 0, m0, M, 0, K);
  stage_load(vb, B, ldb, b_kmajor != 0, n0, N, 0, K);
  for (int k0 = 0; k0 < K; k0 += GK) {
    stage_store(sA, va, a_kmajor != 0);
    stage_store(sB, vb, b_kmajor != 0);
    __syncthreads();
    if (k0 + GK < K) {  // next chunk in flight during this chunk's products
      stage_load(va, A, lda, a_kmajor != 0, m0, M, k0 + GK, K);
      stage_load(vb, B, ldb, b_kmajor != 0, n0, N, k0 + GK, K);
    }
#pragma unroll
    for (int kk = 0; kk < GK; kk += 16) {
      uint32_t af[2][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + 16 * i + g;
        af[i][0] = *reinterpret_cast<const uint32_t*>(&sA[r][kk + 2 * t]);
        af[i][1] = *reinterpret_cast<const uint32_t*>(&sA[r + 8][kk + 2 * t]);
        af[i][2] = *reinterpret_cast<const uint32_t*>(&sA[r][kk + 2 * t + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t*>(&sA[r + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + 8 * j + g;
        bf[j][0] = *reinterpret_cast<const uint32_t*>(&sB[c][kk + 2 * t]);
        bf[j][1] = *reinterpret_cast<const uint32_t*>(&sB[c][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i][0], af[i][1], af[i][2], af[i][3], bf[j][0], bf[j][1]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int m = m0 + wm + 16 * i + g + (e >= 2 ? 8 : 0);
        const int n = n0 + wn + 8 * j + 2 * t + (e & 1);
        if (m >= M || n >= N) continue;
        const int64_t o = (int64_t)m * N + n;
        float v = acc[i][j][e];
        if (EPI == EPI_FWD) {
          v += bias[n];
          if (Z) Z[o] = v;
          if (act) v = gelu(v);
        } else if (EPI == EPI_XGRAD) {
          if (act) v *= gelu_grad(aux[o]);
        }
        out[o] = v;
      }
}

// db[n] = sum_b dZ[b][n] in fp32 (one thread per column)
__global__ void k_colsum(const float* __restrict__ dZ, int B, int N, float* __restrict__ db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float acc = 0.f;
  for (int b = 0; b < B; ++b) acc += dZ[(size_t)b * N + n];
  db[n] = acc;
}

static dim3 gemm_grid(int M, int N) { return dim3((unsigned)((M + GT - 1) / GT), (unsigned)((N + GT - 1) / GT)); }

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
  k_gemm_bf16<float, __nv_bfloat16, EPI_FWD><<<gemm_grid(B, h), GTHREADS, 0, st>>>(
      d_x, in, 1, wb + o.w1, in, 1, B, h, in, d_params + o.b1, nullptr, z1, a1, 1);
  k_gemm_bf16<float, __nv_bfloat16, EPI_FWD><<<gemm_grid(B, h), GTHREADS, 0, st>>>(
      a1, h, 1, wb + o.w2, h, 1, B, h, h, d_params + o.b2, nullptr, z2, a2, 1);
  k_gemm_bf16<float, __nv_bfloat16, EPI_FWD><<<gemm_grid(B, out), GTHREADS, 0, st>>>(
      a2, h, 1, wb + o.w3, h, 1, B, out, h, d_params + o.b3, nullptr, nullptr, d_y, 0);
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
  // layer 3: dW3 = dy^T a2, db3, dz2 = (dy W3) * gelu'(z2)
  k_gemm_bf16<float, float, EPI_STORE><<<gemm_grid(out, h), GTHREADS, 0, st>>>(
      d_dy, out, 0, a2, h, 0, out, h, B, nullptr, nullptr, nullptr, d_grad + o.w3, 0);
  k_colsum<<<grid_for(out, 128), 128, 0, st>>>(d_dy, B, out, d_grad + o.b3);
  k_gemm_bf16<float, __nv_bfloat16, EPI_XGRAD><<<gemm_grid(B, h), GTHREADS, 0, st>>>(
      d_dy, out, 1, wb + o.w3, h, 0, B, h, out, nullptr, z2, nullptr, dz2, 1);
  // layer 2
  k_gemm_bf16<float, float, EPI_STORE><<<gemm_grid(h, h), GTHREADS, 0, st>>>(
      dz2, h, 0, a1, h, 0, h, h, B, nullptr, nullptr, nullptr, d_grad + o.w2, 0);
  k_colsum<<<grid_for(h, 128), 128, 0, st>>>(dz2, B, h, d_grad + o.b2);
  k_gemm_bf16<float, __nv_bfloat16, EPI_XGRAD><<<gemm_grid(B, h), GTHREADS, 0, st>>>(
      dz2, h, 1, wb + o.w2, h, 0, B, h, h, nullptr, z1, nullptr, dz1, 1);
  // layer 1
  k_gemm_bf16<float, float, EPI_STORE><<<gemm_grid(h, in), GTHREADS, 0, st>>>(
      dz1, h, 0, d_x, in, 0, h, in, B, nullptr, nullptr, nullptr, d_grad + o.w1, 0);
  k_colsum<<<grid_for(h, 128), 128, 0, st>>>(dz1, B, h, d_grad + o.b1);
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
