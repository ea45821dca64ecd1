// libaq.so: layout builder, standalone codec kernels, error helpers.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "aq_codec.cuh"
#include "aq_common.cuh"

namespace aq {

static thread_local char g_last_error[256] = "";

void set_last_cuda_error(cudaError_t e, const char* what) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what, cudaGetErrorString(e));
}

// ---------------------------------------------------------- codec kernels

template <class T>
__global__ void __launch_bounds__(128) k_encode(const __grid_constant__ aq_layout L, const T* __restrict__ values,
                                                uint64_t* __restrict__ words, int64_t n,
                                                const int32_t* __restrict__ pid, uint64_t sk,
                                                const float* __restrict__ uf, const double* __restrict__ ud) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ns = L.n_slots;
  double vals[AQ_MAX_SLOTS];
#pragma unroll
  for (int s = 0; s < AQ_MAX_SLOTS; ++s) vals[s] = s < ns ? (double)values[i * ns + s] : 0.0;
  // The values are held as double so that f32 inputs pass through unchanged
  // (every f32 is exact in f64; encode casts back to the compute type).
  const int32_t id = pid ? pid[i] : (int32_t)i;
  encode_record<AQ_MAX_SLOTS, double>(L, vals, words + i * L.n_words, particle_key(sk, id),
                                      uf ? uf + i * ns : nullptr, ud ? ud + i * ns : nullptr);
}

template <class T>
__global__ void __launch_bounds__(128) k_decode(const __grid_constant__ aq_layout L, const uint64_t* __restrict__ words,
                                                T* __restrict__ values, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ns = L.n_slots;
  const uint64_t* w = words + i * L.n_words;
  for (int s = 0; s < ns; ++s) values[i * ns + s] = (T)decode_slot<double>(L, s, w);
}

template <class A, class B>
__global__ void k_state_error(const A* __restrict__ a, const B* __restrict__ b, int64_t n, int ns,
                              double* __restrict__ sq, unsigned long long* __restrict__ mx) {
  extern __shared__ double sh[];  // [ns] sums, [ns] maxima
  for (int s = threadIdx.x; s < 2 * ns; s += blockDim.x) sh[s] = 0.0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * ns;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(i % ns);
    const double d = fabs((double)a[i] - (double)b[i]);
    atomicAdd(&sh[s], d * d);
    // d >= 0, so the IEEE bit pattern orders like an unsigned integer
    atomicMax(reinterpret_cast<unsigned long long*>(&sh[ns + s]), (unsigned long long)__double_as_longlong(d));
  }
  __syncthreads();
  for (int s = threadIdx.x; s < ns; s += blockDim.x) {
    atomicAdd(&sq[s], sh[s]);
    atomicMax(&mx[s], (unsigned long long)__double_as_longlong(sh[ns + s]));
  }
}

}  // namespace aq

using namespace aq;

extern "C" {

int32_t aq_abi_version(void) { return AQ_ABI_VERSION; }

const char* aq_error_string(int32_t code) {
  switch (code) {
    case AQ_OK:
      return "ok";
    case AQ_E_ARG:
      return "bad argument";
    case AQ_E_LAYOUT:
      return "layout does not fit the simulator schema";
    case AQ_E_CUDA:
      return g_last_error[0] ? g_last_error : "CUDA error";
    case AQ_E_NOMEM:
      return "device allocation failed";
    case AQ_E_STATE:
      return "call not valid in the current state";
    case AQ_E_LIMIT:
      return "size above the documented maximum";
    default:
      return "unknown error";
  }
}

int aq_layout_build(int32_t n, const aq_scalar_spec* specs, int32_t compute_f64, int32_t use_dithering,
                    aq_layout* out) {
  if (!specs || !out || n < 1 || n > AQ_MAX_SLOTS) return AQ_E_ARG;
  aq_layout L;
  memset(&L, 0, sizeof(L));
  int gid[AQ_MAX_GROUPS], goff[AQ_MAX_GROUPS], gbits[AQ_MAX_GROUPS], ng = 0;
  int total = 0;
  for (int i = 0; i < n; ++i) {
    const aq_scalar_spec& sp = specs[i];
    aq_slot& S = L.slot[i];
    S.kind = sp.kind;
    S.is_signed = sp.is_signed ? 1 : 0;
    S.group = -1;
    int nb = sp.bits;
    switch (sp.kind) {
      case AQ_FIXED:
      case AQ_INT:
        if (nb < 1 || nb > 32) return AQ_E_ARG;
        break;
      case AQ_FLOAT_EXP:
      case AQ_SHARED_EXP: {
        if (sp.exp_bits < 1 || sp.exp_bits > 8) return AQ_E_ARG;
        const int db = nb - S.is_signed;
        if (db < 1 || db > 23) return AQ_E_ARG;
        S.exp_bits = sp.exp_bits;
        if (sp.kind == AQ_FLOAT_EXP) {
          S.exp_offset = total;
          total += sp.exp_bits;
        } else {
          int g = -1;
          for (int j = 0; j < ng; ++j)
            if (gid[j] == sp.group) g = j;
          if (g < 0) {
            if (ng == AQ_MAX_GROUPS) return AQ_E_LIMIT;
            g = ng++;
            gid[g] = sp.group;
            goff[g] = total;
            gbits[g] = sp.exp_bits;
            total += sp.exp_bits;
            S.exp_first = 1;
          } else if (gbits[g] != sp.exp_bits) {
            return AQ_E_ARG;
          }
          S.group = g;
          S.exp_offset = goff[g];
        }
        break;
      }
      case AQ_RAW_F32:
        nb = 32;
        break;
      case AQ_RAW_F64:
        nb = 64;
        break;
      default:
        return AQ_E_ARG;
    }
    S.bits = nb;
    S.bit_offset = total;
    total += nb;
    if (sp.kind == AQ_FIXED) {
      if (!(sp.range > 0.0) || !isfinite(sp.range) || !isfinite(sp.offset)) return AQ_E_ARG;
      const double scale = S.is_signed ? sp.range / ldexp(1.0, nb - 1) : sp.range / ldexp(1.0, nb);
      S.scale_f64 = scale;
      S.inv_scale_f64 = 1.0 / scale;
      S.offset_f64 = sp.offset;
      S.scale_f32 = (float)scale;
      S.inv_scale_f32 = (float)(1.0 / scale);
      S.offset_f32 = (float)sp.offset;
    }
  }
  L.n_slots = n;
  L.n_groups = ng;
  L.total_bits = total;
  L.n_words = (total + 63) / 64;
  L.compute_f64 = compute_f64 ? 1 : 0;
  L.use_dithering = use_dithering ? 1 : 0;
  *out = L;
  return AQ_OK;
}

int aq_encode(const aq_layout* L, const void* values, int32_t values_f64, uint64_t* words, int64_t n,
              const int32_t* pid, uint64_t seed, int64_t step, const void* uniforms, void* stream) {
  if (!L || n < 0 || (n > 0 && (!values || !words))) return AQ_E_ARG;
  if (L->n_slots < 1 || L->n_slots > AQ_MAX_SLOTS) return AQ_E_ARG;
  if (n == 0) return AQ_OK;
  const uint64_t sk = step_key(seed, step);
  const float* uf = (uniforms && !L->compute_f64) ? (const float*)uniforms : nullptr;
  const double* ud = (uniforms && L->compute_f64) ? (const double*)uniforms : nullptr;
  if (values_f64)
    k_encode<double><<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(*L, (const double*)values, words, n, pid, sk,
                                                                       uf, ud);
  else
    k_encode<float><<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(*L, (const float*)values, words, n, pid, sk,
                                                                      uf, ud);
  AQ_CUDA_TRY(cudaGetLastError());
  return AQ_OK;
}

int aq_decode(const aq_layout* L, const uint64_t* words, void* values, int32_t values_f64, int64_t n,
              void* stream) {
  if (!L || n < 0 || (n > 0 && (!values || !words))) return AQ_E_ARG;
  if (L->n_slots < 1 || L->n_slots > AQ_MAX_SLOTS) return AQ_E_ARG;
  if (n == 0) return AQ_OK;
  if (values_f64)
    k_decode<double><<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(*L, words, (double*)values, n);
  else
    k_decode<float><<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(*L, words, (float*)values, n);
  AQ_CUDA_TRY(cudaGetLastError());
  return AQ_OK;
}

int aq_state_error(const void* a, int32_t a_f64, const void* b, int32_t b_f64, int64_t n, int32_t ns,
                   double* h_sq, double* h_max, void* stream) {
  if (!a || !b || !h_sq || !h_max || n < 0 || ns < 1 || ns > 1024) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  double* d = nullptr;
  AQ_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(double) * 2 * ns, st));
  AQ_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(double) * 2 * ns, st));
  unsigned grid = (unsigned)(num_sms() * 4);
  size_t shm = sizeof(double) * 2 * ns;
  unsigned long long* mx = reinterpret_cast<unsigned long long*>(d + ns);
  if (n > 0) {
    if (a_f64 && b_f64)
      k_state_error<<<grid, 256, shm, st>>>((const double*)a, (const double*)b, n, ns, d, mx);
    else if (a_f64)
      k_state_error<<<grid, 256, shm, st>>>((const double*)a, (const float*)b, n, ns, d, mx);
    else if (b_f64)
      k_state_error<<<grid, 256, shm, st>>>((const float*)a, (const double*)b, n, ns, d, mx);
    else
      k_state_error<<<grid, 256, shm, st>>>((const float*)a, (const float*)b, n, ns, d, mx);
    AQ_CUDA_TRY(cudaGetLastError());
  }
  AQ_CUDA_TRY(cudaMemcpyAsync(h_sq, d, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaMemcpyAsync(h_max, d + ns, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaFreeAsync(d, st));
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  return AQ_OK;
}

}  // extern "C"

// ------------------------------------------ allocation-free state error
//
// aq_state_error_noalloc does the work of aq_state_error without allocating:
// its per-slot sums and maxima live in g_err_scratch, a fixed array of
// device memory that every GPU loading this library holds until the process
// exits (2 * AQ_NOALLOC_MAX_SLOTS doubles, 4 KiB).  Host code may not hand
// the array's name to a kernel (in host code it names a host-side stand-in);
// its device address is looked up once per device with cudaGetSymbolAddress
// while that device is current, and kept in g_err_addr.

namespace aq {

static __device__ __align__(256) double g_err_scratch[2 * AQ_NOALLOC_MAX_SLOTS];
static std::mutex g_err_mu;
static double* g_err_addr[AQ_NOALLOC_MAX_DEVICES];

}  // namespace aq

extern "C" int aq_state_error_noalloc(const void* a, int32_t a_f64, const void* b, int32_t b_f64, int64_t n,
                                      int32_t ns, double* h_sq, double* h_max, void* stream) {
  if (!a || !b || !h_sq || !h_max || n < 0 || ns < 1) return AQ_E_ARG;
  if (ns > AQ_NOALLOC_MAX_SLOTS) return AQ_E_LIMIT;
  int dev = 0;
  AQ_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= AQ_NOALLOC_MAX_DEVICES) return AQ_E_LIMIT;
  double* d = nullptr;
  {
    std::lock_guard<std::mutex> g(g_err_mu);
    if (!g_err_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_err_scratch);
      if (e != cudaSuccess || !p) {
        set_last_cuda_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(g_err_scratch)");
        return AQ_E_CUDA;
      }
      g_err_addr[dev] = static_cast<double*>(p);
    }
    d = g_err_addr[dev];
  }
  cudaStream_t st = as_stream(stream);
  // the array keeps the previous call's sums: clear this call's part
  AQ_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(double) * 2 * ns, st));
  unsigned grid = (unsigned)(num_sms() * 4);
  size_t shm = sizeof(double) * 2 * ns;
  unsigned long long* mx = reinterpret_cast<unsigned long long*>(d + ns);
  if (n > 0) {
    if (a_f64 && b_f64)
      k_state_error<<<grid, 256, shm, st>>>((const double*)a, (const double*)b, n, ns, d, mx);
    else if (a_f64)
      k_state_error<<<grid, 256, shm, st>>>((const double*)a, (const float*)b, n, ns, d, mx);
    else if (b_f64)
      k_state_error<<<grid, 256, shm, st>>>((const float*)a, (const double*)b, n, ns, d, mx);
    else
      k_state_error<<<grid, 256, shm, st>>>((const float*)a, (const float*)b, n, ns, d, mx);
    AQ_CUDA_TRY(cudaGetLastError());
  }
  AQ_CUDA_TRY(cudaMemcpyAsync(h_sq, d, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaMemcpyAsync(h_max, d + ns, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  return AQ_OK;
}
