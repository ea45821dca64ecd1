// libaq.so: the quantized MLS-MPM substep on sm_100a.
//
// Data layout in HBM
//   records  : n x W u64 bit_pack records, kept sorted by grid cell (blocks
//              of 4^3 cells in 3D, 8^2 in 2D, cells inside a block), with a
//              particle-id array that moves with them.
//   grids    : two dense grids of R4 nodes (m, m*v) / (m, v), row-major,
//              used alternately as P2G target and G2P source.
//   binning  : per-cell counts/offsets, per-particle key and rank, and a list
//              of work items (block, first record, count <= 256).
//
// Kernels per substep
//   k_step   : one CTA per work item (persistent loop).  Loads the item's
//              records into shared memory, stages the block's grid tile,
//              G2P (gather, F/J/C/x update) of substep k, encodes the new
//              record (bit_pack_assign), decodes it and P2G of substep k+1
//              into a shared-memory tile, flushed to the grid with
//              vector reductions.  Either phase may be off (first / last
//              substep of a run).
//   k_grid   : grid_op (normalise, gravity, walls) on the accumulated grid
//              and clear of the other grid.
// Binning (k_bin, scan, k_scatter, k_items) runs every sort_interval
// substeps; between re-binnings particles may drift one cell out of their
// block's tile and fall back to global atomics beyond that.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <new>

#include "aq_codec.cuh"
#include "aq_common.cuh"

namespace aq {

constexpr int CH = 256;  // particles per work item = threads per CTA
constexpr int NW = CH / 32;

template <int D>
struct Geo {
  static constexpr int BS = D == 3 ? 4 : 8;  // block edge (cells)
  static constexpr int T = BS + 4;           // tile edge (nodes): 1-cell drift each side + stencil
  static constexpr int XS = D == 3 ? T * T + 4 : T;  // stride of the slowest tile axis (padded)
  static constexpr int TNP = D == 3 ? T * XS : T * T;  // nodes per tile plane incl. padding
  static constexpr int NOFF = D == 3 ? 27 : 9;
};

template <int D, bool HF, bool HM>
struct Sch {
  static constexpr int X = 0, V = D, C = 2 * D, FJ = 2 * D + D * D;
  static constexpr int NFJ = HF ? D * D : 1;
  static constexpr int MAT = FJ + NFJ;
  static constexpr int NS = MAT + (HM ? 1 : 0);
};

template <class R>
struct R4T;
template <>
struct R4T<float> {
  using type = float4;
};
template <>
struct R4T<double> {
  using type = double4;
};

template <class R>
struct SimK {
  int res[3], nb[3];
  int W, friction, bound_clip, n_mat;
  R inv_dx, dx, dt, p_mass, stress_coef, four_inv_dx, grav;
  double lb[3], ub[3];
  R clip_lo[3], clip_hi[3];
  int mat_kind[AQ_MAX_MATERIALS];
  R mu[AQ_MAX_MATERIALS], lam[AQ_MAX_MATERIALS];
};

// ---------------------------------------------------------------- helpers

template <class R>
__device__ __forceinline__ int base_of(R x, const SimK<R>& K, int d, unsigned& fl) {
  const R t = x * K.inv_dx - (R)0.5;
  if (t != t) {
    fl |= AQ_ST_NAN;
    return 0;
  }
  const R lim = (R)(K.res[d] - 3);
  if (t < (R)0) {
    fl |= AQ_ST_OUT_OF_DOMAIN;
    return 0;
  }
  if (t >= lim + (R)1) {
    fl |= AQ_ST_OUT_OF_DOMAIN;
    return K.res[d] - 3;
  }
  return (int)floor(t);
}

template <int D>
__device__ __forceinline__ int64_t cell_index(const int (&res)[3], int i, int j, int k) {
  return D == 3 ? ((int64_t)i * res[1] + j) * res[2] + k : (int64_t)i * res[1] + j;
}

__device__ __forceinline__ void red_add_v4(float4* addr, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}

__device__ __forceinline__ void red_add_node(float4* g, float m, float a, float b, float c) { red_add_v4(g, m, a, b, c); }

__device__ __forceinline__ void red_add_node(double4* g, double m, double a, double b, double c) {
  double* p = reinterpret_cast<double*>(g);
  atomicAdd(p, m);
  atomicAdd(p + 1, a);
  atomicAdd(p + 2, b);
  atomicAdd(p + 3, c);
}

__device__ __forceinline__ void atomic_max_d(double* a, double v) {
  unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
  unsigned long long old = *p;
  while (v > __longlong_as_double((long long)old)) {
    const unsigned long long prev = atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
    if (prev == old) break;
    old = prev;
  }
}

__device__ __forceinline__ void atomic_min_d(double* a, double v) {
  unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
  unsigned long long old = *p;
  while (v < __longlong_as_double((long long)old)) {
    const unsigned long long prev = atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
    if (prev == old) break;
    old = prev;
  }
}

// ------------------------------------------------------------- materials

template <int D, class R>
__device__ __forceinline__ R det(const R* F) {
  if (D == 2) return F[0] * F[3] - F[1] * F[2];
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
         F[2] * (F[3] * F[7] - F[4] * F[6]);
}

template <class R>
__device__ __forceinline__ R rsqrt_r(R v);
template <>
__device__ __forceinline__ float rsqrt_r<float>(float v) {
  return 1.0f / sqrtf(v);
}
template <>
__device__ __forceinline__ double rsqrt_r<double>(double v) {
  return 1.0 / sqrt(v);
}

// Rotation of the polar decomposition: 2D closed form (linalg_impl.py:9-26);
// 3D by Newton's iteration X <- (X + X^-T)/2.
template <int D, class R>
__device__ __forceinline__ void polar_rot(const R* F, R* Rm) {
  if (D == 2) {
    const R x = F[0] + F[3], y = F[2] - F[1];
    const R sc = rsqrt_r<R>(x * x + y * y);
    const R c = x * sc, s = y * sc;
    Rm[0] = c;
    Rm[1] = -s;
    Rm[2] = s;
    Rm[3] = c;
  } else {
    R X[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) X[k] = F[k];
    const R tol = sizeof(R) == 4 ? (R)1e-6 : (R)1e-12;
    for (int it = 0; it < 20; ++it) {
      const R c00 = X[4] * X[8] - X[5] * X[7], c01 = X[5] * X[6] - X[3] * X[8], c02 = X[3] * X[7] - X[4] * X[6];
      const R c10 = X[2] * X[7] - X[1] * X[8], c11 = X[0] * X[8] - X[2] * X[6], c12 = X[1] * X[6] - X[0] * X[7];
      const R c20 = X[1] * X[5] - X[2] * X[4], c21 = X[2] * X[3] - X[0] * X[5], c22 = X[0] * X[4] - X[1] * X[3];
      const R id = (R)1 / (X[0] * c00 + X[1] * c01 + X[2] * c02);
      const R Y[9] = {c00 * id, c01 * id, c02 * id, c10 * id, c11 * id, c12 * id, c20 * id, c21 * id, c22 * id};
      R diff = 0;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const R nx = (R)0.5 * (X[k] + Y[k]);
        diff += (nx - X[k]) * (nx - X[k]);
        X[k] = nx;
      }
      if (diff < tol * tol) break;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) Rm[k] = X[k];
  }
}

// compute_cauchy (mpm_solver.py:1012-1031), plus the fixed-corotated 3D law.
template <int D, bool HF, class R>
__device__ __forceinline__ void cauchy(const SimK<R>& K, int mat, const R* F, R J, R* out) {
  const int mk = K.mat_kind[mat];
  const R mu = K.mu[mat], lam = K.lam[mat];
#pragma unroll
  for (int k = 0; k < D * D; ++k) out[k] = 0;
  if (mk == AQ_MAT_FLUID) {
    const R Jf = HF ? det<D, R>(F) : J;
#pragma unroll
    for (int d = 0; d < D; ++d) out[d * D + d] = lam * (Jf - (R)1);
    return;
  }
  if (!HF) return;
  const R Jd = det<D, R>(F);
  if (D == 2 || mk == AQ_MAT_COROTATED) {
    R Rm[D * D];
    polar_rot<D, R>(F, Rm);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R s = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) s += (F[i * D + k] - Rm[i * D + k]) * F[j * D + k];
        out[i * D + j] = (R)2 * mu * s + (i == j ? lam * Jd * (Jd - (R)1) : (R)0);
      }
  } else {
    const R lj = lam * log(Jd);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R s = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) s += F[i * D + k] * F[j * D + k];
        out[i * D + j] = mu * (s - (i == j ? (R)1 : (R)0)) + lj;
      }
  }
}

// ------------------------------------------------------------ binning

template <int D, class R>
__global__ void __launch_bounds__(256) k_bin(const __grid_constant__ aq_layout L, const SimK<R> K,
                                             const uint64_t* __restrict__ words, int64_t n,
                                             int32_t* __restrict__ keys, int32_t* __restrict__ ranks,
                                             int32_t* __restrict__ cell_count, unsigned* __restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t* w = words + i * K.W;
  unsigned fl = 0;
  int b[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) b[d] = base_of<R>(decode_slot<R>(L, d, w), K, d, fl);
  constexpr int BS = Geo<D>::BS;
  int key;
  if (D == 3) {
    const int blk = ((b[0] / BS) * K.nb[1] + b[1] / BS) * K.nb[2] + b[2] / BS;
    key = blk * 64 + ((b[0] % BS) * BS + b[1] % BS) * BS + b[2] % BS;
  } else {
    const int blk = (b[0] / BS) * K.nb[1] + b[1] / BS;
    key = blk * 64 + (b[0] % BS) * BS + b[1] % BS;
  }
  keys[i] = key;
  ranks[i] = atomicAdd(&cell_count[key], 1);
  if (fl) atomicOr(status, fl);
}

__global__ void __launch_bounds__(256) k_scatter(const uint64_t* __restrict__ win, const int32_t* __restrict__ pin,
                                                 uint64_t* __restrict__ wout, int32_t* __restrict__ pout,
                                                 const int32_t* __restrict__ keys, const int32_t* __restrict__ ranks,
                                                 const int32_t* __restrict__ start, int64_t n, int W) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t dst = (int64_t)start[keys[i]] + ranks[i];
  for (int j = 0; j < W; ++j) wout[dst * W + j] = win[i * W + j];
  pout[dst] = pin[i];
}

__global__ void k_items(const int32_t* __restrict__ start, int nblk, int4* __restrict__ items,
                        int32_t* __restrict__ n_items) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblk) return;
  const int s = start[(int64_t)b * 64], e = start[(int64_t)(b + 1) * 64];
  const int cnt = e - s;
  if (cnt <= 0) return;
  const int k = (cnt + CH - 1) / CH;
  const int at = atomicAdd(n_items, k);
  for (int j = 0; j < k; ++j) items[at + j] = make_int4(b, s + j * CH, min(CH, cnt - j * CH), 0);
}

// Exclusive scan of n int32 counts into out[0..n] (out[n] = total), in
// tiles of 4096: per-tile sums, one CTA scans the tile sums, per-tile scan.
constexpr int SCAN_T = 1024, SCAN_V = 4, SCAN_TILE = SCAN_T * SCAN_V;

__device__ __forceinline__ int block_excl_scan(int v, int* sh, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sh[lane] = s;
  }
  __syncthreads();
  total = sh[(blockDim.x >> 5) - 1];
  const int r = x - v + (warp ? sh[warp - 1] : 0);
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_sums(const int32_t* __restrict__ in, int64_t n,
                                                      int32_t* __restrict__ sums) {
  __shared__ int sh[32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_V;
  int v = 0;
#pragma unroll
  for (int k = 0; k < SCAN_V; ++k) v += base + k < n ? in[base + k] : 0;
  int total;
  block_excl_scan(v, sh, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_top(int32_t* __restrict__ sums, int nt, int32_t* __restrict__ out,
                                                     int64_t n) {
  __shared__ int sh[32];
  const int per = (nt + SCAN_T - 1) / SCAN_T;
  const int b = threadIdx.x * per;
  int v = 0;
  for (int k = 0; k < per; ++k) v += b + k < nt ? sums[b + k] : 0;
  int total;
  int run = block_excl_scan(v, sh, total);
  for (int k = 0; k < per; ++k) {
    if (b + k < nt) {
      const int s = sums[b + k];
      sums[b + k] = run;
      run += s;
    }
  }
  if (threadIdx.x == 0) out[n] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_apply(const int32_t* __restrict__ in, int64_t n,
                                                       const int32_t* __restrict__ offs, int32_t* __restrict__ out) {
  __shared__ int sh[32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_V;
  int loc[SCAN_V], v = 0;
#pragma unroll
  for (int k = 0; k < SCAN_V; ++k) {
    loc[k] = base + k < n ? in[base + k] : 0;
    v += loc[k];
  }
  int total;
  int run = block_excl_scan(v, sh, total) + offs[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_V; ++k) {
    if (base + k < n) out[base + k] = run;
    run += loc[k];
  }
}

// --------------------------------------------------------------- substep

struct StepArgs {
  uint64_t* words;
  const int32_t* pid;
  const int4* items;
  const int32_t* n_items;
  const void* grid_in;   // G2P source (after grid_op)
  void* grid_out;        // P2G target (zeroed)
  unsigned* status;
  unsigned long long* fallbacks;
  double* rmax;
  double* rmin;
  uint64_t sk;           // dithering key of the G2P substep
  int do_g2p, do_p2g, ranges;
};

template <int D, bool HF, bool HM, class R>
__global__ void __launch_bounds__(CH, 2) k_step(const __grid_constant__ aq_layout L, const SimK<R> K,
                                                const StepArgs A) {
  using S = Sch<D, HF, HM>;
  using G = Geo<D>;
  using R4 = typename R4T<R>::type;
  constexpr int NS = S::NS;
  constexpr int T = G::T;
  constexpr int TNP = G::TNP;
  const int W = K.W;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile = reinterpret_cast<R*>(smem_raw);                              // (D+1) planes of TNP
  int32_t* spid = reinterpret_cast<int32_t*>(tile + (D + 1) * TNP);      // CH
  uint64_t* srec = reinterpret_cast<uint64_t*>(spid + CH);               // CH * W (8-byte aligned: see host)

  const int tid = threadIdx.x;
  const int p = (tid & 31) * NW + (tid >> 5);  // lane-major: a warp spans 32 distinct cells
  const int nitems = *A.n_items;
  const R4* gin = reinterpret_cast<const R4*>(A.grid_in);
  R4* gout = reinterpret_cast<R4*>(A.grid_out);
  unsigned fl = 0;
  unsigned nfall = 0;

  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 item = A.items[it];
    const int cnt = item.z;
    const int64_t first = item.y;
    int o[3] = {0, 0, 0};  // tile origin (node coordinates)
    {
      int blk = item.x;
      if (D == 3) {
        o[2] = (blk % K.nb[2]) * G::BS - 1;
        blk /= K.nb[2];
      }
      o[1] = (blk % K.nb[1]) * G::BS - 1;
      o[0] = (blk / K.nb[1]) * G::BS - 1;
    }
    // ---- records and ids of the item into shared memory (coalesced)
    {
      const uint64_t* src = A.words + first * W;
      for (int j = tid; j < cnt * W; j += CH) srec[j] = src[j];
      for (int j = tid; j < cnt; j += CH) spid[j] = A.pid[first + j];
    }
    // ---- stage the grid tile for G2P
    if (A.do_g2p) {
      for (int j = tid; j < TNP; j += CH) {
        int l0, l1, l2 = 0;
        if (D == 3) {
          l0 = j / G::XS;
          const int r = j - l0 * G::XS;
          l1 = r / T;
          l2 = r - l1 * T;
        } else {
          l0 = j / T;
          l1 = j - l0 * T;
        }
        const int g0 = o[0] + l0, g1 = o[1] + l1, g2 = o[2] + l2;
        const bool ok = (D == 3 ? l1 < T : true) && g0 >= 0 && g0 < K.res[0] && g1 >= 0 && g1 < K.res[1] &&
                        (D == 2 || (g2 >= 0 && g2 < K.res[2]));
        R4 v = {0, 0, 0, 0};
        if (ok) v = gin[cell_index<D>(K.res, g0, g1, g2)];
        tile[0 * TNP + j] = v.y;
        tile[1 * TNP + j] = v.z;
        if (D == 3) tile[2 * TNP + j] = v.w;
      }
    }
    __syncthreads();

    const bool active = p < cnt;
    R vals[NS];
    if (active) decode_record<NS, R>(L, srec + p * W, vals);

    // ---------------------------------------------------------------- G2P
    if (A.do_g2p && active) {
      int base[3] = {0, 0, 0};
      R fx[3] = {0, 0, 0}, w[3][3];
      bool in_tile = true;
#pragma unroll
      for (int d = 0; d < D; ++d) {
        base[d] = base_of<R>(vals[S::X + d], K, d, fl);
        fx[d] = vals[S::X + d] * K.inv_dx - (R)base[d];
        w[0][d] = (R)0.5 * ((R)1.5 - fx[d]) * ((R)1.5 - fx[d]);
        w[1][d] = (R)0.75 - (fx[d] - (R)1) * (fx[d] - (R)1);
        w[2][d] = (R)0.5 * (fx[d] - (R)0.5) * (fx[d] - (R)0.5);
        const int l = base[d] - o[d];
        in_tile = in_tile && l >= 0 && l <= T - 3;
      }
      R nv[D], Sm[D][D];
#pragma unroll
      for (int d = 0; d < D; ++d) {
        nv[d] = 0;
#pragma unroll
        for (int e = 0; e < D; ++e) Sm[d][e] = 0;
      }
      auto accum = [&](int a, int b, int c, const R* gv) {
        const R weight = D == 3 ? w[a][0] * w[b][1] * w[c][2] : w[a][0] * w[b][1];
        const int off[3] = {a, b, c};
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const R wg = weight * gv[d];
          nv[d] += wg;
#pragma unroll
          for (int e = 0; e < D; ++e) {
            if (off[e] == 1) Sm[d][e] += wg;
            if (off[e] == 2) Sm[d][e] += (R)2 * wg;
          }
        }
      };
      if (in_tile) {
        const int lb = D == 3 ? (base[0] - o[0]) * G::XS + (base[1] - o[1]) * T + (base[2] - o[2])
                              : (base[0] - o[0]) * T + (base[1] - o[1]);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < (D == 3 ? 3 : 1); ++c) {
              const int idx = lb + (D == 3 ? a * G::XS + b * T + c : a * T + b);
              R gv[D];
#pragma unroll
              for (int d = 0; d < D; ++d) gv[d] = tile[d * TNP + idx];
              accum(a, b, c, gv);
            }
      } else {
        ++nfall;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < (D == 3 ? 3 : 1); ++c) {
              const R4 g = gin[cell_index<D>(K.res, base[0] + a, base[1] + b, D == 3 ? base[2] + c : 0)];
              const R gv[3] = {g.y, g.z, g.w};
              accum(a, b, c, gv);
            }
      }
      // new_C = 4 inv_dx sum w g_v (off - fx)^T;  new_x = x + dt new_v
      R nC[D * D];
#pragma unroll
      for (int d = 0; d < D; ++d)
#pragma unroll
        for (int e = 0; e < D; ++e) nC[d * D + e] = K.four_inv_dx * (Sm[d][e] - nv[d] * fx[e]);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        R nx = vals[S::X + d] + K.dt * nv[d];
        if (K.bound_clip) nx = fmax(fmin(nx, K.clip_hi[d]), K.clip_lo[d]);
        vals[S::X + d] = nx;
        vals[S::V + d] = nv[d];
      }
      const int mat = HM ? min(max((int)vals[S::MAT], 0), K.n_mat - 1) : 0;
      if (HF) {
        R nF[D * D];
#pragma unroll
        for (int i = 0; i < D; ++i)
#pragma unroll
          for (int j = 0; j < D; ++j) {
            R acc = 0;
#pragma unroll
            for (int k = 0; k < D; ++k)
              acc += ((i == k ? (R)1 : (R)0) + K.dt * nC[i * D + k]) * vals[S::FJ + k * D + j];
            nF[i * D + j] = acc;
          }
        if (HM && K.mat_kind[mat] == AQ_MAT_FLUID) {  // fluid in an F record keeps only J
          const R Jn = det<D, R>(nF);
          const R sj = D == 3 ? cbrt(Jn) : sqrt(Jn);
#pragma unroll
          for (int i = 0; i < D; ++i)
#pragma unroll
            for (int j = 0; j < D; ++j) nF[i * D + j] = i == j ? sj : (R)0;
        }
#pragma unroll
        for (int k = 0; k < D * D; ++k) vals[S::FJ + k] = nF[k];
      } else {
        R tr = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) tr += nC[d * D + d];
        vals[S::FJ] = ((R)1 + K.dt * tr) * vals[S::FJ];
      }
#pragma unroll
      for (int k = 0; k < D * D; ++k) vals[S::C + k] = nC[k];
      // bit_pack_assign of the new state; vals become the values a later
      // read of the record returns (input of the next P2G)
      encode_record<NS, R>(L, vals, srec + p * W, particle_key(A.sk, spid[p]), nullptr, nullptr);
    }

    // -------------------------------------------- range detection (opt)
    if (A.ranges && A.do_g2p) {
      const int lane = tid & 31;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        double mx = active ? (double)vals[s] : -INFINITY, mn = active ? (double)vals[s] : INFINITY;
#pragma unroll
        for (int k = 16; k; k >>= 1) {
          mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, k));
          mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, k));
        }
        if (lane == 0) {
          atomic_max_d(A.rmax + s, mx);
          atomic_min_d(A.rmin + s, mn);
        }
      }
    }

    __syncthreads();
    if (A.do_g2p) {  // write the item's records back (coalesced)
      uint64_t* dst = A.words + first * W;
      for (int j = tid; j < cnt * W; j += CH) dst[j] = srec[j];
    }

    // ---------------------------------------------------------------- P2G
    if (A.do_p2g) {
      for (int j = tid; j < (D + 1) * TNP; j += CH) tile[j] = 0;
      __syncthreads();
      if (active) {
        const int mat = HM ? min(max((int)vals[S::MAT], 0), K.n_mat - 1) : 0;
        int base[3] = {0, 0, 0};
        R fx[3] = {0, 0, 0}, w[3][3];
        bool in_tile = true;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          base[d] = base_of<R>(vals[S::X + d], K, d, fl);
          fx[d] = vals[S::X + d] * K.inv_dx - (R)base[d];
          w[0][d] = (R)0.5 * ((R)1.5 - fx[d]) * ((R)1.5 - fx[d]);
          w[1][d] = (R)0.75 - (fx[d] - (R)1) * (fx[d] - (R)1);
          w[2][d] = (R)0.5 * (fx[d] - (R)0.5) * (fx[d] - (R)0.5);
          const int l = base[d] - o[d];
          in_tile = in_tile && l >= 0 && l <= T - 3;
        }
        R cau[D * D];
        cauchy<D, HF, R>(K, mat, vals + S::FJ, vals[S::FJ], cau);
        // affine = stress + m C;  node value = m v + affine (off - fx) dx
        //   = q + A off  with q = m v - affine fx dx, A = affine dx
        R Aff[D * D], q[D];
#pragma unroll
        for (int k = 0; k < D * D; ++k) Aff[k] = (K.stress_coef * cau[k] + K.p_mass * vals[S::C + k]) * K.dx;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          R s = K.p_mass * vals[S::V + d];
#pragma unroll
          for (int e = 0; e < D; ++e) s -= Aff[d * D + e] * fx[e];
          q[d] = s;
        }
        if (!in_tile) ++nfall;
        const int lb = D == 3 ? (base[0] - o[0]) * G::XS + (base[1] - o[1]) * T + (base[2] - o[2])
                              : (base[0] - o[0]) * T + (base[1] - o[1]);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < (D == 3 ? 3 : 1); ++c) {
              const R weight = D == 3 ? w[a][0] * w[b][1] * w[c][2] : w[a][0] * w[b][1];
              const int off[3] = {a, b, c};
              R mv[3] = {0, 0, 0};
#pragma unroll
              for (int d = 0; d < D; ++d) {
                R s = q[d];
#pragma unroll
                for (int e = 0; e < D; ++e) {
                  if (off[e] == 1) s += Aff[d * D + e];
                  if (off[e] == 2) s += (R)2 * Aff[d * D + e];
                }
                mv[d] = weight * s;
              }
              const R m = weight * K.p_mass;
              if (in_tile) {
                const int idx = lb + (D == 3 ? a * G::XS + b * T + c : a * T + b);
                atomicAdd(&tile[idx], m);
#pragma unroll
                for (int d = 0; d < D; ++d) atomicAdd(&tile[(1 + d) * TNP + idx], mv[d]);
              } else {
                R4* g = gout + cell_index<D>(K.res, base[0] + a, base[1] + b, D == 3 ? base[2] + c : 0);
                red_add_node(g, m, mv[0], mv[1], mv[2]);
              }
            }
      }
      __syncthreads();
      // flush the tile: one vector reduction per touched node
      for (int j = tid; j < TNP; j += CH) {
        const R m = tile[j];
        if (m == (R)0) continue;
        int l0, l1, l2 = 0;
        if (D == 3) {
          l0 = j / G::XS;
          const int r = j - l0 * G::XS;
          l1 = r / T;
          l2 = r - l1 * T;
        } else {
          l0 = j / T;
          l1 = j - l0 * T;
        }
        const int g0 = o[0] + l0, g1 = o[1] + l1, g2 = o[2] + l2;
        if (g0 < 0 || g0 >= K.res[0] || g1 < 0 || g1 >= K.res[1] || (D == 3 && (g2 < 0 || g2 >= K.res[2])))
          continue;
        red_add_node(gout + cell_index<D>(K.res, g0, g1, g2), m, tile[TNP + j], tile[2 * TNP + j],
                     D == 3 ? tile[3 * TNP + j] : (R)0);
      }
    }
    __syncthreads();
  }
  if (fl) atomicOr(A.status, fl);
  if (nfall) atomicAdd(A.fallbacks, (unsigned long long)nfall);
}

// grid_op (mpm_solver.py:633-665) on `acc`; zero `clr`.
template <int D, class R>
__global__ void __launch_bounds__(256) k_grid(const SimK<R> K, void* acc_, void* clr_, int64_t ncell) {
  using R4 = typename R4T<R>::type;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  R4* acc = reinterpret_cast<R4*>(acc_);
  R4* clr = reinterpret_cast<R4*>(clr_);
  if (clr) clr[c] = R4{0, 0, 0, 0};
  if (!acc) return;
  int I[3];
  if (D == 3) {
    I[2] = (int)(c % K.res[2]);
    I[1] = (int)((c / K.res[2]) % K.res[1]);
    I[0] = (int)(c / ((int64_t)K.res[2] * K.res[1]));
  } else {
    I[1] = (int)(c % K.res[1]);
    I[0] = (int)(c / K.res[1]);
    I[2] = 0;
  }
  R4 g = acc[c];
  const R inv_m = (R)1 / (g.x + (R)1e-10);
  R v[3] = {inv_m * g.y, inv_m * g.z, D == 3 ? inv_m * g.w : (R)0};
  v[1] -= K.dt * K.grav;
  if (K.friction && I[1] < K.lb[1] && v[1] < (R)0) {  // n = (0,1,0), v = (v - n (n.v)) * 0.02
    v[1] = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) v[d] *= (R)0.02;
  }
#pragma unroll
  for (int k = 0; k < D; ++k) {
    if (I[k] < K.lb[k] && v[k] < (R)0) v[k] = 0;
    if (I[k] > K.ub[k] && v[k] > (R)0) v[k] = 0;
  }
  acc[c] = R4{g.x, v[0], v[1], v[2]};
}

// decode records into particle order
template <class T>
__global__ void __launch_bounds__(128) k_get_state(const __grid_constant__ aq_layout L,
                                                   const uint64_t* __restrict__ words,
                                                   const int32_t* __restrict__ pid, T* __restrict__ out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ns = L.n_slots;
  const uint64_t* w = words + i * L.n_words;
  const int64_t dst = pid[i];
  for (int s = 0; s < ns; ++s) out[dst * ns + s] = (T)decode_slot<double>(L, s, w);
}

__global__ void k_words_permute(const uint64_t* __restrict__ in, const int32_t* __restrict__ pid,
                                uint64_t* __restrict__ out, int64_t n, int W, int to_particle_order) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t a = to_particle_order ? (int64_t)pid[i] : i;
  const int64_t b = to_particle_order ? i : (int64_t)pid[i];
  for (int j = 0; j < W; ++j) out[a * W + j] = in[b * W + j];
}

__global__ void k_iota(int32_t* p, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = (int32_t)i;
}

template <int D, class R>
__global__ void __launch_bounds__(256) k_loss(const __grid_constant__ aq_layout L, const SimK<R> K,
                                              const uint64_t* __restrict__ words, int64_t n, double* out) {
  __shared__ double sh[8];
  double acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t* w = words + i * K.W;
    double vv = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const double v = (double)decode_slot<R>(L, D + d, w);
      vv += v * v;
    }
    if (D == 3)
      acc += 0.5 * (double)K.p_mass * vv + (double)K.grav * (double)K.p_mass * (double)decode_slot<R>(L, 1, w);
    else
      acc += vv;
  }
#pragma unroll
  for (int k = 16; k; k >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, k);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[k];
    atomicAdd(out, s);
  }
}

// ------------------------------------------------------------------ host

struct SimBase {
  virtual ~SimBase() {}
  virtual int substeps(int n, cudaStream_t st) = 0;
  virtual int loss(double* h, cudaStream_t st) = 0;
  virtual int sort(cudaStream_t st) = 0;
  virtual size_t smem_bytes() const = 0;
};

}  // namespace aq

struct aq_sim {
  aq_params P;
  aq_layout L;
  int W = 0, NS = 0, D = 0;
  int64_t n = 0;
  uint64_t* words[2] = {nullptr, nullptr};
  int32_t* pid[2] = {nullptr, nullptr};
  int cur = 0;
  void* grid[2] = {nullptr, nullptr};
  int zero_grid = 0;
  int64_t ncell = 0, nkeys = 0;
  int nblk = 0;
  int32_t *keys = nullptr, *ranks = nullptr, *cell_count = nullptr, *cell_start = nullptr, *scan_sums = nullptr;
  int4* items = nullptr;
  int32_t* n_items = nullptr;
  int64_t max_items = 0;
  unsigned* status = nullptr;
  unsigned long long* fallbacks = nullptr;
  double *rmax = nullptr, *rmin = nullptr;
  double* dloss = nullptr;
  int ranges_on = 0;
  int64_t step = 0;
  int since_sort = 0;
  bool sorted = false;
  int64_t launches = 0;
  int step_grid = 0;
  aq::SimBase* impl = nullptr;
  // kernel timing (aq_sim_profile_*): event pairs per kernel kind
  static constexpr int PROF_CAP = 8192;
  int prof_on = 0;
  cudaEvent_t* prof_ev[2] = {nullptr, nullptr};  // [PROF_CAP * 2]
  int prof_n[2] = {0, 0};
};

namespace aq {

template <int D, bool HF, bool HM, class R>
struct SimImpl final : SimBase {
  aq_sim* s;
  SimK<R> K;
  explicit SimImpl(aq_sim* sim) : s(sim) {
    const aq_params& P = sim->P;
    memset(&K, 0, sizeof(K));
    for (int d = 0; d < 3; ++d) {
      K.res[d] = d < D ? P.res[d] : 1;
      K.nb[d] = d < D ? (P.res[d] + Geo<D>::BS - 1) / Geo<D>::BS : 1;
      K.lb[d] = P.lb[d];
      K.ub[d] = P.ub[d];
      K.clip_lo[d] = (R)(P.lb[d] * P.dx);
      K.clip_hi[d] = (R)(P.ub[d] * P.dx);
    }
    K.W = sim->W;
    K.friction = P.use_friction;
    K.bound_clip = P.use_bound_clip;
    K.n_mat = P.n_materials < 1 ? 1 : P.n_materials;
    K.inv_dx = (R)(1.0 / P.dx);
    K.dx = (R)P.dx;
    K.dt = (R)P.dt;
    K.p_mass = (R)P.p_mass;
    K.stress_coef = (R)(-(P.dt * P.p_vol * 4.0 * (1.0 / P.dx) * (1.0 / P.dx)));
    K.four_inv_dx = (R)(4.0 * (1.0 / P.dx));
    K.grav = (R)P.gravity;
    for (int m = 0; m < AQ_MAX_MATERIALS; ++m) {
      K.mat_kind[m] = P.mat[m].kind;
      K.mu[m] = (R)P.mat[m].mu;
      K.lam[m] = (R)P.mat[m].lam;
    }
  }

  size_t smem_bytes() const override {
    size_t b = sizeof(R) * (D + 1) * Geo<D>::TNP + sizeof(int32_t) * CH;
    b = (b + 15) & ~(size_t)15;
    return b + sizeof(uint64_t) * (size_t)CH * s->W;
  }

  int sort(cudaStream_t st) override {
    aq_sim* S_ = s;
    const int64_t n = S_->n;
    AQ_CUDA_TRY(cudaMemsetAsync(S_->cell_count, 0, sizeof(int32_t) * S_->nkeys, st));
    AQ_CUDA_TRY(cudaMemsetAsync(S_->n_items, 0, sizeof(int32_t), st));
    k_bin<D, R><<<grid_for(n, 256), 256, 0, st>>>(S_->L, K, S_->words[S_->cur], n, S_->keys, S_->ranks, S_->cell_count,
                                                  S_->status);
    const int nt = (int)((S_->nkeys + SCAN_TILE - 1) / SCAN_TILE);
    k_scan_sums<<<nt, SCAN_T, 0, st>>>(S_->cell_count, S_->nkeys, S_->scan_sums);
    k_scan_top<<<1, SCAN_T, 0, st>>>(S_->scan_sums, nt, S_->cell_start, S_->nkeys);
    k_scan_apply<<<nt, SCAN_T, 0, st>>>(S_->cell_count, S_->nkeys, S_->scan_sums, S_->cell_start);
    const int nxt = 1 - S_->cur;
    k_scatter<<<grid_for(n, 256), 256, 0, st>>>(S_->words[S_->cur], S_->pid[S_->cur], S_->words[nxt], S_->pid[nxt],
                                                S_->keys, S_->ranks, S_->cell_start, n, S_->W);
    k_items<<<grid_for(S_->nblk, 256), 256, 0, st>>>(S_->cell_start, S_->nblk, S_->items, S_->n_items);
    AQ_CUDA_TRY(cudaGetLastError());
    S_->cur = nxt;
    S_->launches += 6;
    S_->since_sort = 0;
    S_->sorted = true;
    return AQ_OK;
  }

  int launch_step(int do_g2p, int do_p2g, void* gin, void* gout, cudaStream_t st) {
    aq_sim* S_ = s;
    StepArgs a;
    a.words = S_->words[S_->cur];
    a.pid = S_->pid[S_->cur];
    a.items = S_->items;
    a.n_items = S_->n_items;
    a.grid_in = gin;
    a.grid_out = gout;
    a.status = S_->status;
    a.fallbacks = S_->fallbacks;
    a.rmax = S_->rmax;
    a.rmin = S_->rmin;
    a.sk = step_key(S_->P.seed, S_->step);
    a.do_g2p = do_g2p;
    a.do_p2g = do_p2g;
    a.ranges = S_->ranges_on;
    const bool prof = S_->prof_on && S_->prof_n[0] < aq_sim::PROF_CAP;
    if (prof) AQ_CUDA_TRY(cudaEventRecord(S_->prof_ev[0][2 * S_->prof_n[0]], st));
    k_step<D, HF, HM, R><<<S_->step_grid, CH, smem_bytes(), st>>>(S_->L, K, a);
    AQ_CUDA_TRY(cudaGetLastError());
    if (prof) AQ_CUDA_TRY(cudaEventRecord(S_->prof_ev[0][2 * S_->prof_n[0]++ + 1], st));
    S_->launches += 1;
    return AQ_OK;
  }

  int launch_grid(void* acc, void* clr, cudaStream_t st) {
    const bool prof = s->prof_on && s->prof_n[1] < aq_sim::PROF_CAP;
    if (prof) AQ_CUDA_TRY(cudaEventRecord(s->prof_ev[1][2 * s->prof_n[1]], st));
    k_grid<D, R><<<grid_for(s->ncell, 256), 256, 0, st>>>(K, acc, clr, s->ncell);
    AQ_CUDA_TRY(cudaGetLastError());
    if (prof) AQ_CUDA_TRY(cudaEventRecord(s->prof_ev[1][2 * s->prof_n[1]++ + 1], st));
    s->launches += 1;
    return AQ_OK;
  }

  int substeps(int n, cudaStream_t st) override {
    aq_sim* S_ = s;
    const int interval = S_->P.sort_interval < 1 ? 1 : S_->P.sort_interval;
    int rc;
    while (n > 0) {
      if (!S_->sorted || S_->since_sort >= interval) {
        if ((rc = sort(st))) return rc;
      }
      int m = interval - S_->since_sort;
      if (m > n) m = n;
      int a = S_->zero_grid;
      if ((rc = launch_step(0, 1, nullptr, S_->grid[a], st))) return rc;
      for (int k = 0; k < m; ++k) {
        const int b = 1 - a;
        if ((rc = launch_grid(S_->grid[a], S_->grid[b], st))) return rc;
        if (k + 1 < m) {
          if ((rc = launch_step(1, 1, S_->grid[a], S_->grid[b], st))) return rc;
          ++S_->step;
          a = b;
        } else {
          if ((rc = launch_step(1, 0, S_->grid[a], nullptr, st))) return rc;
          ++S_->step;
          S_->zero_grid = b;
        }
      }
      S_->since_sort += m;
      n -= m;
    }
    return AQ_OK;
  }

  int loss(double* h, cudaStream_t st) override {
    AQ_CUDA_TRY(cudaMemsetAsync(s->dloss, 0, sizeof(double), st));
    k_loss<D, R><<<num_sms() * 4, 256, 0, st>>>(s->L, K, s->words[s->cur], s->n, s->dloss);
    AQ_CUDA_TRY(cudaGetLastError());
    AQ_CUDA_TRY(cudaMemcpyAsync(h, s->dloss, sizeof(double), cudaMemcpyDeviceToHost, st));
    AQ_CUDA_TRY(cudaStreamSynchronize(st));
    return AQ_OK;
  }
};

template <int D, bool HF, bool HM, class R>
static int make_impl(aq_sim* s) {
  auto* im = new (std::nothrow) SimImpl<D, HF, HM, R>(s);
  if (!im) return AQ_E_NOMEM;
  s->impl = im;
  const size_t smem = im->smem_bytes();
  AQ_CUDA_TRY(cudaFuncSetAttribute(k_step<D, HF, HM, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  AQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_step<D, HF, HM, R>, CH, smem));
  if (occ < 1) occ = 1;
  s->step_grid = occ * num_sms();
  return AQ_OK;
}

template <int D, class R>
static int make_impl_d(aq_sim* s) {
  const bool hf = s->P.has_F != 0, hm = s->P.has_mat != 0;
  if (hf && hm) return make_impl<D, true, true, R>(s);
  if (hf) return make_impl<D, true, false, R>(s);
  if (hm) return make_impl<D, false, true, R>(s);
  return make_impl<D, false, false, R>(s);
}

static void free_sim(aq_sim* s) {
  if (!s) return;
  delete s->impl;
  for (int k = 0; k < 2; ++k) {
    if (s->prof_ev[k]) {
      for (int j = 0; j < 2 * aq_sim::PROF_CAP; ++j) cudaEventDestroy(s->prof_ev[k][j]);
      delete[] s->prof_ev[k];
    }
  }
  void* ptrs[] = {s->words[0], s->words[1], s->pid[0], s->pid[1], s->grid[0], s->grid[1], s->keys, s->ranks,
                  s->cell_count, s->cell_start, s->scan_sums, s->items, s->n_items, s->status, s->fallbacks,
                  s->rmax, s->rmin, s->dloss};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete s;
}

}  // namespace aq

using namespace aq;

extern "C" {

int aq_sim_create(const aq_params* P, const aq_layout* L, aq_sim** out) {
  if (!P || !L || !out) return AQ_E_ARG;
  *out = nullptr;
  const int D = P->dim;
  if (D != 2 && D != 3) return AQ_E_ARG;
  if (P->precision != 0 && P->precision != 1) return AQ_E_ARG;
  if (P->n_particles < 1 || P->n_particles > 0x7fffffffLL) return AQ_E_ARG;
  for (int d = 0; d < D; ++d)
    if (P->res[d] < 3 || P->res[d] > 8192) return AQ_E_ARG;
  if (!(P->dx > 0) || !(P->dt > 0)) return AQ_E_ARG;
  const int ns = 2 * D + D * D + (P->has_F ? D * D : 1) + (P->has_mat ? 1 : 0);
  if (L->n_slots != ns) return AQ_E_LAYOUT;
  if (P->n_materials < 0 || P->n_materials > AQ_MAX_MATERIALS) return AQ_E_ARG;
  for (int m = 0; m < (P->n_materials ? P->n_materials : 1); ++m) {
    const int k = P->mat[m].kind;
    if (k != AQ_MAT_FLUID && k != AQ_MAT_ELASTIC && k != AQ_MAT_COROTATED) return AQ_E_ARG;
    if (!P->has_F && k != AQ_MAT_FLUID) return AQ_E_LAYOUT;
  }

  aq_sim* s = new (std::nothrow) aq_sim();
  if (!s) return AQ_E_NOMEM;
  s->P = *P;
  s->L = *L;
  s->D = D;
  s->W = L->n_words;
  s->NS = ns;
  s->n = P->n_particles;
  int nb[3] = {1, 1, 1};
  const int BS = D == 3 ? 4 : 8;
  s->ncell = 1;
  for (int d = 0; d < D; ++d) {
    nb[d] = (P->res[d] + BS - 1) / BS;
    s->ncell *= P->res[d];
  }
  s->nblk = nb[0] * nb[1] * nb[2];
  s->nkeys = (int64_t)s->nblk * 64;
  s->max_items = s->n / CH + s->nblk + 1;
  const size_t rsz = P->precision ? sizeof(double) : sizeof(float);
  const int64_t n = s->n;
  const int nt = (int)((s->nkeys + SCAN_TILE - 1) / SCAN_TILE);
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes < 16 ? 16 : bytes);
  };
  alloc((void**)&s->words[0], sizeof(uint64_t) * (n * s->W + 2));
  alloc((void**)&s->words[1], sizeof(uint64_t) * (n * s->W + 2));
  alloc((void**)&s->pid[0], sizeof(int32_t) * n);
  alloc((void**)&s->pid[1], sizeof(int32_t) * n);
  alloc(&s->grid[0], rsz * 4 * s->ncell);
  alloc(&s->grid[1], rsz * 4 * s->ncell);
  alloc((void**)&s->keys, sizeof(int32_t) * n);
  alloc((void**)&s->ranks, sizeof(int32_t) * n);
  alloc((void**)&s->cell_count, sizeof(int32_t) * s->nkeys);
  alloc((void**)&s->cell_start, sizeof(int32_t) * (s->nkeys + 1));
  alloc((void**)&s->scan_sums, sizeof(int32_t) * (nt + 1));
  alloc((void**)&s->items, sizeof(int4) * s->max_items);
  alloc((void**)&s->n_items, sizeof(int32_t));
  alloc((void**)&s->status, sizeof(unsigned));
  alloc((void**)&s->fallbacks, sizeof(unsigned long long));
  alloc((void**)&s->rmax, sizeof(double) * AQ_MAX_SLOTS);
  alloc((void**)&s->rmin, sizeof(double) * AQ_MAX_SLOTS);
  alloc((void**)&s->dloss, sizeof(double));
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "cudaMalloc");
    free_sim(s);
    return AQ_E_NOMEM;
  }
  e = cudaMemset(s->grid[0], 0, rsz * 4 * s->ncell);
  if (e == cudaSuccess) e = cudaMemset(s->grid[1], 0, rsz * 4 * s->ncell);
  if (e == cudaSuccess) e = cudaMemset(s->words[0], 0, sizeof(uint64_t) * (n * s->W + 2));
  if (e == cudaSuccess) e = cudaMemset(s->status, 0, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(s->fallbacks, 0, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "cudaMemset");
    free_sim(s);
    return AQ_E_CUDA;
  }
  k_iota<<<grid_for(n, 256), 256>>>(s->pid[0], n);
  int rc;
  if (D == 3)
    rc = P->precision ? make_impl_d<3, double>(s) : make_impl_d<3, float>(s);
  else
    rc = P->precision ? make_impl_d<2, double>(s) : make_impl_d<2, float>(s);
  if (rc == AQ_OK && s->impl->smem_bytes() > 227 * 1024) rc = AQ_E_LIMIT;
  if (rc == AQ_OK) {
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      set_last_cuda_error(e, "aq_sim_create");
      rc = AQ_E_CUDA;
    }
  }
  if (rc != AQ_OK) {
    free_sim(s);
    return rc;
  }
  *out = s;
  return AQ_OK;
}

int aq_sim_destroy(aq_sim* s) {
  if (!s) return AQ_E_ARG;
  cudaDeviceSynchronize();
  free_sim(s);
  return AQ_OK;
}

int aq_sim_set_state(aq_sim* s, const void* values, int32_t values_f64, void* stream) {
  if (!s || !values) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  k_iota<<<grid_for(s->n, 256), 256, 0, st>>>(s->pid[s->cur], s->n);
  AQ_CUDA_TRY(cudaGetLastError());
  int rc = aq_encode(&s->L, values, values_f64, s->words[s->cur], s->n, nullptr, s->P.seed, -1, nullptr, stream);
  s->sorted = false;
  s->launches += 2;
  return rc;
}

int aq_sim_get_state(aq_sim* s, void* values, int32_t values_f64, void* stream) {
  if (!s || !values) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  if (values_f64)
    k_get_state<double><<<grid_for(s->n, 128), 128, 0, st>>>(s->L, s->words[s->cur], s->pid[s->cur], (double*)values,
                                                             s->n);
  else
    k_get_state<float><<<grid_for(s->n, 128), 128, 0, st>>>(s->L, s->words[s->cur], s->pid[s->cur], (float*)values,
                                                            s->n);
  AQ_CUDA_TRY(cudaGetLastError());
  s->launches += 1;
  return AQ_OK;
}

int aq_sim_set_words(aq_sim* s, const uint64_t* words, void* stream) {
  if (!s || !words) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  k_iota<<<grid_for(s->n, 256), 256, 0, st>>>(s->pid[s->cur], s->n);
  AQ_CUDA_TRY(cudaMemcpyAsync(s->words[s->cur], words, sizeof(uint64_t) * s->n * s->W, cudaMemcpyDeviceToDevice, st));
  s->sorted = false;
  s->launches += 1;
  return AQ_OK;
}

int aq_sim_get_words(aq_sim* s, uint64_t* words, void* stream) {
  if (!s || !words) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  k_words_permute<<<grid_for(s->n, 256), 256, 0, st>>>(s->words[s->cur], s->pid[s->cur], words, s->n, s->W, 1);
  AQ_CUDA_TRY(cudaGetLastError());
  s->launches += 1;
  return AQ_OK;
}

int aq_sim_substeps(aq_sim* s, int32_t n, void* stream) {
  if (!s || n < 0) return AQ_E_ARG;
  if (n == 0) return AQ_OK;
  return s->impl->substeps(n, as_stream(stream));
}

int aq_sim_loss(aq_sim* s, int32_t kind, double* h_out, void* stream) {
  if (!s || !h_out || kind != 0) return AQ_E_ARG;
  s->launches += 1;
  return s->impl->loss(h_out, as_stream(stream));
}

int aq_sim_ranges_enable(aq_sim* s, int32_t on, void* stream) {
  if (!s) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  if (on) {
    double mx[AQ_MAX_SLOTS], mn[AQ_MAX_SLOTS];
    for (int k = 0; k < AQ_MAX_SLOTS; ++k) {
      mx[k] = -INFINITY;
      mn[k] = INFINITY;
    }
    AQ_CUDA_TRY(cudaMemcpyAsync(s->rmax, mx, sizeof(mx), cudaMemcpyHostToDevice, st));
    AQ_CUDA_TRY(cudaMemcpyAsync(s->rmin, mn, sizeof(mn), cudaMemcpyHostToDevice, st));
    AQ_CUDA_TRY(cudaStreamSynchronize(st));
  }
  s->ranges_on = on ? 1 : 0;
  return AQ_OK;
}

int aq_sim_ranges_get(aq_sim* s, double* h_max, double* h_min, void* stream) {
  if (!s || !h_max || !h_min) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  AQ_CUDA_TRY(cudaMemcpyAsync(h_max, s->rmax, sizeof(double) * s->NS, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaMemcpyAsync(h_min, s->rmin, sizeof(double) * s->NS, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  return AQ_OK;
}

int aq_sim_status(aq_sim* s, uint32_t* h_flags, int64_t* h_fallbacks, int32_t clear, void* stream) {
  if (!s) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  unsigned f = 0;
  unsigned long long fb = 0;
  AQ_CUDA_TRY(cudaMemcpyAsync(&f, s->status, sizeof(f), cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaMemcpyAsync(&fb, s->fallbacks, sizeof(fb), cudaMemcpyDeviceToHost, st));
  if (clear) {
    AQ_CUDA_TRY(cudaMemsetAsync(s->status, 0, sizeof(unsigned), st));
    AQ_CUDA_TRY(cudaMemsetAsync(s->fallbacks, 0, sizeof(unsigned long long), st));
  }
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_flags) *h_flags = f;
  if (h_fallbacks) *h_fallbacks = (int64_t)fb;
  return AQ_OK;
}

int aq_sim_step_count(const aq_sim* s, int64_t* h_out) {
  if (!s || !h_out) return AQ_E_ARG;
  *h_out = s->step;
  return AQ_OK;
}

int aq_sim_launches(const aq_sim* s, int64_t* h_out) {
  if (!s || !h_out) return AQ_E_ARG;
  *h_out = s->launches;
  return AQ_OK;
}

int aq_sim_profile_enable(aq_sim* s, int32_t on) {
  if (!s) return AQ_E_ARG;
  if (on) {
    for (int k = 0; k < 2; ++k) {
      if (!s->prof_ev[k]) {
        s->prof_ev[k] = new (std::nothrow) cudaEvent_t[2 * aq_sim::PROF_CAP];
        if (!s->prof_ev[k]) return AQ_E_NOMEM;
        for (int j = 0; j < 2 * aq_sim::PROF_CAP; ++j) AQ_CUDA_TRY(cudaEventCreate(&s->prof_ev[k][j]));
      }
      s->prof_n[k] = 0;
    }
  }
  s->prof_on = on ? 1 : 0;
  return AQ_OK;
}

int aq_sim_profile_get(aq_sim* s, int32_t which, double* h_total_ms, int64_t* h_launches) {
  if (!s || which < 0 || which > 1 || !h_total_ms || !h_launches) return AQ_E_ARG;
  double tot = 0.0;
  const int n = s->prof_n[which];
  for (int j = 0; j < n; ++j) {
    AQ_CUDA_TRY(cudaEventSynchronize(s->prof_ev[which][2 * j + 1]));
    float ms = 0.f;
    AQ_CUDA_TRY(cudaEventElapsedTime(&ms, s->prof_ev[which][2 * j], s->prof_ev[which][2 * j + 1]));
    tot += ms;
  }
  s->prof_n[which] = 0;
  *h_total_ms = tot;
  *h_launches = n;
  return AQ_OK;
}

}  // extern "C"
