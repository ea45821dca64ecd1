// libaq.so: hand-written adjoint of the MLS-MPM substep with segment
// checkpointing, for the quantization sensitivities of the reference's
// autodiff pass (MPMSolver.run_forward_with_ad_nlogn, mpm_exps/engine/
// mpm_solver.py:1093-1302; Taichi's generated p2g.grad / grid_op.grad /
// g2p.grad, taichi_submission/taichi/transforms/auto_diff.cpp).
//
// State: n x NS unquantized values per particle in the record slot order
// x(d), v(d), C(d*d), F(d*d) | J; one material (fluid, or the reference's
// elastic law).  Forward substep s -> s' (same formulas as k_step):
//   P2G  m_i  = sum_p w_ip m,   P_i = sum_p w_ip (m v_p + A_p dpos_ip),
//        A_p = k sigma(F_p) + m C_p,  k = -dt p_vol 4/dx^2,
//        dpos_ip = x_i - x_p,  w_ip = prod_d N(x_pd/dx - i_d)
//   grid v_i = P_i / (m_i + 1e-10) - dt g e_y, then wall masks per component
//   G2P  v'_p = sum_i w_ip v_i,  C'_p = 4/dx^2 sum_i w_ip v_i dpos_ip^T,
//        x'_p = x_p + dt v'_p,  F'_p = (I + dt C'_p) F_p  (J'_p = (1+dt tr C'_p) J_p)
// Reverse (bars are adjoints), per substep:
//   G2P^T   Fbar += (I+dt C')^T F'bar;  C'bar += dt F'bar F^T;
//           v'bar += dt x'bar;  xbar += x'bar;
//           vbar_i += w v'bar + (4/dx^2) w C'bar dpos;
//           wbar_ip = v_i.v'bar + (4/dx^2) v_i^T C'bar dpos;
//           xbar -= (4/dx^2) w C'bar^T v_i  (through dpos);  xbar += wbar grad_x w
//   grid^T  masked components get no gradient; Pbar = vbar/(m+eps),
//           mbar = -vbar.P/(m+eps)^2
//   P2G^T   vbar += w m Pbar_i;  Abar += w Pbar_i dpos^T;
//           wbar = m mbar_i + Pbar_i.(m v + A dpos);  xbar -= w A^T Pbar_i;
//           xbar += wbar grad_x w;  Cbar += m Abar;  sigma_bar = k Abar;
//           Fbar += dsigma/dF^T sigma_bar  (fluid: Jbar += la tr(sigma_bar);
//           2D: fixed-corotated with the closed-form rotation derivative;
//           3D reference law: mu (sbar + sbar^T) F + la sum(sbar) F^-T)
// The derivative of the B-spline base index is zero almost everywhere.
//
// Sensitivities: sens[s] = sum over substeps t = 1..T-1 and particles of
// (dL/d state_t[s])^2 in f64, the quantity accu_grad accumulates
// (mpm_solver.py:1232-1271; the initial and the final state are not
// accumulated there either, :1190-1196).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <new>
#include <vector>

#include "aq_common.cuh"
#include "aq_kernels.cuh"

namespace aq {

template <class R>
struct AdK {
  int res[3], D, NS, HF, mat;
  R inv_dx, dx, dt, p_mass, kst, four_inv_dx2, grav, mu, lam;
  double lb[3], ub[3];
  int bound_clip, friction;
  R clip_lo[3], clip_hi[3];
  // rotating SDF collider (3D; col_on = 0: none), the fields collider_at
  // reads; col_c, col_s, col_yshift are this substep's angle and height
  int col_on, col_n, col_dims[3], col_off[3], col_lo[3], col_hi[3];
  const float* col_sdf;
  const float* col_nrm;
  R col_omega, col_c, col_s;
  int col_yshift;
};

template <int D>
__device__ __forceinline__ int64_t ad_cell(const int (&res)[3], const int* I) {
  return D == 3 ? ((int64_t)I[0] * res[1] + I[1]) * res[2] + I[2] : (int64_t)I[0] * res[1] + I[1];
}

template <int D, class R>
__device__ __forceinline__ void ad_weights(const R* x, const AdK<R>& K, int* base, R* fx, R (&w)[3][3],
                                           R (&dw)[3][3]) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    R t = x[d] * K.inv_dx - (R)0.5;
    int b = (int)floor(t);
    b = min(max(b, 0), K.res[d] - 3);
    base[d] = b;
    fx[d] = x[d] * K.inv_dx - (R)b;
    w[0][d] = (R)0.5 * ((R)1.5 - fx[d]) * ((R)1.5 - fx[d]);
    w[1][d] = (R)0.75 - (fx[d] - (R)1) * (fx[d] - (R)1);
    w[2][d] = (R)0.5 * (fx[d] - (R)0.5) * (fx[d] - (R)0.5);
    // dN/dx (per unit x: chain with inv_dx)
    dw[0][d] = -((R)1.5 - fx[d]) * K.inv_dx;
    dw[1][d] = (R)-2 * (fx[d] - (R)1) * K.inv_dx;
    dw[2][d] = (fx[d] - (R)0.5) * K.inv_dx;
  }
}

template <int D, class R>
__device__ __forceinline__ R inv_det_cof(const R* F, R* cof) {  // cofactor matrix (dJ/dF) and J
  if (D == 2) {
    cof[0] = F[3];
    cof[1] = -F[2];
    cof[2] = -F[1];
    cof[3] = F[0];
    return F[0] * F[3] - F[1] * F[2];
  }
  cof[0] = F[4] * F[8] - F[5] * F[7];
  cof[1] = F[5] * F[6] - F[3] * F[8];
  cof[2] = F[3] * F[7] - F[4] * F[6];
  cof[3] = F[2] * F[7] - F[1] * F[8];
  cof[4] = F[0] * F[8] - F[2] * F[6];
  cof[5] = F[1] * F[6] - F[0] * F[7];
  cof[6] = F[1] * F[5] - F[2] * F[4];
  cof[7] = F[2] * F[3] - F[0] * F[5];
  cof[8] = F[0] * F[4] - F[1] * F[3];
  return F[0] * cof[0] + F[1] * cof[1] + F[2] * cof[2];
}

// stress sigma(F) of the reference materials
template <int D, bool HF, class R>
__device__ __forceinline__ void ad_sigma(const AdK<R>& K, const R* s, R* sig) {
  typedef Sch<D, HF, false> S;
#pragma unroll
  for (int k = 0; k < D * D; ++k) sig[k] = 0;
  if (!HF) {
#pragma unroll
    for (int d = 0; d < D; ++d) sig[d * D + d] = K.lam * (s[S::FJ] - (R)1);
    return;
  }
  const R* F = s + S::FJ;
  R cof[9];
  const R J = inv_det_cof<D, R>(F, cof);
  if (K.mat == AQ_MAT_FLUID) {
#pragma unroll
    for (int d = 0; d < D; ++d) sig[d * D + d] = K.lam * (J - (R)1);
    return;
  }
  if (D == 2) {
    R Rm[4];
    polar_rot<2, R>(F, Rm);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        R a = 0;
#pragma unroll
        for (int k = 0; k < 2; ++k) a += (F[i * 2 + k] - Rm[i * 2 + k]) * F[j * 2 + k];
        sig[i * 2 + j] = (R)2 * K.mu * a + (i == j ? K.lam * J * (J - (R)1) : (R)0);
      }
  } else {
    const R lj = K.lam * log(J);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        R a = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) a += F[i * 3 + k] * F[j * 3 + k];
        sig[i * 3 + j] = K.mu * (a - (i == j ? (R)1 : (R)0)) + lj;
      }
  }
}

// Fbar (or Jbar) += dsigma/dF^T sbar
template <int D, bool HF, class R>
__device__ __forceinline__ void ad_sigma_bwd(const AdK<R>& K, const R* s, const R* sb, R* gb) {
  typedef Sch<D, HF, false> S;
  R tr = 0, sum = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) tr += sb[d * D + d];
#pragma unroll
  for (int k = 0; k < D * D; ++k) sum += sb[k];
  if (!HF) {
    gb[S::FJ] += K.lam * tr;
    return;
  }
  const R* F = s + S::FJ;
  R* Fb = gb + S::FJ;
  R cof[9];
  const R J = inv_det_cof<D, R>(F, cof);
  if (K.mat == AQ_MAT_FLUID) {
#pragma unroll
    for (int k = 0; k < D * D; ++k) Fb[k] += K.lam * tr * cof[k];
    return;
  }
  if (D == 2) {
    // sigma = 2 mu (F - R) F^T + la J (J-1) I,  R = [[c,-s],[s,c]]
    R Rm[4];
    polar_rot<2, R>(F, Rm);
    R G[4], Gb[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) G[k] = F[k] - Rm[k];
    // Gbar = 2 mu sbar F ; Fbar += 2 mu sbar^T G
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        R a = 0, b = 0;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          a += sb[i * 2 + k] * F[k * 2 + j];
          b += sb[k * 2 + i] * G[k * 2 + j];
        }
        Gb[i * 2 + j] = (R)2 * K.mu * a;
        Fb[i * 2 + j] += (R)2 * K.mu * b + Gb[i * 2 + j];
      }
    const R Jb = K.lam * ((R)2 * J - (R)1) * tr;
#pragma unroll
    for (int k = 0; k < 4; ++k) Fb[k] += Jb * cof[k];
    // Rbar = -Gbar ; c = x/r, s = y/r with x = F00+F11, y = F10-F01
    const R cb = -(Gb[0] + Gb[3]);
    const R sbb = -(-Gb[1] + Gb[2]);
    const R x = F[0] + F[3], y = F[2] - F[1];
    const R r2 = x * x + y * y, r = sqrt(r2), r3 = r2 * r;
    const R xb = (cb * y * y - sbb * x * y) / r3;
    const R yb = (-cb * x * y + sbb * x * x) / r3;
    Fb[0] += xb;
    Fb[3] += xb;
    Fb[2] += yb;
    Fb[1] -= yb;
  } else {
    // sigma = mu (F F^T - I) + la log J (every entry)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        R a = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) a += (sb[i * 3 + k] + sb[k * 3 + i]) * F[k * 3 + j];
        Fb[i * 3 + j] += K.mu * a + K.lam * sum * cof[i * 3 + j] / J;
      }
  }
}

template <int D>
__device__ __forceinline__ void offs(int o, int* off) {
  off[0] = D == 3 ? o / 9 : o / 3;
  off[1] = D == 3 ? (o / 3) % 3 : o % 3;
  off[2] = D == 3 ? o % 3 : 0;
}

// ------------------------------------------------------------- forward

// Runs of equal keys over consecutive lanes of a warp.  The state is sorted
// by base cell, so a run holds the warp's particles of one cell, which add
// into the same 3^D nodes: run_sum adds a value over the lane's run in
// log2(longest run) shuffle steps, and the run's first lane makes the one
// global atomic for the whole run instead of one per particle.
struct WarpRuns {
  int lane, end, steps;  // end: last lane of this lane's run
  bool head;             // this lane starts its run
};

__device__ __forceinline__ WarpRuns warp_runs(long long key) {
  WarpRuns r;
  r.lane = threadIdx.x & 31;
  const long long prev = __shfl_up_sync(0xffffffffu, key, 1);
  r.head = r.lane == 0 || prev != key;
  const unsigned starts = __ballot_sync(0xffffffffu, r.head);
  const unsigned later = r.lane == 31 ? 0u : (starts & (0xffffffffu << (r.lane + 1)));
  r.end = later ? __ffs(later) - 2 : 31;
  const int len = r.head ? r.end - r.lane + 1 : 1;
  const int maxlen = (int)__reduce_max_sync(0xffffffffu, (unsigned)len);
  int steps = 0;
  while ((1 << steps) < maxlen) ++steps;
  r.steps = steps;
  return r;
}

// After the call the run's first lane holds the sum of v over the run.
template <class R>
__device__ __forceinline__ R run_sum(R v, const WarpRuns& r) {
  for (int k = 0; k < r.steps; ++k) {
    const int d = 1 << k;
    const R o = __shfl_down_sync(0xffffffffu, v, d);
    if (r.lane + d <= r.end) v += o;
  }
  return v;
}

template <int D, bool HF, class R>
__global__ void __launch_bounds__(128) k_ad_p2g(const AdK<R> K, const R* __restrict__ st, int64_t n,
                                                R* __restrict__ grid) {
  typedef Sch<D, HF, false> S;
  const int64_t p0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = p0 < n;
  if (__all_sync(0xffffffffu, !active)) return;
  const int64_t p = active ? p0 : n - 1;  // lanes past the end take part in the shuffles only
  const R* s = st + p * K.NS;
  int base[3];
  R fx[3], w[3][3], dw[3][3];
  ad_weights<D, R>(s + S::X, K, base, fx, w, dw);
  R sig[9], A[9];
  ad_sigma<D, HF, R>(K, s, sig);
#pragma unroll
  for (int k = 0; k < D * D; ++k) A[k] = K.kst * sig[k] + K.p_mass * s[S::C + k];
  const WarpRuns runs = warp_runs(active ? (long long)ad_cell<D>(K.res, base) : -1 - (long long)(threadIdx.x & 31));
  const R on = active ? (R)1 : (R)0;
  for (int o = 0; o < (D == 3 ? 27 : 9); ++o) {
    int off[3], I[3];
    offs<D>(o, off);
    R wt = on, dpos[3];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      wt *= w[off[d]][d];
      dpos[d] = ((R)off[d] - fx[d]) * K.dx;
      I[d] = base[d] + off[d];
    }
    R val[4];
    val[0] = run_sum(wt * K.p_mass, runs);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      R a = K.p_mass * s[S::V + d];
#pragma unroll
      for (int e = 0; e < D; ++e) a += A[d * D + e] * dpos[e];
      val[1 + d] = run_sum(wt * a, runs);
    }
    if (active && runs.head) {
      R* g = grid + 4 * ad_cell<D>(K.res, I);
#pragma unroll
      for (int k = 0; k < 1 + D; ++k) atomicAdd(g + k, val[k]);
    }
  }
}

// wall mask of component k at node I given the velocity sign (grid_op)
template <class R>
__device__ __forceinline__ bool ad_wall(const AdK<R>& K, const int* I, int k, R vk) {
  return (I[k] < K.lb[k] && vk < (R)0) || (I[k] > K.ub[k] && vk > (R)0);
}

template <int D, class R>
__global__ void __launch_bounds__(256) k_ad_grid(const AdK<R> K, const R* __restrict__ grid, R* __restrict__ gv,
                                                 int64_t ncell) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int I[3] = {0, 0, 0};
  if (D == 3) {
    I[2] = (int)(c % K.res[2]);
    I[1] = (int)((c / K.res[2]) % K.res[1]);
    I[0] = (int)(c / ((int64_t)K.res[2] * K.res[1]));
  } else {
    I[1] = (int)(c % K.res[1]);
    I[0] = (int)(c / K.res[1]);
  }
  const R* g = grid + 4 * c;
  const R inv_m = (R)1 / (g[0] + (R)1e-10);
  R v[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) v[d] = inv_m * g[1 + d];
  v[1] -= K.dt * K.grav;
#pragma unroll
  for (int k = 0; k < D; ++k)
    if (ad_wall<R>(K, I, k, v[k])) v[k] = 0;
  if (D == 3 && K.col_on) collide_node<R, true>(K, I[0], I[1], I[2], v);  // sdf_collision_no_arg
#pragma unroll
  for (int d = 0; d < 3; ++d) gv[4 * c + d] = d < D ? v[d] : (R)0;
  gv[4 * c + 3] = 0;
}

template <int D, bool HF, class R>
__global__ void __launch_bounds__(128) k_ad_g2p(const AdK<R> K, const R* __restrict__ st, const R* __restrict__ gv,
                                                R* __restrict__ out, int64_t n) {
  typedef Sch<D, HF, false> S;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const R* s = st + p * K.NS;
  R* so = out + p * K.NS;
  int base[3];
  R fx[3], w[3][3], dw[3][3];
  ad_weights<D, R>(s + S::X, K, base, fx, w, dw);
  R nv[3] = {0, 0, 0}, nC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int o = 0; o < (D == 3 ? 27 : 9); ++o) {
    int off[3], I[3];
    offs<D>(o, off);
    R wt = 1, dpos[3];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      wt *= w[off[d]][d];
      dpos[d] = ((R)off[d] - fx[d]) * K.dx;
      I[d] = base[d] + off[d];
    }
    const R* g = gv + 4 * ad_cell<D>(K.res, I);
#pragma unroll
    for (int d = 0; d < D; ++d) {
      nv[d] += wt * g[d];
#pragma unroll
      for (int e = 0; e < D; ++e) nC[d * D + e] += K.four_inv_dx2 * wt * g[d] * dpos[e];
    }
  }
#pragma unroll
  for (int d = 0; d < D; ++d) {
    so[S::X + d] = s[S::X + d] + K.dt * nv[d];
    so[S::V + d] = nv[d];
  }
#pragma unroll
  for (int k = 0; k < D * D; ++k) so[S::C + k] = nC[k];
  if (HF) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R a = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) a += ((i == k ? (R)1 : (R)0) + K.dt * nC[i * D + k]) * s[S::FJ + k * D + j];
        so[S::FJ + i * D + j] = a;
      }
  } else {
    R tr = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) tr += nC[d * D + d];
    so[S::FJ] = ((R)1 + K.dt * tr) * s[S::FJ];
  }
}

// ------------------------------------------------------------- reverse

// G2P^T: from the adjoint of the new state (ab_out) to the adjoint of the
// old state's x and F|J (ab_in, overwritten) and the grid velocity adjoint
// (gvb, accumulated).
template <int D, bool HF, class R>
__global__ void __launch_bounds__(128) k_ad_g2p_bwd(const AdK<R> K, const R* __restrict__ st,
                                                    const R* __restrict__ gv, const R* __restrict__ ab_out,
                                                    R* __restrict__ ab_in, R* __restrict__ gvb, int64_t n) {
  typedef Sch<D, HF, false> S;
  const int64_t p0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = p0 < n;
  if (__all_sync(0xffffffffu, !active)) return;
  const int64_t p = active ? p0 : n - 1;  // lanes past the end take part in the shuffles only
  const R* s = st + p * K.NS;
  const R* bo = ab_out + p * K.NS;
  R* bi = ab_in + p * K.NS;
  int base[3];
  R fx[3], w[3][3], dw[3][3];
  ad_weights<D, R>(s + S::X, K, base, fx, w, dw);
  const WarpRuns runs = warp_runs(active ? (long long)ad_cell<D>(K.res, base) : -1 - (long long)(threadIdx.x & 31));
  // recompute new C (needed for F' = (I + dt C') F)
  R nC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int o = 0; o < (D == 3 ? 27 : 9); ++o) {
    int off[3], I[3];
    offs<D>(o, off);
    R wt = 1, dpos[3];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      wt *= w[off[d]][d];
      dpos[d] = ((R)off[d] - fx[d]) * K.dx;
      I[d] = base[d] + off[d];
    }
    const R* g = gv + 4 * ad_cell<D>(K.res, I);
#pragma unroll
    for (int d = 0; d < D; ++d)
#pragma unroll
      for (int e = 0; e < D; ++e) nC[d * D + e] += K.four_inv_dx2 * wt * g[d] * dpos[e];
  }
  R xb[3] = {0, 0, 0}, vpb[3] = {0, 0, 0}, Cpb[9];
#pragma unroll
  for (int k = 0; k < D * D; ++k) Cpb[k] = bo[S::C + k];
  R FJb[9];
  if (HF) {
    // F' = (I + dt C') F
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R a = 0, c = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
          a += ((k == i ? (R)1 : (R)0) + K.dt * nC[k * D + i]) * bo[S::FJ + k * D + j];  // (I+dtC')^T F'bar
          c += bo[S::FJ + i * D + k] * s[S::FJ + j * D + k];                            // F'bar F^T
        }
        FJb[i * D + j] = a;
        Cpb[i * D + j] += K.dt * c;
      }
  } else {
    R tr = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) tr += nC[d * D + d];
    FJb[0] = ((R)1 + K.dt * tr) * bo[S::FJ];
    const R trb = K.dt * s[S::FJ] * bo[S::FJ];
#pragma unroll
    for (int d = 0; d < D; ++d) Cpb[d * D + d] += trb;
  }
#pragma unroll
  for (int d = 0; d < D; ++d) {
    xb[d] = bo[S::X + d];
    vpb[d] = bo[S::V + d] + K.dt * bo[S::X + d];
  }
  for (int o = 0; o < (D == 3 ? 27 : 9); ++o) {
    int off[3], I[3];
    offs<D>(o, off);
    R wt = 1, dpos[3];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      wt *= w[off[d]][d];
      dpos[d] = ((R)off[d] - fx[d]) * K.dx;
      I[d] = base[d] + off[d];
    }
    const int64_t cell = ad_cell<D>(K.res, I);
    const R* g = gv + 4 * cell;
    R wb = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      R cd = 0;  // (C'bar dpos)_d
#pragma unroll
      for (int e = 0; e < D; ++e) cd += Cpb[d * D + e] * dpos[e];
      const R vb = run_sum(active ? wt * (vpb[d] + K.four_inv_dx2 * cd) : (R)0, runs);
      if (active && runs.head) atomicAdd(gvb + 4 * cell + d, vb);
      wb += g[d] * (vpb[d] + K.four_inv_dx2 * cd);
    }
    // through dpos = x_i - x_p: xbar -= 4/dx^2 w C'bar^T v_i
#pragma unroll
    for (int e = 0; e < D; ++e) {
      R a = 0;
#pragma unroll
      for (int d = 0; d < D; ++d) a += Cpb[d * D + e] * g[d];
      xb[e] -= K.four_inv_dx2 * wt * a;
    }
    // through w
#pragma unroll
    for (int d = 0; d < D; ++d) {
      R gw = dw[off[d]][d];
#pragma unroll
      for (int e = 0; e < D; ++e)
        if (e != d) gw *= w[off[e]][e];
      xb[d] += wb * gw;
    }
  }
  if (!active) return;
  for (int k = 0; k < K.NS; ++k) bi[k] = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) bi[S::X + d] = xb[d];
  if (HF) {
#pragma unroll
    for (int k = 0; k < D * D; ++k) bi[S::FJ + k] = FJb[k];
  } else {
    bi[S::FJ] = FJb[0];
  }
}

// grid^T: from the velocity adjoint to the (m, P) adjoint, in place in gvb
template <int D, class R>
__global__ void __launch_bounds__(256) k_ad_grid_bwd(const AdK<R> K, const R* __restrict__ grid,
                                                     R* __restrict__ gvb, int64_t ncell) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int I[3] = {0, 0, 0};
  if (D == 3) {
    I[2] = (int)(c % K.res[2]);
    I[1] = (int)((c / K.res[2]) % K.res[1]);
    I[0] = (int)(c / ((int64_t)K.res[2] * K.res[1]));
  } else {
    I[1] = (int)(c % K.res[1]);
    I[0] = (int)(c / K.res[1]);
  }
  const R* g = grid + 4 * c;
  const R me = g[0] + (R)1e-10;
  const R inv_m = (R)1 / me;
  R v[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) v[d] = inv_m * g[1 + d];
  v[1] -= K.dt * K.grav;
  R vb[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) vb[d] = gvb[4 * c + d];
  if (D == 3 && K.col_on) {
    // collider^T: where the node is inside and moving into the surface
    // (relative to the collider), the forward removed the normal part of
    // the velocity, v' = v - ((v - cv).n) n, so vbar' = vbar - (vbar.n) n
    R nrm[3], cv[3];
    if (collider_at<R, true>(K, I[0], I[1], I[2], nrm, cv)) {
      R dn = 0, bn = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const R vw = ad_wall<R>(K, I, k, v[k]) ? (R)0 : v[k];  // the collider's input
        dn += (vw - cv[k]) * nrm[k];
        bn += vb[k] * nrm[k];
      }
      if (dn < (R)0)
#pragma unroll
        for (int k = 0; k < 3; ++k) vb[k] -= bn * nrm[k];
    }
  }
  R mb = 0, Pb[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) {
    R b = vb[d];
    if (ad_wall<R>(K, I, d, v[d])) b = 0;
    Pb[d] = b * inv_m;
    mb -= b * g[1 + d] * inv_m * inv_m;
  }
  gvb[4 * c + 0] = mb;
#pragma unroll
  for (int d = 0; d < 3; ++d) gvb[4 * c + 1 + d] = d < D ? Pb[d] : (R)0;
}

// P2G^T: adds the old-state adjoint through P2G into ab_in
template <int D, bool HF, class R>
__global__ void __launch_bounds__(128) k_ad_p2g_bwd(const AdK<R> K, const R* __restrict__ st,
                                                    const R* __restrict__ gb, R* __restrict__ ab_in, int64_t n) {
  typedef Sch<D, HF, false> S;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const R* s = st + p * K.NS;
  R* bi = ab_in + p * K.NS;
  int base[3];
  R fx[3], w[3][3], dw[3][3];
  ad_weights<D, R>(s + S::X, K, base, fx, w, dw);
  R sig[9], A[9];
  ad_sigma<D, HF, R>(K, s, sig);
#pragma unroll
  for (int k = 0; k < D * D; ++k) A[k] = K.kst * sig[k] + K.p_mass * s[S::C + k];
  R xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0}, Ab[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int o = 0; o < (D == 3 ? 27 : 9); ++o) {
    int off[3], I[3];
    offs<D>(o, off);
    R wt = 1, dpos[3];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      wt *= w[off[d]][d];
      dpos[d] = ((R)off[d] - fx[d]) * K.dx;
      I[d] = base[d] + off[d];
    }
    const R* g = gb + 4 * ad_cell<D>(K.res, I);
    const R mb = g[0];
    R wb = K.p_mass * mb;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const R Pb = g[1 + d];
      R a = K.p_mass * s[S::V + d];
#pragma unroll
      for (int e = 0; e < D; ++e) a += A[d * D + e] * dpos[e];
      wb += Pb * a;
      vb[d] += wt * K.p_mass * Pb;
#pragma unroll
      for (int e = 0; e < D; ++e) {
        Ab[d * D + e] += wt * Pb * dpos[e];
        xb[e] -= wt * A[d * D + e] * Pb;  // through dpos = x_i - x_p
      }
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
      R gw = dw[off[d]][d];
#pragma unroll
      for (int e = 0; e < D; ++e)
        if (e != d) gw *= w[off[e]][e];
      xb[d] += wb * gw;
    }
  }
  R sb[9];
#pragma unroll
  for (int k = 0; k < D * D; ++k) {
    bi[S::C + k] += K.p_mass * Ab[k];
    sb[k] = K.kst * Ab[k];
  }
#pragma unroll
  for (int d = 0; d < D; ++d) {
    bi[S::X + d] += xb[d];
    bi[S::V + d] += vb[d];
  }
  ad_sigma_bwd<D, HF, R>(K, s, sb, bi);
}

template <class R>
__global__ void k_ad_accum(const R* __restrict__ ab, int64_t n, int ns, double* __restrict__ sens) {
  extern __shared__ double shs[];
  for (int s = threadIdx.x; s < ns; s += blockDim.x) shs[s] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * ns; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = (double)ab[i];
    atomicAdd(&shs[i % ns], v * v);
  }
  __syncthreads();
  for (int s = threadIdx.x; s < ns; s += blockDim.x) atomicAdd(&sens[s], shs[s]);
}

// Particle order for locality: the key of a particle is its base cell
// (row-major), clamped to the grid; sorting the state by it once per forward
// pass puts the particles a warp scatters from and gathers into next to
// each other on the grid (they move little over an adjoint horizon).
template <class R>
__global__ void k_ad_keys(const R* __restrict__ st, int64_t n, int ns, int D, int r0, int r1, int r2, R inv_dx,
                          int32_t* __restrict__ keys, int32_t* __restrict__ idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int res[3] = {r0, r1, r2};
  int64_t key = 0;
  for (int d = 0; d < D; ++d) {
    const R t = st[i * ns + d] * inv_dx - (R)0.5;
    int b = t == t ? (int)floor(t) : 0;
    b = min(max(b, 0), res[d] - 1);
    key = key * res[d] + b;
  }
  keys[i] = (int32_t)key;
  idx[i] = (int32_t)i;
}

// rows of a state: out[i] = in[perm[i]] (gather) or out[perm[i]] = in[i]
template <class R>
__global__ void k_ad_permute(const R* __restrict__ in, R* __restrict__ out, const int32_t* __restrict__ perm, int64_t n,
                             int ns, int gather) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * ns) return;
  const int64_t i = k / ns, s = k - i * ns;
  const int64_t j = perm[i];
  if (gather)
    out[i * ns + s] = in[j * ns + s];
  else
    out[j * ns + s] = in[i * ns + s];
}

// --------------------------------------------------------------- host

struct AdBase {
  virtual ~AdBase() {}
  // t: index of the substep (the collider's angle and height depend on it)
  virtual int step(const void* in, void* out, int t, cudaStream_t st) = 0;
  virtual int step_bwd(const void* s_in, const void* ab_out, void* ab_in, int t, cudaStream_t st) = 0;
  virtual int accum(const void* ab, double* sens, cudaStream_t st) = 0;
  virtual int sort_keys(const void* s0, int32_t* keys, int32_t* idx, cudaStream_t st) = 0;
  virtual int permute(const void* in, void* out, bool gather, cudaStream_t st) = 0;
};

}  // namespace aq

struct aq_adjoint {
  aq_params P;
  int D = 0, NS = 0;
  int64_t n = 0, ncell = 0;
  size_t rsz = 4;
  void* grid = nullptr;  // (m, P) per node
  void* gv = nullptr;    // grid velocity per node
  void* gvb = nullptr;   // velocity adjoint, then (m, P) adjoint
  std::vector<void*> ckpt;  // states at multiples of the checkpoint interval (every > 0), or the initial state
  std::vector<void*> seg;   // states of one segment (recomputed); two ping-pong states (every == 0)
  std::vector<void*> stash;  // bisection checkpointing: one state per recursion level, plus a scratch state
  int T = 0, every = 0;
  int32_t* perm = nullptr;  // sorted position -> caller's particle index (length n)
  int64_t recomputed = 0;   // forward substeps run again by the last backward pass
  double* dsens = nullptr;
  aq::AdBase* impl = nullptr;
  // SDF collider (aq_adjoint_set_collider): caller-owned volumes; at
  // substep t the angle is theta + omega dt t and the height
  // height + rate dt t (step_collider_difftaichi, mpm_solver.py:1554-1559)
  int col_on = 0, col_center = 0, col_dims[3] = {0, 0, 0}, col_off[3] = {0, 0, 0};
  const float* col_sdf = nullptr;
  const float* col_nrm = nullptr;
  double col_theta = 0, col_height = 0, col_omega = 0, col_rate = 0;
};

namespace aq {

template <int D, bool HF, class R>
struct AdImpl final : AdBase {
  aq_adjoint* a;
  AdK<R> K;
  explicit AdImpl(aq_adjoint* adj) : a(adj) {
    const aq_params& P = adj->P;
    memset(&K, 0, sizeof(K));
    for (int d = 0; d < 3; ++d) {
      K.res[d] = d < D ? P.res[d] : 1;
      K.lb[d] = P.lb[d];
      K.ub[d] = P.ub[d];
    }
    K.D = D;
    K.NS = adj->NS;
    K.HF = HF;
    K.mat = P.mat[0].kind;
    K.inv_dx = (R)(1.0 / P.dx);
    K.dx = (R)P.dx;
    K.dt = (R)P.dt;
    K.p_mass = (R)P.p_mass;
    K.kst = (R)(-(P.dt * P.p_vol * 4.0 * (1.0 / P.dx) * (1.0 / P.dx)));
    K.four_inv_dx2 = (R)(4.0 / (P.dx * P.dx));
    K.grav = (R)P.gravity;
    K.mu = (R)P.mat[0].mu;
    K.lam = (R)P.mat[0].lam;
  }
  void set_substep(int t) {
    K.col_on = a->col_on;
    if (!K.col_on) return;
    K.col_n = a->col_center;
    for (int d = 0; d < 3; ++d) {
      K.col_dims[d] = a->col_dims[d];
      K.col_off[d] = a->col_off[d];
      K.col_lo[d] = (int)a->P.lb[d];
      K.col_hi[d] = (int)a->P.ub[d];
    }
    K.col_sdf = a->col_sdf;
    K.col_nrm = a->col_nrm;
    K.col_omega = (R)a->col_omega;
    const double th = a->col_theta + a->col_omega * a->P.dt * t;
    const double h = a->col_height + a->col_rate * a->P.dt * t;
    K.col_c = (R)cos(th);
    K.col_s = (R)sin(th);
    K.col_yshift = (int)(h / a->P.dx + 0.5);
  }
  int step(const void* in, void* out, int t, cudaStream_t st) override {
    set_substep(t);
    const size_t gbytes = sizeof(R) * 4 * a->ncell;
    AQ_CUDA_TRY(cudaMemsetAsync(a->grid, 0, gbytes, st));
    k_ad_p2g<D, HF, R><<<grid_for(a->n, 128), 128, 0, st>>>(K, (const R*)in, a->n, (R*)a->grid);
    k_ad_grid<D, R><<<grid_for(a->ncell, 256), 256, 0, st>>>(K, (const R*)a->grid, (R*)a->gv, a->ncell);
    k_ad_g2p<D, HF, R><<<grid_for(a->n, 128), 128, 0, st>>>(K, (const R*)in, (const R*)a->gv, (R*)out, a->n);
    AQ_CUDA_TRY(cudaGetLastError());
    return AQ_OK;
  }
  int step_bwd(const void* s_in, const void* ab_out, void* ab_in, int t, cudaStream_t st) override {
    set_substep(t);
    const size_t gbytes = sizeof(R) * 4 * a->ncell;
    // recompute the grid of this substep
    AQ_CUDA_TRY(cudaMemsetAsync(a->grid, 0, gbytes, st));
    k_ad_p2g<D, HF, R><<<grid_for(a->n, 128), 128, 0, st>>>(K, (const R*)s_in, a->n, (R*)a->grid);
    k_ad_grid<D, R><<<grid_for(a->ncell, 256), 256, 0, st>>>(K, (const R*)a->grid, (R*)a->gv, a->ncell);
    AQ_CUDA_TRY(cudaMemsetAsync(a->gvb, 0, gbytes, st));
    k_ad_g2p_bwd<D, HF, R><<<grid_for(a->n, 128), 128, 0, st>>>(K, (const R*)s_in, (const R*)a->gv,
                                                                 (const R*)ab_out, (R*)ab_in, (R*)a->gvb, a->n);
    k_ad_grid_bwd<D, R><<<grid_for(a->ncell, 256), 256, 0, st>>>(K, (const R*)a->grid, (R*)a->gvb, a->ncell);
    k_ad_p2g_bwd<D, HF, R><<<grid_for(a->n, 128), 128, 0, st>>>(K, (const R*)s_in, (const R*)a->gvb, (R*)ab_in,
                                                                 a->n);
    AQ_CUDA_TRY(cudaGetLastError());
    return AQ_OK;
  }
  int accum(const void* ab, double* sens, cudaStream_t st) override {
    k_ad_accum<R><<<num_sms() * 2, 256, sizeof(double) * a->NS, st>>>((const R*)ab, a->n, a->NS, sens);
    AQ_CUDA_TRY(cudaGetLastError());
    return AQ_OK;
  }
  int sort_keys(const void* s0, int32_t* keys, int32_t* idx, cudaStream_t st) override {
    k_ad_keys<R><<<grid_for(a->n, 256), 256, 0, st>>>((const R*)s0, a->n, a->NS, D, K.res[0], K.res[1], K.res[2],
                                                      K.inv_dx, keys, idx);
    AQ_CUDA_TRY(cudaGetLastError());
    return AQ_OK;
  }
  int permute(const void* in, void* out, bool gather, cudaStream_t st) override {
    k_ad_permute<R><<<grid_for(a->n * a->NS, 256), 256, 0, st>>>((const R*)in, (R*)out, a->perm, a->n, a->NS,
                                                                 gather ? 1 : 0);
    AQ_CUDA_TRY(cudaGetLastError());
    return AQ_OK;
  }
};

// Sort the particles by base cell: a->perm[sorted position] = caller's index.
static int ad_make_perm(aq_adjoint* a, const void* d_s0, cudaStream_t st) {
  if (!a->perm) AQ_CUDA_TRY(cudaMalloc((void**)&a->perm, sizeof(int32_t) * a->n));
  int32_t* tmp = nullptr;  // keys in, keys out, idx in
  AQ_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(int32_t) * 3 * a->n, st));
  int32_t *kin = tmp, *kout = tmp + a->n, *iin = tmp + 2 * a->n;
  int rc = a->impl->sort_keys(d_s0, kin, iin, st);
  int bits = 1;
  while (bits < 31 && (int64_t(1) << bits) < a->ncell) ++bits;
  size_t tb = 0;
  // keys are non-negative: sorted as unsigned over their low `bits` bits
  uint32_t *uk = reinterpret_cast<uint32_t*>(kin), *uo = reinterpret_cast<uint32_t*>(kout);
  if (rc == AQ_OK &&
      cub::DeviceRadixSort::SortPairs(nullptr, tb, uk, uo, iin, a->perm, (int)a->n, 0, bits, st) != cudaSuccess)
    rc = AQ_E_CUDA;
  void* temp = nullptr;
  if (rc == AQ_OK && cudaMallocAsync(&temp, tb ? tb : 1, st) != cudaSuccess) rc = AQ_E_NOMEM;
  if (rc == AQ_OK &&
      cub::DeviceRadixSort::SortPairs(temp, tb, uk, uo, iin, a->perm, (int)a->n, 0, bits, st) != cudaSuccess)
    rc = AQ_E_CUDA;
  if (temp) cudaFreeAsync(temp, st);
  cudaFreeAsync(tmp, st);
  return rc;
}

// Run substeps t0 .. t0 + k - 1 from the state in `in` (k >= 1), landing the
// state t0 + k in `dst` and using `tmp` as the other buffer; `in` is kept.
static int ad_run(aq_adjoint* a, const void* in, int t0, int k, void* dst, void* tmp, cudaStream_t st) {
  void* bufs[2] = {dst, tmp};
  int j = (k % 2 == 1) ? 0 : 1;  // so that the last substep writes dst
  const void* src = in;
  for (int i = 0; i < k; ++i) {
    void* out = bufs[j];
    const int rc = a->impl->step(src, out, t0 + i, st);
    if (rc) return rc;
    src = out;
    j ^= 1;
  }
  a->recomputed += k;
  return AQ_OK;
}

// Bisection checkpointing (the reference's logarithmic stash,
// run_forward_with_ad_nlogn / rerun_from / cnt_ending_zero,
// mpm_solver.py:1093-1137,1201-1207, restated as a recursion): to reverse
// substeps [t0, t1) from the state t0 in `buf`, run forward to the midpoint
// m, keep the state m in this level's stash, reverse [m, t1) with it, then
// reverse [t0, m) from `buf` (reusing the level's stash, which is free
// again).  Memory: one state per level (ceil(log2 T)); recomputation: about
// T log2(T) / 2 substeps.  ab[cur] holds the adjoint of state t1 on entry and
// of state t0 on return.
static int ad_reverse_bisect(aq_adjoint* a, int t0, int t1, const void* buf, int level, void** ab, int& cur,
                             cudaStream_t st) {
  if (t1 - t0 == 1) {
    int rc = a->impl->step_bwd(buf, ab[cur], ab[1 - cur], t0, st);
    if (rc) return rc;
    cur = 1 - cur;
    if (t0 >= 1 && (rc = a->impl->accum(ab[cur], a->dsens, st))) return rc;
    return AQ_OK;
  }
  const int m = t0 + (t1 - t0 + 1) / 2;
  void* mid = a->stash[level];
  int rc = ad_run(a, buf, t0, m - t0, mid, a->stash.back(), st);
  if (rc) return rc;
  if ((rc = ad_reverse_bisect(a, m, t1, mid, level + 1, ab, cur, st))) return rc;
  return ad_reverse_bisect(a, t0, m, buf, level, ab, cur, st);
}

template <int D, class R>
static AdBase* make_ad(aq_adjoint* a) {
  if (a->P.has_F) return new (std::nothrow) AdImpl<D, true, R>(a);
  return new (std::nothrow) AdImpl<D, false, R>(a);
}

static void free_ad(aq_adjoint* a) {
  if (!a) return;
  delete a->impl;
  for (void* p : a->ckpt)
    if (p) cudaFree(p);
  for (void* p : a->seg)
    if (p) cudaFree(p);
  for (void* p : a->stash)
    if (p) cudaFree(p);
  if (a->perm) cudaFree(a->perm);
  if (a->grid) cudaFree(a->grid);
  if (a->gv) cudaFree(a->gv);
  if (a->gvb) cudaFree(a->gvb);
  if (a->dsens) cudaFree(a->dsens);
  delete a;
}

}  // namespace aq

using namespace aq;

extern "C" {

int aq_adjoint_create(const aq_params* P, aq_adjoint** out) {
  if (!P || !out) return AQ_E_ARG;
  *out = nullptr;
  const int D = P->dim;
  if (D != 2 && D != 3) return AQ_E_ARG;
  if (P->has_mat) return AQ_E_LAYOUT;
  if (P->n_particles < 1 || P->n_particles > 0x7fffffffLL) return AQ_E_ARG;
  for (int d = 0; d < D; ++d)
    if (P->res[d] < 3 || P->res[d] > 8192) return AQ_E_ARG;
  const int mk = P->mat[0].kind;
  if (mk != AQ_MAT_FLUID && mk != AQ_MAT_ELASTIC) return AQ_E_ARG;  // reference materials only
  if (!P->has_F && mk != AQ_MAT_FLUID) return AQ_E_LAYOUT;
  if (P->use_friction) return AQ_E_ARG;  // the reference's AD scenes run without friction
  aq_adjoint* a = new (std::nothrow) aq_adjoint();
  if (!a) return AQ_E_NOMEM;
  a->P = *P;
  a->D = D;
  a->NS = 2 * D + D * D + (P->has_F ? D * D : 1);
  a->n = P->n_particles;
  a->rsz = P->precision ? sizeof(double) : sizeof(float);
  a->ncell = 1;
  for (int d = 0; d < D; ++d) a->ncell *= P->res[d];
  cudaError_t e = cudaMalloc(&a->grid, a->rsz * 4 * a->ncell);
  if (e == cudaSuccess) e = cudaMalloc(&a->gv, a->rsz * 4 * a->ncell);
  if (e == cudaSuccess) e = cudaMalloc(&a->gvb, a->rsz * 4 * a->ncell);
  if (e == cudaSuccess) e = cudaMalloc((void**)&a->dsens, sizeof(double) * a->NS);
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "cudaMalloc");
    free_ad(a);
    return AQ_E_NOMEM;
  }
  if (D == 3)
    a->impl = P->precision ? make_ad<3, double>(a) : make_ad<3, float>(a);
  else
    a->impl = P->precision ? make_ad<2, double>(a) : make_ad<2, float>(a);
  if (!a->impl) {
    free_ad(a);
    return AQ_E_NOMEM;
  }
  *out = a;
  return AQ_OK;
}

int aq_adjoint_set_collider(aq_adjoint* a, const float* d_sdf, const float* d_normal, const int32_t* dims,
                            const int32_t* offset, int32_t center, double theta, double height, double omega,
                            double height_rate) {
  if (!a) return AQ_E_ARG;
  if (!d_sdf) {
    a->col_on = 0;
    return AQ_OK;
  }
  if (a->D != 3 || !d_normal || !dims || !offset) return AQ_E_ARG;
  for (int k = 0; k < 3; ++k)
    if (dims[k] < 1) return AQ_E_ARG;
  a->col_on = 1;
  a->col_center = center;
  a->col_sdf = d_sdf;
  a->col_nrm = d_normal;
  for (int k = 0; k < 3; ++k) {
    a->col_dims[k] = dims[k];
    a->col_off[k] = offset[k];
  }
  a->col_theta = theta;
  a->col_height = height;
  a->col_omega = omega;
  a->col_rate = height_rate;
  return AQ_OK;
}

int aq_adjoint_destroy(aq_adjoint* a) {
  if (!a) return AQ_E_ARG;
  cudaDeviceSynchronize();
  free_ad(a);
  return AQ_OK;
}

int aq_adjoint_forward(aq_adjoint* a, const void* d_s0, int32_t n_substeps, int32_t every, void* d_sT,
                       void* stream) {
  if (!a || !d_s0 || !d_sT || n_substeps < 1 || every < 0) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  const size_t sbytes = a->rsz * a->NS * a->n;
  const bool bisect = every == 0;
  const int nck = bisect ? 1 : (n_substeps + every - 1) / every;
  const int nseg = bisect ? 2 : every + 1;
  for (void* p : a->ckpt) cudaFree(p);
  a->ckpt.assign(nck, nullptr);
  for (int k = 0; k < nck; ++k) AQ_CUDA_TRY(cudaMalloc(&a->ckpt[k], sbytes));
  if ((int)a->seg.size() != nseg) {
    for (void* p : a->seg) cudaFree(p);
    a->seg.assign(nseg, nullptr);
    for (int k = 0; k < nseg; ++k) AQ_CUDA_TRY(cudaMalloc(&a->seg[k], sbytes));
  }
  for (void* p : a->stash) cudaFree(p);
  a->stash.clear();
  a->T = n_substeps;
  a->every = every;
  // the state is kept sorted by base cell (a->perm); the caller's order is
  // restored for d_sT here and for the gradients in aq_adjoint_backward
  int rc = ad_make_perm(a, d_s0, st);
  if (rc) return rc;
  if ((rc = a->impl->permute(d_s0, a->seg[0], true, st))) return rc;
  int cur = 0;
  for (int t = 0; t < n_substeps; ++t) {
    if ((bisect && t == 0) || (!bisect && t % every == 0))
      AQ_CUDA_TRY(cudaMemcpyAsync(a->ckpt[bisect ? 0 : t / every], a->seg[cur], sbytes, cudaMemcpyDeviceToDevice, st));
    rc = a->impl->step(a->seg[cur], a->seg[1 - cur], t, st);
    if (rc) return rc;
    cur = 1 - cur;
  }
  return a->impl->permute(a->seg[cur], d_sT, false, st);
}

int aq_adjoint_backward(aq_adjoint* a, const void* d_seed, void* d_grad_s0, double* h_sens, void* stream) {
  if (!a || !d_seed || a->T < 1) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  const size_t sbytes = a->rsz * a->NS * a->n;
  void* ab[2] = {nullptr, nullptr};
  AQ_CUDA_TRY(cudaMallocAsync(&ab[0], sbytes, st));
  AQ_CUDA_TRY(cudaMallocAsync(&ab[1], sbytes, st));
  int rc0 = a->impl->permute(d_seed, ab[0], true, st);  // into the sorted order of the forward pass
  if (rc0) return rc0;
  AQ_CUDA_TRY(cudaMemsetAsync(a->dsens, 0, sizeof(double) * a->NS, st));
  int cur = 0;  // ab[cur] = adjoint of state t+1
  const int T = a->T, every = a->every;
  a->recomputed = 0;
  if (every == 0) {
    int levels = 1;
    while ((1 << levels) < T) ++levels;
    if (a->stash.empty()) {
      a->stash.assign(levels + 1, nullptr);  // one per level, the last one is scratch
      for (void*& p : a->stash) AQ_CUDA_TRY(cudaMalloc(&p, sbytes));
    }
    const int rc = ad_reverse_bisect(a, 0, T, a->ckpt[0], 0, ab, cur, st);
    if (rc) return rc;
  }
  for (int sgi = every == 0 ? -1 : (T - 1) / every; sgi >= 0; --sgi) {
    const int t0 = sgi * every, t1 = std::min(T, t0 + every);
    AQ_CUDA_TRY(cudaMemcpyAsync(a->seg[0], a->ckpt[sgi], sbytes, cudaMemcpyDeviceToDevice, st));
    for (int t = t0; t < t1 - 1; ++t) {
      const int rc = a->impl->step(a->seg[t - t0], a->seg[t - t0 + 1], t, st);
      if (rc) return rc;
    }
    for (int t = t1 - 1; t >= t0; --t) {
      const int rc = a->impl->step_bwd(a->seg[t - t0], ab[cur], ab[1 - cur], t, st);
      if (rc) return rc;
      cur = 1 - cur;  // ab[cur] = adjoint of state t
      if (t >= 1) {
        const int rc2 = a->impl->accum(ab[cur], a->dsens, st);
        if (rc2) return rc2;
      }
    }
  }
  if (d_grad_s0) {
    const int rc = a->impl->permute(ab[cur], d_grad_s0, false, st);
    if (rc) return rc;
  }
  if (h_sens) AQ_CUDA_TRY(cudaMemcpyAsync(h_sens, a->dsens, sizeof(double) * a->NS, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaFreeAsync(ab[0], st));
  AQ_CUDA_TRY(cudaFreeAsync(ab[1], st));
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  return AQ_OK;
}

}  // extern "C"
