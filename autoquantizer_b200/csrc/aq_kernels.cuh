// Device code of the quantized MLS-MPM substep (sm_100a).
//
// This header is compiled twice: by nvcc into libaq.so with the record
// layout read from the kernel parameter (RtLayout), and at simulator
// creation by NVRTC with the layout as a constexpr (a JitLayout generated
// by aq_jit.cu), so that bit offsets, scales and slot kinds fold into the
// instruction stream the way the reference's per-field LLVM codegen does
// (codegen_llvm_quant.cpp).
//
// Data layout in HBM
//   records  : n x W u64 bit_pack records, grouped by 4^3 (3D) or 8^2 (2D)
//              cell block; inside a block slot-major (the first record of
//              every cell in cell order, then the second of every cell, ...),
//              so that 32 consecutive records lie in 32 different cells
//              except where a slot has fewer than 32 cells.  Stored in
//              groups of 32 records with their words interleaved in pairs
//              (grec_word, aq_codec.cuh): a warp's record loads and stores
//              are coalesced 16-byte vectors.  A particle-id array moves
//              with the records.
//   grids    : two dense grids of R4 nodes (m, m v), row-major: one holds
//              the P2G sums of substep k (grid_op is applied as tiles are
//              staged from it), the other receives the P2G of substep k+1
//              (cleared by the host before the launch).
//   binning  : per-cell counts/offsets, per-particle key and rank, and one
//              work item per occupied block (block, first record, count).
//
// k_step, persistent CTAs of CH = 64 threads (two warps) claiming work items
// (whole cell blocks, the fullest first) from a counter:
//   1. stage the block's grid tile (7^3 nodes in 3D: the block, the cell
//      below it and the stencil) in shared memory, applying grid_op (and
//      the SDF collider when compiled in) to every node (G2P source);
//   2. the warps take the block's records 32 at a time (units), without
//      CTA barriers between units; per unit each lane loads its record into
//      registers (layout-specialized build, short records) or its shared
//      slot, and
//      a. G2P of substep k: gather 3^d nodes (z-separable sums), new v, C,
//         x, F|J; bit_pack_assign into the record, which also yields the
//         values a later decode returns; record written back to HBM;
//      b. P2G of substep k+1 from those values into the warp's private tile
//         of float4 nodes with plain shared-memory read-add-writes, offset
//         by offset with __syncwarp ordering (lanes that share a base cell
//         take turns, found with __match_any_sync);
//   3. the warp tiles are summed (and re-zeroed) over the box of touched
//      nodes and flushed with one red.global.add.v4.f32 per node.
// G2P or P2G may be off (first / last substep of a run).
#pragma once

#include "aq_codec.cuh"
#include "aq_step_config.h"

#ifdef __CUDACC_RTC__
#define AQ_POS_INF __int_as_float(0x7f800000)
#else
#include <math.h>
#define AQ_POS_INF INFINITY
#endif

namespace aq {

// Threads per CTA.  Two warps per work item: the warps of an item wait for
// each other only at its staging and flush barriers, and the fewer warps an
// item has, the less time they spend waiting there and the fewer private
// tiles its flush sums (at the same 24 resident warps per SM, 64-thread CTAs
// measured 2.7 % faster than 128-thread CTAs on the 3D mixed scene, 96
// 2.4 %, 32 4.5 % slower: shared memory then holds 17 CTAs only).
constexpr int CH = AQ_CH;  // AQ_CH: aq_step_config.h
constexpr int NWARP = CH / 32;
// CTAs per SM the register allocation of k_step must allow: the layout's
// choice (LA::kMinBlocks) for float, 512 / CH (128 registers) for double.
// Short records kept in registers run best at 768 / CH CTAs (80 registers:
// more resident warps beat the extra spills); records in shared-memory
// slots at 512 / CH.
#ifndef AQ_STEP_MIN_BLOCKS
#define AQ_STEP_MIN_BLOCKS(R, LA) (sizeof(R) == 8 ? 512 / AQ_CH : LA::kMinBlocks)
#endif

template <int D>
struct Geo {
  static constexpr int BS = D == 3 ? 4 : 8;          // block edge (cells)
  // tile edge: base cells of a block's particles span the block and the
  // cell below it, plus the 3-node stencil; 2D keeps one cell of slack for
  // drift between re-binnings (3D particles that drift out take the global
  // fallback path: a 7-node tile leaves room in L1 for the 4 CTAs per SM)
  static constexpr int T = D == 3 ? BS + 3 : BS + 4;
  // stride of the slowest tile axis, padded to 4 mod 8 nodes so that
  // neighbouring x planes fall in different 16-byte bank groups
  static constexpr int XS = D == 3 ? (T * T + 3) / 8 * 8 + 4 : T;
  static constexpr int TNP = D == 3 ? T * XS : T * T;  // nodes per tile plane incl. padding
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
  typedef float4 type;
};
template <>
struct R4T<double> {
  typedef double4 type;
};

template <class R>
struct SimK {
  int res[3], nb[3];
  int W, WS, friction, bound_clip, n_mat, _pad;
  R inv_dx, dx, dt, p_mass, stress_coef, four_inv_dx, grav;
  double lb[3], ub[3];
  R clip_lo[3], clip_hi[3];
  int mat_kind[AQ_MAX_MATERIALS];
  R mu[AQ_MAX_MATERIALS], lam[AQ_MAX_MATERIALS];
  // SDF collider (3D; col_on = 0: none): signed distance and normal volumes
  // (float, col_dims, placed at grid index col_off), rotation centre at
  // (col_n, ., col_n), rotated indices clamped to [col_lo, col_hi]
  int col_on, col_n, col_dims[3], col_off[3], col_lo[3], col_hi[3];
  const float* col_sdf;
  const float* col_nrm;
  R col_omega;
  R col_c, col_s;  // cos and sin of the collider angle this launch
  int col_yshift;  // collider height in cells this launch, int(height / dx + 0.5)
  int col_node_cv;  // 1: collider velocity omega x r from the node itself (sdf_collision_no_arg)
  // sparse grids (k_step's SP): grid block -> pool slot (-1: none), the
  // slots handed out so far, each slot's block, the pools' capacity
  int32_t* bptr;
  int32_t* n_alloc;
  int32_t* pool_blk;
  int pool_cap;
};

struct StepArgs {
  uint64_t* words;
  const int32_t* pid;
  const int4* items;
  const int32_t* n_items;
  int32_t* item_ctr;       // next unclaimed item of this launch (starts at zero)
  int32_t* item_ctr_next;  // the next launch's counter, zeroed by this launch
  const void* grid_in;  // G2P source (after grid_op)
  void* grid_out;       // P2G target (zeroed)
  unsigned* status;
  unsigned long long* fallbacks;
  double* rmax;
  double* rmin;
  uint64_t sk;          // dithering key of the G2P substep
  int do_g2p, do_p2g, ranges;
  int raw_in;           // grid_in holds P2G sums: apply grid_op while reading
};

// Layout from the kernel parameter (nvcc build).
struct RtLayout {
  static constexpr bool kRegRecord = false;  // records pass through shared memory
  static constexpr int kWords = 0;            // runtime word count
  static constexpr int kMinBlocks = 512 / AQ_CH;
  static __device__ __forceinline__ const aq_layout& get(const aq_layout& p) { return p; }
};

// ---------------------------------------------------------------- helpers

template <class R>
__device__ __forceinline__ int base_of(R x, const SimK<R>& K, int d, unsigned& fl) {
  const R t = x * K.inv_dx - (R)0.5;
  if (t != t) {
    fl |= AQ_ST_NAN;
    return 0;
  }
  if (t < (R)0) {
    fl |= AQ_ST_OUT_OF_DOMAIN;
    return 0;
  }
  if (t >= (R)(K.res[d] - 2)) {
    fl |= AQ_ST_OUT_OF_DOMAIN;
    return K.res[d] - 3;
  }
  return (int)floor(t);
}

template <int D>
__device__ __forceinline__ int64_t cell_index(const int (&res)[3], int i, int j, int k) {
  return D == 3 ? ((int64_t)i * res[1] + j) * res[2] + k : (int64_t)i * res[1] + j;
}

__device__ __forceinline__ void red_add_node(float4* g, float m, float a, float b, float c) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(g), "f"(m), "f"(a), "f"(b), "f"(c)
               : "memory");
}

__device__ __forceinline__ void red_add_node(double4* g, double m, double a, double b, double c) {
  double* p = reinterpret_cast<double*>(g);
  atomicAdd(p, m);
  atomicAdd(p + 1, a);
  atomicAdd(p + 2, b);
  atomicAdd(p + 3, c);
}

// Order-preserving map of doubles to unsigned 64-bit keys (key(a) < key(b)
// iff a < b, NaN aside): non-negative values get the sign bit set, negative
// ones are inverted.  Lets shared-memory 64-bit atomicMax/atomicMin keep
// running extremes without compare-and-swap loops.
__device__ __forceinline__ unsigned long long ord_key(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_val(unsigned long long k) {
  return __longlong_as_double((long long)((k >> 63) ? (k & 0x7fffffffffffffffull) : ~k));
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

// ------------------------------------------------------------ sparse grids
// A sparse grid stores its nodes in pools of node blocks (the BS^D nodes of
// one grid block, row-major inside it), reached through a table from grid
// block (row-major over blocks) to pool slot; -1: the block holds no node,
// which reads as zero.  Both pools (P2G target and G2P source) share the
// table.  Slots are handed out by one counter; the pools' slots at and
// beyond it are kept zero.

template <int D>
__device__ __forceinline__ int64_t block_of(const int (&nb)[3], int i0, int i1, int i2) {
  constexpr int BS = Geo<D>::BS;
  return D == 3 ? ((int64_t)(i0 / BS) * nb[1] + i1 / BS) * nb[2] + i2 / BS : (int64_t)(i0 / BS) * nb[1] + i1 / BS;
}

template <int D>
__device__ __forceinline__ int64_t node_in_slot(int slot, int i0, int i1, int i2) {
  constexpr int BS = Geo<D>::BS;
  const int l0 = i0 & (BS - 1), l1 = i1 & (BS - 1), l2 = i2 & (BS - 1);
  return (int64_t)slot * 64 + (D == 3 ? (l0 * BS + l1) * BS + l2 : l0 * BS + l1);
}

// Pool slot of an in-grid tile node from an item's table of the 3^D blocks
// around its block (ob: the item's block coordinates)
template <int D>
__device__ __forceinline__ int tile_slot(const int* sslot, int ob0, int ob1, int ob2, int g0, int g1, int g2) {
  constexpr int BS = Geo<D>::BS;
  const int a0 = g0 / BS - ob0 + 1, a1 = g1 / BS - ob1 + 1, a2 = D == 3 ? g2 / BS - ob2 + 1 : 0;
  return sslot[D == 3 ? (a0 * 3 + a1) * 3 + a2 : a0 * 3 + a1];
}

// Slot of block blk for a write, handed out now if the block has none: take
// a slot from the counter, then install it unless another thread installed
// one first (the slot taken is then left unused, still zero).  No waiting.
// -1: the pools are full.  Out of line: it runs for few writes.
static __device__ __noinline__ int claim_slot(int32_t* bptr, int32_t* n_alloc, int32_t* pool_blk, int cap, int64_t blk) {
  const int s = bptr[blk];
  if (s >= 0) return s;
  const int mine = atomicAdd(n_alloc, 1);
  if (mine >= cap) return -1;
  const int old = atomicCAS(bptr + blk, -1, mine);
  if (old == -1) {
    pool_blk[mine] = (int32_t)blk;
    return mine;
  }
  return old;
}

// grid_op (mpm_solver.py:633-665) of one node (m, m v) at grid index I:
// velocity, gravity, optional friction on the floor, sticky walls.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// Grid post-process of the rotating SDF collider (sdf_collision and
// rot_scene, mpm_solver.py:1459-1480,1515-1540): the node's index is rotated
// by -theta about (n, ., n) and lowered by the collider height; where the
// signed distance there is below -1e-5 the velocity relative to the
// collider (omega x r, r = (rotated index - (n, I1, n)) dx) loses its
// component into the surface along the rotated normal.
// KT: any parameter block with the collider fields (SimK, the adjoint's AdK).
// Returns whether node I is inside the collider, and there the rotated
// normal and the collider's velocity omega x r: r from the rotated index
// (sdf_collision) or, with NODE_CV, from the node itself
// (sdf_collision_no_arg, mpm_solver.py:1510, the reference's autodiff path).
// whether a parameter block asks for the node's own position in omega x r:
// the simulator's per-launch choice, none for other blocks
template <class KT>
__device__ __forceinline__ bool col_node_cv_of(const KT&) {
  return false;
}
template <class R>
__device__ __forceinline__ bool col_node_cv_of(const SimK<R>& K) {
  return K.col_node_cv != 0;
}

template <class R, bool NODE_CV = false, class KT>
__device__ __forceinline__ bool collider_at(const KT& K, int I0, int I1, int I2, R (&nrm)[3], R (&cv)[3]) {
  const int n = K.col_n;
  const int i0 = I0 >= 2 * n ? I0 - 2 * n : I0, i2 = I2 >= 2 * n ? I2 - 2 * n : I2;
  const R c = K.col_c, s = K.col_s;
  const R o0 = (R)(i0 - n), o2 = (R)(i2 - n);
  // each operation rounded on its own (no FMA contraction), so that the
  // truncation to an index matches a plain CPU evaluation
  const R x = add_rn(add_rn(sub_rn(mul_rn(c, o0), mul_rn(s, o2)), (R)n), (R)0.5);
  const R z = add_rn(add_rn(add_rn(mul_rn(s, o0), mul_rn(c, o2)), (R)n), (R)0.5);
  int r[3] = {(int)x, I1 - K.col_yshift, (int)z};
#pragma unroll
  for (int k = 0; k < 3; ++k) r[k] = max(min(r[k], K.col_hi[k]), K.col_lo[k]);
  const int a = r[0] - K.col_off[0], b = r[1] - K.col_off[1], e = r[2] - K.col_off[2];
  if (a < 0 || a >= K.col_dims[0] || b < 0 || b >= K.col_dims[1] || e < 0 || e >= K.col_dims[2]) return false;
  const int64_t q = ((int64_t)a * K.col_dims[1] + b) * K.col_dims[2] + e;
  if (!(K.col_sdf[q] < -1e-5f)) return false;
  const R g0 = (R)K.col_nrm[3 * q], g1 = (R)K.col_nrm[3 * q + 1], g2 = (R)K.col_nrm[3 * q + 2];
  nrm[0] = c * g0 + s * g2;
  nrm[1] = g1;
  nrm[2] = -s * g0 + c * g2;
  const bool from_node = NODE_CV || col_node_cv_of(K);
  const R rx = (R)((from_node ? I0 : r[0]) - n) * K.dx, rz = (R)((from_node ? I2 : r[2]) - n) * K.dx;
  cv[0] = K.col_omega * rz;
  cv[1] = (R)0;
  cv[2] = -K.col_omega * rx;
  return true;
}

template <class R, bool NODE_CV = false, class KT>
__device__ __forceinline__ void collide_node(const KT& K, int I0, int I1, int I2, R (&v)[3]) {
  R nrm[3], cv[3];
  if (!collider_at<R, NODE_CV>(K, I0, I1, I2, nrm, cv)) return;
  R vr[3], dn = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    vr[k] = v[k] - cv[k];
    dn += vr[k] * nrm[k];
  }
  dn = dn < (R)0 ? dn : (R)0;
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = cv[k] + (vr[k] - dn * nrm[k]);
}

template <int D, class R, bool COL, class R4>
__device__ __forceinline__ R4 grid_op_node(const SimK<R>& K, R4 g, int I0, int I1, int I2) {
  const int I[3] = {I0, I1, I2};
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
  if (COL && D == 3 && K.col_on) collide_node<R>(K, I0, I1, I2, v);
  g.y = v[0];
  g.z = v[1];
  g.w = v[2];
  return g;
}

// ------------------------------------------------------------- materials

template <int D, class R>
__device__ __forceinline__ R det(const R* F) {
  if (D == 2) return F[0] * F[3] - F[1] * F[2];
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
         F[2] * (F[3] * F[7] - F[4] * F[6]);
}

// Rotation of the polar decomposition: 2D closed form (linalg_impl.py:9-26);
// 3D by Newton's iteration X <- (X + X^-T)/2 (Higham 1986).
template <int D, class R>
__device__ __forceinline__ void polar_rot(const R* F, R* Rm) {
  if (D == 2) {
    const R x = F[0] + F[3], y = F[2] - F[1];
    const R sc = (R)1 / sqrt(x * x + y * y);
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
      // leave together: a converged lane's extra iteration changes X by
      // rounding noise only, and the warp stays converged
      if (__all_sync(__activemask(), diff < tol * tol)) break;
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

template <int D, class R>
__device__ __forceinline__ void bspline(const R* x, const SimK<R>& K, int* base, R* fx, R (&w)[3][3], unsigned& fl) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    base[d] = base_of<R>(x[d], K, d, fl);
    fx[d] = x[d] * K.inv_dx - (R)base[d];
    w[0][d] = (R)0.5 * ((R)1.5 - fx[d]) * ((R)1.5 - fx[d]);
    w[1][d] = (R)0.75 - (fx[d] - (R)1) * (fx[d] - (R)1);
    w[2][d] = (R)0.5 * (fx[d] - (R)0.5) * (fx[d] - (R)0.5);
  }
}

// ------------------------------------------------------------ the step

// COL: compiled with the SDF collider (the library's own build always is;
// the layout-specialized build only when a collider is set).  SP: sparse
// grids (grid_in / grid_out are node pools reached through K.bptr).
template <int D, bool HF, bool HM, class R, class LA, bool COL = true, bool SP = false>
__global__ void __launch_bounds__(CH, AQ_STEP_MIN_BLOCKS(R, LA)) k_step(const __grid_constant__ aq_layout Lp, const SimK<R> K,
                                                const StepArgs A) {
  typedef Sch<D, HF, HM> S;
  typedef Geo<D> G;
  typedef typename R4T<R>::type R4;
  constexpr int NS = S::NS;
  constexpr int T = G::T;
  constexpr int TNP = G::TNP;
  auto&& L = LA::get(Lp);  // a reference (RtLayout) or a folded constant (JitLayout)
  const int W = L.n_words;
  const int WS = K.WS;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  R4* gtile = reinterpret_cast<R4*>(smem_raw);                      // TNP nodes (m, v): G2P source
  R4* ptile = gtile + TNP;                                     // NWARP x TNP (m, m v): P2G, per warp
  uint64_t* srec = reinterpret_cast<uint64_t*>(ptile + NWARP * TNP);  // CH x WS: each thread's record (RtLayout)
  __shared__ int sbox[6];  // tile-coordinate box of the item's P2G base cells (min[3], max[3])
  __shared__ int s_next;   // the CTA's next work item, claimed from A.item_ctr
  __shared__ int sslot[SP ? 27 : 1];  // sparse grids: pool slots of the 3^D blocks around the item's block
  // range detection: the CTA's running max / min per slot (ord_key order)
  __shared__ unsigned long long s_rmax[AQ_MAX_SLOTS], s_rmin[AQ_MAX_SLOTS];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nitems = *A.n_items;
  if (A.ranges && A.do_g2p && tid < NS) {
    s_rmax[tid] = 0ull;   // below every key
    s_rmin[tid] = ~0ull;  // above every key
  }
  const R4* gin = reinterpret_cast<const R4*>(A.grid_in);
  R4* gout = reinterpret_cast<R4*>(A.grid_out);
  unsigned fl = 0, nfall = 0;
  // the thread's record words: registers when the layout (and so the word
  // count and every bit offset) is a compile-time constant and the record
  // short, else a slot of shared memory
  uint64_t rrec[LA::kRegRecord ? LA::kWords : 1];
  uint64_t* const myrec = LA::kRegRecord ? rrec : srec + tid * WS;
  R4 zero4;
  zero4.x = zero4.y = zero4.z = zero4.w = 0;
  if (A.do_p2g)  // private tiles start at zero; the flush of every item re-zeroes them
    for (int j = tid; j < NWARP * TNP; j += CH) ptile[j] = zero4;

  // Work items are whole cell blocks, claimed one at a time from a counter
  // (largest imbalance: one item).  Inside an item the warps take the
  // block's records 32 at a time (units u = warp, warp + NWARP, ...), with
  // no CTA barrier between units: the grid tile is staged once per item and
  // the warp tiles are flushed once per item.
  if (tid == 0) {
    if (blockIdx.x == 0) *A.item_ctr_next = 0;
    s_next = atomicAdd(A.item_ctr, 1);
  }
  __syncthreads();
  for (int it = s_next; it < nitems; it = s_next) {
    const int4 item = A.items[it];
    const int cnt = item.z;
    const int64_t first = item.y;
    const int nunits = (cnt + 31) >> 5;
    if (tid < 6) sbox[tid] = tid < 3 ? T : -1;
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
    // block coordinates of the item (sparse grids); a tile node lies in the
    // blocks ob - 1 .. ob + 1
    const int ob0 = SP ? (o[0] + 1) / G::BS : 0, ob1 = SP ? (o[1] + 1) / G::BS : 0,
              ob2 = (SP && D == 3) ? (o[2] + 1) / G::BS : 0;
    if (SP) {
      if (tid < (D == 3 ? 27 : 9)) {
        const int e0 = D == 3 ? tid / 9 : tid / 3, e1 = D == 3 ? (tid / 3) % 3 : tid % 3, e2 = D == 3 ? tid % 3 : 1;
        const int b0 = ob0 + e0 - 1, b1 = ob1 + e1 - 1, b2 = ob2 + e2 - 1;
        int sl = -1;
        if (b0 >= 0 && b0 < K.nb[0] && b1 >= 0 && b1 < K.nb[1] && (D == 2 || (b2 >= 0 && b2 < K.nb[2])))
          sl = K.bptr[D == 3 ? ((int64_t)b0 * K.nb[1] + b1) * K.nb[2] + b2 : (int64_t)b0 * K.nb[1] + b1];
        sslot[tid] = sl;
      }
      __syncthreads();
    }
    if (A.do_g2p) {  // stage the grid tile (m, v after grid_op)
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
        R4 g = zero4;
        if (ok) {
          if (SP) {
            const int sl = tile_slot<D>(sslot, ob0, ob1, ob2, g0, g1, g2);
            if (sl >= 0) g = gin[node_in_slot<D>(sl, g0, g1, g2)];
          } else {
            g = gin[cell_index<D>(K.res, g0, g1, g2)];
          }
          if (A.raw_in) g = grid_op_node<D, R, COL>(K, g, g0, g1, g2);
        }
        gtile[j] = g;
      }
    }
    __syncthreads();

    for (int u = warp; u < nunits; u += NWARP) {
      const int64_t rec = first + 32 * u + lane;
      const bool active = 32 * u + lane < cnt;
      int32_t pid = 0;
      if (active) {  // grouped storage: the warp's 16-byte pair loads coalesce
        load_grec<LA::kWords>(A.words, rec, W, myrec);
        pid = __ldg(A.pid + rec);
      }
      R vals[NS];
      if (active) {
        if (A.do_g2p) {  // G2P reads x, F|J and the material id; v and C are rewritten
          constexpr unsigned XFM = ((1u << D) - 1u) | (((1u << S::NFJ) - 1u) << S::FJ) | (HM ? 1u << S::MAT : 0u);
          decode_record<NS, R, XFM>(L, myrec, vals);
#pragma unroll
          for (int k = S::V; k < S::FJ; ++k) vals[k] = 0;
        } else {
          decode_record<NS, R>(L, myrec, vals);
        }
      }

      // ---------------------------------------------------------------- G2P
      if (A.do_g2p && active) {
        int base[3] = {0, 0, 0};
        R fx[3] = {0, 0, 0}, w[3][3];
        bspline<D, R>(vals + S::X, K, base, fx, w, fl);
        bool in_tile = true;
#pragma unroll
        for (int d = 0; d < D; ++d) {
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
        const int lb = in_tile ? (D == 3 ? (base[0] - o[0]) * G::XS + (base[1] - o[1]) * T + (base[2] - o[2])
                                         : (base[0] - o[0]) * T + (base[1] - o[1]))
                               : 0;
        if (D == 3 && in_tile) {
          // separable in z: per (a, b) the three z-neighbours are summed
          // with weights w_c and c w_c first (P, Q), then spread with w_a w_b
          const R tw2 = (R)2 * w[2][2];
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              const R4* gp = gtile + lb + a * G::XS + b * T;
              const R4 g0 = gp[0], g1 = gp[1], g2 = gp[2];
              const R P[3] = {w[0][2] * g0.y + w[1][2] * g1.y + w[2][2] * g2.y,
                              w[0][2] * g0.z + w[1][2] * g1.z + w[2][2] * g2.z,
                              w[0][2] * g0.w + w[1][2] * g1.w + w[2][2] * g2.w};
              const R Q[3] = {w[1][2] * g1.y + tw2 * g2.y, w[1][2] * g1.z + tw2 * g2.z, w[1][2] * g1.w + tw2 * g2.w};
              const R wab = w[a][0] * w[b][1];
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                const R wp = wab * P[d];
                nv[d] += wp;
                if (a == 1) Sm[d][0] += wp;
                if (a == 2) Sm[d][0] += (R)2 * wp;
                if (b == 1) Sm[d][1] += wp;
                if (b == 2) Sm[d][1] += (R)2 * wp;
                Sm[d][2] += wab * Q[d];
              }
            }
        } else if (D == 2 && in_tile) {
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              const R weight = w[a][0] * w[b][1];
              const R4 g = gtile[lb + a * T + b];
              const R gv[3] = {g.y, g.z, g.w};
              const int off[3] = {a, b, 0};
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
            }
        } else {
          // outside the tile (rare): the global grid, one node per iteration
          // (a rolled loop keeps this cold path out of the instruction cache)
          ++nfall;
#pragma unroll 1
          for (int k = 0; k < (D == 3 ? 27 : 9); ++k) {
            const int a = D == 3 ? k / 9 : k / 3, b = D == 3 ? (k / 3) % 3 : k % 3, c = D == 3 ? k % 3 : 0;
            const R wa = a == 0 ? w[0][0] : (a == 1 ? w[1][0] : w[2][0]);
            const R wb = b == 0 ? w[0][1] : (b == 1 ? w[1][1] : w[2][1]);
            const R wc = c == 0 ? w[0][2] : (c == 1 ? w[1][2] : w[2][2]);
            const R wab = wa * wb;
            const R weight = D == 3 ? wab * wc : wab;
            const int n0 = base[0] + a, n1 = base[1] + b, n2 = D == 3 ? base[2] + c : 0;
            R4 g;
            if (SP) {
              const int sl = K.bptr[block_of<D>(K.nb, n0, n1, n2)];
              g = sl >= 0 ? gin[node_in_slot<D>(sl, n0, n1, n2)] : zero4;
            } else {
              g = gin[cell_index<D>(K.res, n0, n1, n2)];
            }
            if (A.raw_in) g = grid_op_node<D, R, COL>(K, g, n0, n1, n2);
            const R gv[3] = {g.y, g.z, g.w};
            const R offr[3] = {(R)a, (R)b, (R)c};
#pragma unroll
            for (int d = 0; d < D; ++d) {
              const R wg = weight * gv[d];
              nv[d] += wg;
#pragma unroll
              for (int e = 0; e < D; ++e) Sm[d][e] += offr[e] * wg;
            }
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
        encode_record<NS, R>(L, vals, myrec, particle_key(A.sk, pid), (const float*)0, (const double*)0);
        store_grec<LA::kWords>(A.words, rec, W, myrec);
      }

      // -------------------------------------------- range detection (opt)
      if (A.ranges && A.do_g2p) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          double mx = active ? (double)vals[s] : -(double)AQ_POS_INF;
          double mn = active ? (double)vals[s] : (double)AQ_POS_INF;
#pragma unroll
          for (int k = 16; k; k >>= 1) {
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, k));
            mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, k));
          }
          if (lane == 0) {
            atomicMax(&s_rmax[s], ord_key(mx));
            atomicMin(&s_rmin[s], ord_key(mn));
          }
        }
      }

      // ---------------------------------------------------------------- P2G
      if (A.do_p2g) {
        int base[3] = {0, 0, 0};
        R fx[3] = {0, 0, 0}, w[3][3];
        R Aff[D * D], q[D];
        bool in_tile = false;
        int lb = 0;
        if (active) {
          const int mat = HM ? min(max((int)vals[S::MAT], 0), K.n_mat - 1) : 0;
          bspline<D, R>(vals + S::X, K, base, fx, w, fl);
          in_tile = true;
#pragma unroll
          for (int d = 0; d < D; ++d) {
            const int l = base[d] - o[d];
            in_tile = in_tile && l >= 0 && l <= T - 3;
          }
          R cau[D * D];
          cauchy<D, HF, R>(K, mat, vals + S::FJ, vals[S::FJ], cau);
          // node value = m v + affine (off - fx) dx = q + Aff off,
          // q = m v - affine fx dx, Aff = (stress + m C) dx
#pragma unroll
          for (int k = 0; k < D * D; ++k) Aff[k] = (K.stress_coef * cau[k] + K.p_mass * vals[S::C + k]) * K.dx;
#pragma unroll
          for (int d = 0; d < D; ++d) {
            R s = K.p_mass * vals[S::V + d];
#pragma unroll
            for (int e = 0; e < D; ++e) s -= Aff[d * D + e] * fx[e];
            q[d] = s;
          }
          if (in_tile) {
            lb = D == 3 ? (base[0] - o[0]) * G::XS + (base[1] - o[1]) * T + (base[2] - o[2])
                        : (base[0] - o[0]) * T + (base[1] - o[1]);
          } else {
            ++nfall;
          }
        }
        {  // grow the item's box by this warp's in-tile base cells
          int mn[3], mx[3];
#pragma unroll
          for (int d = 0; d < D; ++d) {
            const int l = base[d] - o[d];
            mn[d] = __reduce_min_sync(0xffffffffu, (active && in_tile) ? l : T);
            mx[d] = __reduce_max_sync(0xffffffffu, (active && in_tile) ? l : -1);
          }
          if (lane == 0 && mx[0] >= 0) {
#pragma unroll
            for (int d = 0; d < D; ++d) {
              atomicMin(&sbox[d], mn[d]);
              atomicMax(&sbox[3 + d], mx[d]);
            }
          }
        }
        // Lanes of a warp with the same base cell add into the same nodes and
        // take turns (rank among peers); lanes of different base cells never
        // share a node for the same stencil offset.  Binning orders records so
        // that a warp's lanes are in different cells: one turn is the norm.
        const int key = (active && in_tile) ? lb : -1 - lane;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        const int rounds = __reduce_max_sync(0xffffffffu, (unsigned)__popc(peers));
        R4* mytile = ptile + warp * TNP;
        for (int r = 0; r < rounds; ++r) {
          const bool mine = active && rank == r;
          const unsigned tm = __ballot_sync(0xffffffffu, mine && in_tile);  // lanes writing the tile this round
          if (mine && in_tile) {
            // Lanes add into their nodes offset by offset.  Lanes whose base
            // cells are neighbours reach the same node at different offsets,
            // so every offset's read-modify-write must be visible to the warp
            // before the next one reads: __syncwarp orders them (without it
            // the compiler and the shared-memory pipeline may overlap them
            // and lose updates).
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
              for (int b = 0; b < 3; ++b) {
                const R wab = w[a][0] * w[b][1];
                R qab[3];
#pragma unroll
                for (int d = 0; d < D; ++d) {
                  R s = q[d];
                  if (a == 1) s += Aff[d * D + 0];
                  if (a == 2) s += (R)2 * Aff[d * D + 0];
                  if (b == 1) s += Aff[d * D + 1];
                  if (b == 2) s += (R)2 * Aff[d * D + 1];
                  qab[d] = s;
                }
#pragma unroll
                for (int c = 0; c < (D == 3 ? 3 : 1); ++c) {
                  const R weight = D == 3 ? wab * w[c][2] : wab;
                  R mv[3] = {0, 0, 0};
#pragma unroll
                  for (int d = 0; d < D; ++d) {
                    R s = qab[d];
                    if (D == 3 && c == 1) s += Aff[d * D + 2];
                    if (D == 3 && c == 2) s += (R)2 * Aff[d * D + 2];
                    mv[d] = weight * s;
                  }
                  R4& t = mytile[lb + (D == 3 ? a * G::XS + b * T + c : a * T + b)];
                  R4 v = t;
                  v.x += weight * K.p_mass;
                  v.y += mv[0];
                  v.z += mv[1];
                  v.w += mv[2];
                  t = v;
                  __syncwarp(tm);
                }
              }
          } else if (mine) {  // outside the tile: straight to the global grid
            // sparse grids: slots of the (at most 2^D) blocks under the stencil
            int fsl[D == 3 ? 8 : 4];
            const int fb0 = base[0] / G::BS, fb1 = base[1] / G::BS, fb2 = D == 3 ? base[2] / G::BS : 0;
            if (SP) {
#pragma unroll 1
              for (int qb = 0; qb < (D == 3 ? 8 : 4); ++qb) {
                const int c0 = fb0 + (D == 3 ? qb >> 2 : qb >> 1), c1 = fb1 + (D == 3 ? (qb >> 1) & 1 : qb & 1),
                          c2 = D == 3 ? fb2 + (qb & 1) : 0;
                int sl = -1;
                if (c0 < K.nb[0] && c1 < K.nb[1] && (D == 2 || c2 < K.nb[2])) {
                  const int64_t bk = D == 3 ? ((int64_t)c0 * K.nb[1] + c1) * K.nb[2] + c2 : (int64_t)c0 * K.nb[1] + c1;
                  sl = claim_slot(K.bptr, K.n_alloc, K.pool_blk, K.pool_cap, bk);
                  if (sl < 0) fl |= AQ_ST_POOL_FULL;
                }
                fsl[qb] = sl;
              }
            }
            // one node per iteration: a rolled loop keeps this cold path
            // out of the instruction cache
#pragma unroll 1
            for (int k = 0; k < (D == 3 ? 27 : 9); ++k) {
              const int a = D == 3 ? k / 9 : k / 3, b = D == 3 ? (k / 3) % 3 : k % 3, c = D == 3 ? k % 3 : 0;
              const R wa = a == 0 ? w[0][0] : (a == 1 ? w[1][0] : w[2][0]);
              const R wb = b == 0 ? w[0][1] : (b == 1 ? w[1][1] : w[2][1]);
              const R wc = c == 0 ? w[0][2] : (c == 1 ? w[1][2] : w[2][2]);
              const R weight = D == 3 ? wa * wb * wc : wa * wb;
              R mv[3] = {0, 0, 0};
#pragma unroll
              for (int d = 0; d < D; ++d) {
                R s = q[d];
                s += (R)a * Aff[d * D + 0];
                s += (R)b * Aff[d * D + 1];
                if (D == 3) s += (R)c * Aff[d * D + 2];
                mv[d] = weight * s;
              }
              const int n0 = base[0] + a, n1 = base[1] + b, n2 = D == 3 ? base[2] + c : 0;
              if (SP) {
                const int qb = D == 3 ? ((n0 / G::BS - fb0) << 2) | ((n1 / G::BS - fb1) << 1) | (n2 / G::BS - fb2)
                                      : ((n0 / G::BS - fb0) << 1) | (n1 / G::BS - fb1);
                const int sl = fsl[qb];
                if (sl >= 0)
                  red_add_node(gout + node_in_slot<D>(sl, n0, n1, n2), weight * K.p_mass, mv[0], mv[1], mv[2]);
              } else {
                red_add_node(gout + cell_index<D>(K.res, n0, n1, n2), weight * K.p_mass, mv[0], mv[1], mv[2]);
              }
            }
          }
          __syncwarp();
        }
      }
    }  // units
    __syncthreads();
    if (A.do_p2g) {
      // sum the warp tiles, re-zero them, flush: one vector reduction per
      // node of the box the item's particles touched (base box + 2); the
      // tiles are zero outside it
      const int e0 = sbox[3] - sbox[0] + 3, e1 = sbox[4] - sbox[1] + 3, e2 = D == 3 ? sbox[5] - sbox[2] + 3 : 1;
      const int nbox = sbox[3] >= 0 ? e0 * e1 * e2 : 0;
      const float ie1 = 1.0f / (float)e1, ie2 = 1.0f / (float)e2;  // exact floors: j < 2^10, e <= 12
      for (int j = tid; j < nbox; j += CH) {
        const int q = D == 3 ? (int)(((float)j + 0.5f) * ie2) : j;
        const int l2 = D == 3 ? sbox[2] + (j - q * e2) : 0;
        const int i0 = (int)(((float)q + 0.5f) * ie1);
        const int l0 = sbox[0] + i0, l1 = sbox[1] + (q - i0 * e1);
        const int t = D == 3 ? l0 * G::XS + l1 * T + l2 : l0 * T + l1;
        R4 sum = zero4;
#pragma unroll
        for (int k = 0; k < NWARP; ++k) {
          const R4 v = ptile[k * TNP + t];
          sum.x += v.x;
          sum.y += v.y;
          sum.z += v.z;
          sum.w += v.w;
          ptile[k * TNP + t] = zero4;
        }
        if (sum.x == (R)0) continue;
        const int g0 = o[0] + l0, g1 = o[1] + l1, g2 = o[2] + l2;
        if (g0 < 0 || g0 >= K.res[0] || g1 < 0 || g1 >= K.res[1] || (D == 3 && (g2 < 0 || g2 >= K.res[2])))
          continue;
        if (SP) {
          int sl = tile_slot<D>(sslot, ob0, ob1, ob2, g0, g1, g2);
          if (sl < 0) sl = claim_slot(K.bptr, K.n_alloc, K.pool_blk, K.pool_cap, block_of<D>(K.nb, g0, g1, g2));
          if (sl >= 0)
            red_add_node(gout + node_in_slot<D>(sl, g0, g1, g2), sum.x, sum.y, sum.z, sum.w);
          else
            fl |= AQ_ST_POOL_FULL;
        } else {
          red_add_node(gout + cell_index<D>(K.res, g0, g1, g2), sum.x, sum.y, sum.z, sum.w);
        }
      }
    }
    if (tid == 0) s_next = atomicAdd(A.item_ctr, 1);
    __syncthreads();
  }
  if (fl) atomicOr(A.status, fl);
  if (nfall) atomicAdd(A.fallbacks, (unsigned long long)nfall);
  if (A.ranges && A.do_g2p && tid < NS) {  // one merge per CTA and slot
    if (s_rmax[tid] != 0ull) atomic_max_d(A.rmax + tid, ord_val(s_rmax[tid]));
    if (s_rmin[tid] != ~0ull) atomic_min_d(A.rmin + tid, ord_val(s_rmin[tid]));
  }
}

}  // namespace aq
