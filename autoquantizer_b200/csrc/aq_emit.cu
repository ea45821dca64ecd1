// Mesh voxelizer of the particle emitters (add_mesh / seed_from_voxels,
// mpm_exps/engine/mpm_solver.py:1356-1440; the voxelizer,
// mpm_exps/engine/voxelizer.py:17-119).
//
// Every triangle adds +1 (normal facing +z) or -1 to the voxels of each
// (x, y) column whose centre its xy projection covers, from z = padding up
// to the height where the column meets the triangle; voxels left positive
// are inside the mesh.  Here one warp takes one triangle and its lanes
// stride over the triangle's column box; each covered column records +-1 at
// z = padding and -+1 at its height in a difference array, and a second
// kernel turns every column into its running sum, which equals the
// reference's per-voxel increments exactly (integer arithmetic).  Floating
// point is double with every product and sum rounded on its own (no FMA
// contraction), so results agree bit for bit with a plain CPU evaluation.
#include <algorithm>

#include "aq_common.cuh"

namespace aq {
namespace {

struct V3 {
  double x, y, z;
};

__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
__device__ __forceinline__ double dot3(V3 a, V3 b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
__device__ __forceinline__ double cross2(double ax, double ay, double bx, double by) {
  return __dsub_rn(__dmul_rn(ax, by), __dmul_rn(ay, bx));
}

// floor to int of a column bound; coordinates beyond +-1e9 voxels clamp
__device__ __forceinline__ int ifloor(double x) { return (int)floor(fmin(fmax(x, -1e9), 1e9)); }

// inside_ccw (voxelizer.py:10-13): p left of (or on) all three edges
__device__ __forceinline__ bool inside_ccw(double px, double py, V3 a, V3 b, V3 c) {
  const double ax = __dsub_rn(a.x, px), ay = __dsub_rn(a.y, py);
  const double bx = __dsub_rn(b.x, px), by = __dsub_rn(b.y, py);
  const double cx = __dsub_rn(c.x, px), cy = __dsub_rn(c.y, py);
  return cross2(ax, ay, bx, by) >= 0.0 && cross2(bx, by, cx, cy) >= 0.0 && cross2(cx, cy, ax, ay) >= 0.0;
}

// voxelize_triangles (voxelizer.py:53-105) into the difference array vox
// (res[0] x res[1] x res[2] int32, zeroed by the caller).
__global__ void __launch_bounds__(256) k_voxel_tris(const double* __restrict__ tris, int64_t n_tris, int rx, int ry,
                                                    int rz, double dx, double inv_dx, int padding, double jitter_scale,
                                                    int32_t* __restrict__ vox) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  // the reference's fixed vertex jitter, which keeps column centres off edges
  const V3 jit = {__dmul_rn(-0.057616723909439505, jitter_scale), __dmul_rn(-0.25608986292614977, jitter_scale),
                  __dmul_rn(0.06716309129743714, jitter_scale)};
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < n_tris; t += warps) {
    const double* T = tris + 9 * t;
    const V3 a = {__dadd_rn(T[0], jit.x), __dadd_rn(T[1], jit.y), __dadd_rn(T[2], jit.z)};
    const V3 b = {__dadd_rn(T[3], jit.x), __dadd_rn(T[4], jit.y), __dadd_rn(T[5], jit.z)};
    const V3 c = {__dadd_rn(T[6], jit.x), __dadd_rn(T[7], jit.y), __dadd_rn(T[8], jit.z)};
    const double lo0 = fmin(fmin(a.x, b.x), c.x), hi0 = fmax(fmax(a.x, b.x), c.x);
    const double lo1 = fmin(fmin(a.y, b.y), c.y), hi1 = fmax(fmax(a.y, b.y), c.y);
    const int p_min = max(padding, ifloor(__dmul_rn(lo0, inv_dx)));
    const int p_max = min(rx - padding, ifloor(__dmul_rn(hi0, inv_dx)) + 1);
    const int q_min = max(padding, ifloor(__dmul_rn(lo1, inv_dx)));
    const int q_max = min(ry - padding, ifloor(__dmul_rn(hi1, inv_dx)) + 1);
    // normalized() of (b - a) x (c - a): times the reciprocal of its length
    const V3 e1 = sub3(b, a), e2 = sub3(c, a);
    V3 nrm = {__dsub_rn(__dmul_rn(e1.y, e2.z), __dmul_rn(e1.z, e2.y)),
              __dsub_rn(__dmul_rn(e1.z, e2.x), __dmul_rn(e1.x, e2.z)),
              __dsub_rn(__dmul_rn(e1.x, e2.y), __dmul_rn(e1.y, e2.x))};
    const double inv_len = __ddiv_rn(1.0, __dsqrt_rn(dot3(nrm, nrm)));
    nrm = {__dmul_rn(nrm.x, inv_len), __dmul_rn(nrm.y, inv_len), __dmul_rn(nrm.z, inv_len)};
    if (!(fabs(nrm.z) >= 1e-10)) continue;  // also skips degenerate (NaN) triangles
    const int np = p_max - p_min, nq = q_max - q_min;
    if (np <= 0 || nq <= 0) continue;
    const int inc = nrm.z > 0 ? 1 : -1;
    const int64_t cells = (int64_t)np * nq;
    for (int64_t k = lane; k < cells; k += 32) {
      const int p = p_min + (int)(k / nq), q = q_min + (int)(k % nq);
      const double px = __dmul_rn(__dadd_rn((double)p, 0.5), dx), py = __dmul_rn(__dadd_rn((double)q, 0.5), dx);
      if (!(inside_ccw(px, py, a, b, c) || inside_ccw(px, py, a, c, b))) continue;
      const V3 base = {px, py, 0.0};
      const double h = __dadd_rn(__dmul_rn(__ddiv_rn(-dot3(nrm, sub3(base, a)), nrm.z), inv_dx), 0.5);
      // min(int(h), ry - padding), int() truncating toward zero; columns
      // whose height is at most padding get nothing
      if (!(h >= (double)(padding + 1))) continue;
      const int height = h >= (double)(ry - padding) ? ry - padding : (int)h;
      if (height <= padding) continue;
      int32_t* col = vox + ((int64_t)p * ry + q) * rz;
      atomicAdd(col + padding, inc);
      if (height < rz) atomicAdd(col + height, -inc);
    }
  }
}

// running sum along z of every (x, y) column
__global__ void __launch_bounds__(256) k_voxel_prefix(int32_t* __restrict__ vox, int64_t cols, int rz) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t* v = vox + c * rz;
    int32_t run = 0;
    for (int z = 0; z < rz; ++z) {
      run += v[z];
      v[z] = run;
    }
  }
}

}  // namespace
}  // namespace aq

using namespace aq;

extern "C" int aq_voxelize(const double* d_tris, int64_t n_tris, const int32_t* res, double dx, int32_t padding,
                           double jitter_scale, int32_t* d_voxels, void* stream) {
  if (!res || !d_voxels || n_tris < 0 || (n_tris > 0 && !d_tris) || !(dx > 0) || padding < 0) return AQ_E_ARG;
  for (int k = 0; k < 3; ++k)
    if (res[k] < 1 || res[k] > 65536 || 2 * padding >= res[k]) return AQ_E_ARG;
  const int64_t cols = (int64_t)res[0] * res[1], cells = cols * res[2];
  cudaStream_t st = as_stream(stream);
  AQ_CUDA_TRY(cudaMemsetAsync(d_voxels, 0, sizeof(int32_t) * cells, st));
  if (n_tris > 0) {
    const unsigned nb = (unsigned)std::min<int64_t>(grid_for(n_tris * 32, 256), (int64_t)num_sms() * 16);
    k_voxel_tris<<<nb, 256, 0, st>>>(d_tris, n_tris, res[0], res[1], res[2], dx, 1.0 / dx, padding, jitter_scale,
                                     d_voxels);
    AQ_CUDA_TRY(cudaGetLastError());
  }
  const unsigned nb = (unsigned)std::min<int64_t>(grid_for(cols, 256), (int64_t)num_sms() * 8);
  k_voxel_prefix<<<nb, 256, 0, st>>>(d_voxels, cols, res[2]);
  AQ_CUDA_TRY(cudaGetLastError());
  return AQ_OK;
}
