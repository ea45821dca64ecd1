/* ORACLE - test infrastructure only (never linked into the library).
 *
 * CPU restatement of the mesh voxelizer that the particle emitters use
 * (mpm_exps/engine/voxelizer.py:53-105, voxelize_triangles, with fill at
 * :47-51 and inside_ccw at :10-13), written as the reference states it: a
 * loop over triangles, over the columns of each triangle's xy bounding box,
 * and the per-voxel fill of every covered column.  Double precision, each
 * operation rounded on its own (-ffp-contract=off). */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "aq_oracle.h"

static double cross2(double ax, double ay, double bx, double by) { return ax * by - ay * bx; }

static int inside_ccw(double px, double py, const double* a, const double* b, const double* c) {
  return cross2(a[0] - px, a[1] - py, b[0] - px, b[1] - py) >= 0.0 &&
         cross2(b[0] - px, b[1] - py, c[0] - px, c[1] - py) >= 0.0 &&
         cross2(c[0] - px, c[1] - py, a[0] - px, a[1] - py) >= 0.0;
}

static int ifloor(double x) { return (int)floor(fmin(fmax(x, -1e9), 1e9)); }
static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

void or_voxelize(const double* tris, int64_t n_tris, const int32_t* res, double dx, int32_t padding,
                 double jitter_scale, int32_t* vox) {
  const int rx = res[0], ry = res[1], rz = res[2];
  const double inv_dx = 1.0 / dx;
  const double jit[3] = {-0.057616723909439505 * jitter_scale, -0.25608986292614977 * jitter_scale,
                         0.06716309129743714 * jitter_scale};
  memset(vox, 0, sizeof(int32_t) * (size_t)rx * ry * rz);
  for (int64_t t = 0; t < n_tris; ++t) {
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) {
      a[k] = tris[9 * t + k] + jit[k];
      b[k] = tris[9 * t + 3 + k] + jit[k];
      c[k] = tris[9 * t + 6 + k] + jit[k];
    }
    const double lo0 = fmin(fmin(a[0], b[0]), c[0]), hi0 = fmax(fmax(a[0], b[0]), c[0]);
    const double lo1 = fmin(fmin(a[1], b[1]), c[1]), hi1 = fmax(fmax(a[1], b[1]), c[1]);
    const int p_min = imax(padding, ifloor(lo0 * inv_dx)), p_max = imin(rx - padding, ifloor(hi0 * inv_dx) + 1);
    const int q_min = imax(padding, ifloor(lo1 * inv_dx)), q_max = imin(ry - padding, ifloor(hi1 * inv_dx) + 1);
    const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const double inv_len = 1.0 / sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int k = 0; k < 3; ++k) n[k] = n[k] * inv_len;
    if (!(fabs(n[2]) >= 1e-10)) continue;
    for (int p = p_min; p < p_max; ++p)
      for (int q = q_min; q < q_max; ++q) {
        const double px = (p + 0.5) * dx, py = (q + 0.5) * dx;
        if (!(inside_ccw(px, py, a, b, c) || inside_ccw(px, py, a, c, b))) continue;
        const double d = n[0] * (px - a[0]) + n[1] * (py - a[1]) + n[2] * (0.0 - a[2]);
        const double h = -d / n[2] * inv_dx + 0.5;
        if (!(h >= (double)(padding + 1))) continue;
        const int height = h >= (double)(ry - padding) ? ry - padding : (int)h;
        const int inc = n[2] > 0 ? 1 : -1;
        for (int i = padding; i < height && i < rz; ++i) vox[((int64_t)p * ry + q) * rz + i] += inc;
      }
  }
}
