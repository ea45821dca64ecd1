/*
 * ORACLE - test infrastructure only (see aq_oracle.h).  Scalar CPU
 * restatement of MPMSolver.substep (mpm_exps/engine/mpm_solver.py:624-631):
 * P2G (:590-622), grid_op (:633-665), G2P (:667-758), compute_cauchy
 * (:1012-1031), compute_ek (:1043-1052), over records encoded with the
 * bit_pack codec of aq_oracle_codec.c.  Compiled twice: REAL=float (_f32)
 * and REAL=double (_f64), as the reference runs with default_fp f32 (3D
 * drivers) or f64 (2D drivers).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "aq_oracle.h"
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#define SUF(x) x##_f64
#endif

typedef REAL R;

void or_encode_record(const or_layout* L, const double* vals, uint64_t* w, uint64_t pk,
                      const double* uniforms);
void or_decode_record(const or_layout* L, const uint64_t* w, double* vals);
uint64_t or_step_key(uint64_t seed, int64_t step);
uint64_t or_particle_key(uint64_t step_key, int32_t pid);

#define MAXS OR_MAX_SLOTS

static R SUF(det)(int D, const R* F) {
  if (D == 2) return F[0] * F[3] - F[1] * F[2];
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
         F[2] * (F[3] * F[7] - F[4] * F[6]);
}

/* polar_decompose2d (linalg_impl.py:9-26) */
static void SUF(polar2)(const R* A, R* Rm) {
  R x = A[0] + A[3], y = A[2] - A[1];
  R scale = (R)1.0 / (R)sqrt(x * x + y * y);
  R c = x * scale, s = y * scale;
  Rm[0] = c;
  Rm[1] = -s;
  Rm[2] = s;
  Rm[3] = c;
}

/* Rotation factor of a 3x3 polar decomposition by Newton's iteration
 * X <- (X + X^-T)/2 (Higham 1986); used only by the fixed-corotated 3D
 * material, which the reference does not have. */
static void SUF(polar3)(const R* A, R* X) {
  for (int k = 0; k < 9; ++k) X[k] = A[k];
  const R tol = sizeof(R) == 4 ? (R)1e-6 : (R)1e-12;
  for (int it = 0; it < 20; ++it) {
    R c00 = X[4] * X[8] - X[5] * X[7], c01 = X[5] * X[6] - X[3] * X[8], c02 = X[3] * X[7] - X[4] * X[6];
    R c10 = X[2] * X[7] - X[1] * X[8], c11 = X[0] * X[8] - X[2] * X[6], c12 = X[1] * X[6] - X[0] * X[7];
    R c20 = X[1] * X[5] - X[2] * X[4], c21 = X[2] * X[3] - X[0] * X[5], c22 = X[0] * X[4] - X[1] * X[3];
    R d = X[0] * c00 + X[1] * c01 + X[2] * c02;
    R id = (R)1.0 / d; /* X^-T = cofactor / det */
    R Y[9] = {c00 * id, c01 * id, c02 * id, c10 * id, c11 * id, c12 * id, c20 * id, c21 * id, c22 * id};
    R diff = 0;
    for (int k = 0; k < 9; ++k) {
      R nx = (R)0.5 * (X[k] + Y[k]);
      diff += (nx - X[k]) * (nx - X[k]);
      X[k] = nx;
    }
    if (diff < tol * tol) break;
  }
}

typedef struct {
  int D, has_F, has_mat, nslots;
  R inv_dx, dx, dt, p_mass, stress_coef, four_inv_dx, g;
  R lbx[3], ubx[3];
} SUF(consts);

static void SUF(cauchy)(const or_params* P, int D, int mk, double mu, double lam, const R* F, R J,
                        int has_F, R* out) {
  for (int k = 0; k < D * D; ++k) out[k] = 0;
  if (mk == 0) { /* fluid: diag(la*(J-1)) */
    R Jf = has_F ? SUF(det)(D, F) : J;
    for (int d = 0; d < D; ++d) out[d * D + d] = (R)lam * (Jf - (R)1.0);
    return;
  }
  R Jd = SUF(det)(D, F);
  if (D == 2 || mk == 2) {
    R Rm[9];
    if (D == 2)
      SUF(polar2)(F, Rm);
    else
      SUF(polar3)(F, Rm);
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {
        R s = 0;
        for (int k = 0; k < D; ++k) s += (F[i * D + k] - Rm[i * D + k]) * F[j * D + k];
        out[i * D + j] = (R)2.0 * (R)mu * s + (i == j ? (R)lam * Jd * (Jd - (R)1.0) : (R)0.0);
      }
  } else { /* reference 3D law: mu(FF^T - I) + la*log(J) on every entry */
    R lj = (R)lam * (R)log(Jd);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        R s = 0;
        for (int k = 0; k < 3; ++k) s += F[i * 3 + k] * F[j * 3 + k];
        out[i * 3 + j] = (R)mu * (s - (i == j ? (R)1.0 : (R)0.0)) + lj;
      }
  }
}

static void SUF(unpack)(int D, int has_F, const double* vals, R* x, R* v, R* C, R* F, R* J, int* mat,
                        int has_mat) {
  int s = 0;
  for (int d = 0; d < D; ++d) x[d] = (R)vals[s++];
  for (int d = 0; d < D; ++d) v[d] = (R)vals[s++];
  for (int k = 0; k < D * D; ++k) C[k] = (R)vals[s++];
  if (has_F) {
    for (int k = 0; k < D * D; ++k) F[k] = (R)vals[s++];
    *J = 1;
  } else {
    *J = (R)vals[s++];
  }
  *mat = has_mat ? (int)vals[s] : 0;
}

static int SUF(base_of)(R xv, R inv_dx, int res, int* flags) {
  R t = xv * inv_dx - (R)0.5;
  if (t != t) {
    *flags |= 2;
    return 0;
  }
  int b = (int)floor(t);
  if (b < 0) {
    *flags |= 1;
    b = 0;
  }
  if (b > res - 3) {
    *flags |= 1;
    b = res - 3;
  }
  return b;
}

/* One substep over n records.  grid: ncells*4 REAL scratch.  ranges_max/min
 * (optional, n_slots each) accumulate the decoded new state.  Returns the
 * status flags (1 = out of domain, 2 = NaN). */
/* grid post-process of the rotating SDF collider: rot_scene
 * (mpm_solver.py:1515-1540) then sdf_collision (:1459-1480), or
 * sdf_collision_no_arg (:1482-1512) when col_node_cv is set */
static void SUF(collide)(const or_params* P, const int* I, R* v) {
  const int n = P->col_n;
  const int i0 = I[0] >= 2 * n ? I[0] - 2 * n : I[0], i2 = I[2] >= 2 * n ? I[2] - 2 * n : I[2];
  const R c = (R)P->col_c, s = (R)P->col_s;
  const R o0 = (R)(i0 - n), o2 = (R)(i2 - n);
  const R x = c * o0 - s * o2 + (R)n + (R)0.5;
  const R z = s * o0 + c * o2 + (R)n + (R)0.5;
  int r[3] = {(int)x, I[1] - P->col_yshift, (int)z};
  for (int k = 0; k < 3; ++k) {
    const int lo = (int)P->lb[k], hi = (int)P->ub[k];
    r[k] = r[k] > hi ? hi : r[k];
    r[k] = r[k] < lo ? lo : r[k];
  }
  const int a = r[0] - P->col_off[0], b = r[1] - P->col_off[1], e = r[2] - P->col_off[2];
  if (a < 0 || a >= P->col_dims[0] || b < 0 || b >= P->col_dims[1] || e < 0 || e >= P->col_dims[2]) return;
  const int64_t q = ((int64_t)a * P->col_dims[1] + b) * P->col_dims[2] + e;
  if (!(P->col_sdf[q] < -1e-5f)) return; /* sdf(): the value where below -1e-5, else 1 */
  const R g0 = (R)P->col_nrm[3 * q], g1 = (R)P->col_nrm[3 * q + 1], g2 = (R)P->col_nrm[3 * q + 2];
  const R nrm[3] = {c * g0 + s * g2, g1, -s * g0 + c * g2};
  const R dx = (R)P->dx, om = (R)P->col_omega;
  const int px = P->col_node_cv ? I[0] : r[0], pz = P->col_node_cv ? I[2] : r[2];
  const R rx = (R)(px - n) * dx, rz = (R)(pz - n) * dx;
  const R cv[3] = {om * rz, (R)0, -om * rx}; /* (0, omega, 0) x r */
  R vr[3], dn = 0;
  for (int k = 0; k < 3; ++k) {
    vr[k] = v[k] - cv[k];
    dn += vr[k] * nrm[k];
  }
  dn = dn < (R)0 ? dn : (R)0;
  for (int k = 0; k < 3; ++k) v[k] = cv[k] + (vr[k] - dn * nrm[k]);
}

int SUF(or_substep)(const or_params* P, const or_layout* L, uint64_t* words, const int32_t* pid,
                    int64_t n, int64_t step, R* grid, double* vals_scratch, double* rmax,
                    double* rmin) {
  const int D = P->dim, W = L->n_words, NS = L->n;
  const int rx = P->res[0], ry = P->res[1], rz = D == 3 ? P->res[2] : 1;
  const int64_t ncell = (int64_t)rx * ry * rz;
  const R inv_dx = (R)(1.0 / P->dx), dx = (R)P->dx, dt = (R)P->dt, p_mass = (R)P->p_mass;
  const R stress_coef = (R)(-(P->dt * P->p_vol * 4.0 * (1.0 / P->dx) * (1.0 / P->dx)));
  const R four_inv_dx = (R)(4.0 * (1.0 / P->dx));
  const R g = (R)P->g;
  int flags = 0;
  int nthreads = P->threads > 1 ? P->threads : 1;
  (void)nthreads;

  for (int64_t p = 0; p < n; ++p) or_decode_record(L, words + p * W, vals_scratch + p * NS);
  memset(grid, 0, sizeof(R) * 4 * (size_t)ncell);

  /* ---- P2G (p2g_bls, mpm_solver.py:590-622) ---- */
#pragma omp parallel for num_threads(nthreads) reduction(| : flags) schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    R x[3], v[3], C[9], F[9], J;
    int mat;
    SUF(unpack)(D, P->has_F, vals_scratch + p * NS, x, v, C, F, &J, &mat, P->has_mat);
    int base[3] = {0, 0, 0};
    R fx[3] = {0, 0, 0}, w[3][3];
    int res3[3] = {rx, ry, rz};
    for (int d = 0; d < D; ++d) {
      base[d] = SUF(base_of)(x[d], inv_dx, res3[d], &flags);
      fx[d] = x[d] * inv_dx - (R)base[d];
      w[0][d] = (R)0.5 * ((R)1.5 - fx[d]) * ((R)1.5 - fx[d]);
      w[1][d] = (R)0.75 - (fx[d] - (R)1.0) * (fx[d] - (R)1.0);
      w[2][d] = (R)0.5 * (fx[d] - (R)0.5) * (fx[d] - (R)0.5);
    }
    int mk = P->mat_kind[mat & 3];
    R cau[9], aff[9];
    SUF(cauchy)(P, D, mk, P->mat_mu[mat & 3], P->mat_lam[mat & 3], F, J, P->has_F, cau);
    for (int k = 0; k < D * D; ++k) aff[k] = stress_coef * cau[k] + p_mass * C[k];
    int n3 = D == 3 ? 27 : 9;
    for (int o = 0; o < n3; ++o) {
      int off[3] = {D == 3 ? o / 9 : o / 3, D == 3 ? (o / 3) % 3 : o % 3, D == 3 ? o % 3 : 0};
      R dpos[3], weight = 1;
      for (int d = 0; d < D; ++d) {
        dpos[d] = ((R)off[d] - fx[d]) * dx;
        weight *= w[off[d]][d];
      }
      int64_t cell = ((int64_t)(base[0] + off[0]) * ry + (base[1] + off[1])) * rz + (D == 3 ? base[2] + off[2] : 0);
      R* gc = grid + 4 * cell;
      for (int d = 0; d < D; ++d) {
        R ad = 0;
        for (int e = 0; e < D; ++e) ad += aff[d * D + e] * dpos[e];
        R c = weight * (p_mass * v[d] + ad);
#pragma omp atomic
        gc[1 + d] += c;
      }
      R cm = weight * p_mass;
#pragma omp atomic
      gc[0] += cm;
    }
  }

  /* ---- grid_op (mpm_solver.py:633-665) ---- */
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int64_t c = 0; c < ncell; ++c) {
    int I[3] = {(int)(c / ((int64_t)ry * rz)), (int)((c / rz) % ry), (int)(c % rz)};
    R* gc = grid + 4 * c;
    R inv_m = (R)1.0 / (gc[0] + (R)1e-10);
    R vo[3] = {0, 0, 0};
    for (int d = 0; d < D; ++d) vo[d] = inv_m * gc[1 + d];
    vo[1] -= dt * g;
    if (P->friction) {
      if (I[1] < P->lb[1] && vo[1] < 0) {
        R nv = vo[1]; /* n = (0,1,0): v - n (n.v), then * 0.02 */
        vo[1] = vo[1] - nv;
        for (int d = 0; d < D; ++d) vo[d] = vo[d] * (R)0.02;
      }
    }
    for (int k = 0; k < D; ++k) {
      if (I[k] < P->lb[k] && vo[k] < 0) vo[k] = 0;
      if (I[k] > P->ub[k] && vo[k] > 0) vo[k] = 0;
    }
    if (D == 3 && P->col_on) SUF(collide)(P, I, vo);
    for (int d = 0; d < D; ++d) gc[1 + d] = vo[d];
  }

  /* ---- G2P (g2p_bls, mpm_solver.py:667-758) ---- */
  const uint64_t sk = or_step_key(P->seed, step);
#pragma omp parallel for num_threads(nthreads) reduction(| : flags) schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    R x[3], v[3], C[9], F[9], J;
    int mat;
    SUF(unpack)(D, P->has_F, vals_scratch + p * NS, x, v, C, F, &J, &mat, P->has_mat);
    int base[3] = {0, 0, 0};
    R fx[3] = {0, 0, 0}, w[3][3];
    int res3[3] = {rx, ry, rz};
    for (int d = 0; d < D; ++d) {
      base[d] = SUF(base_of)(x[d], inv_dx, res3[d], &flags);
      fx[d] = x[d] * inv_dx - (R)base[d];
      w[0][d] = (R)0.5 * ((R)1.5 - fx[d]) * ((R)1.5 - fx[d]);
      w[1][d] = (R)0.75 - (fx[d] - (R)1.0) * (fx[d] - (R)1.0);
      w[2][d] = (R)0.5 * (fx[d] - (R)0.5) * (fx[d] - (R)0.5);
    }
    R nv[3] = {0, 0, 0}, nC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int n3 = D == 3 ? 27 : 9;
    for (int o = 0; o < n3; ++o) {
      int off[3] = {D == 3 ? o / 9 : o / 3, D == 3 ? (o / 3) % 3 : o % 3, D == 3 ? o % 3 : 0};
      R dpos[3], weight = 1;
      for (int d = 0; d < D; ++d) {
        dpos[d] = (R)off[d] - fx[d];
        weight *= w[off[d]][d];
      }
      int64_t cell = ((int64_t)(base[0] + off[0]) * ry + (base[1] + off[1])) * rz + (D == 3 ? base[2] + off[2] : 0);
      const R* gc = grid + 4 * cell;
      R s = four_inv_dx * weight;
      for (int d = 0; d < D; ++d) {
        nv[d] += weight * gc[1 + d];
        for (int e = 0; e < D; ++e) nC[d * D + e] += s * (gc[1 + d] * dpos[e]);
      }
    }
    double out[MAXS];
    int s = 0;
    for (int d = 0; d < D; ++d) {
      R nx = x[d] + dt * nv[d];
      if (P->bound_clip) {
        R hi = (R)(P->ub[d] * P->dx), lo = (R)(P->lb[d] * P->dx);
        nx = nx < hi ? nx : hi;
        nx = nx > lo ? nx : lo;
      }
      out[s++] = (double)nx;
    }
    for (int d = 0; d < D; ++d) out[s++] = (double)nv[d];
    for (int k = 0; k < D * D; ++k) out[s++] = (double)nC[k];
    int mk = P->mat_kind[mat & 3];
    if (P->has_F) {
      R A[9], nF[9];
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) A[i * D + j] = (i == j ? (R)1.0 : (R)0.0) + dt * nC[i * D + j];
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
          R acc = 0;
          for (int k = 0; k < D; ++k) acc += A[i * D + k] * F[k * D + j];
          nF[i * D + j] = acc;
        }
      if (mk == 0 && P->has_mat) { /* fluid particle in an F record: keep only J */
        R Jn = SUF(det)(D, nF);
        R sj = (R)pow((double)Jn, 1.0 / D);
        for (int i = 0; i < D; ++i)
          for (int j = 0; j < D; ++j) nF[i * D + j] = i == j ? sj : (R)0.0;
      }
      for (int k = 0; k < D * D; ++k) out[s++] = (double)nF[k];
    } else {
      R tr = 0;
      for (int d = 0; d < D; ++d) tr += nC[d * D + d];
      out[s++] = (double)(((R)1.0 + dt * tr) * J);
    }
    if (P->has_mat) out[s++] = (double)mat;
    or_encode_record(L, out, words + p * W, or_particle_key(sk, pid ? pid[p] : (int32_t)p), NULL);
  }

  if (rmax && rmin) {
    for (int64_t p = 0; p < n; ++p) {
      double vv[MAXS];
      or_decode_record(L, words + p * W, vv);
      for (int s = 0; s < NS; ++s) {
        if (vv[s] > rmax[s]) rmax[s] = vv[s];
        if (vv[s] < rmin[s]) rmin[s] = vv[s];
      }
    }
  }
  return flags;
}

/* compute_ek (mpm_solver.py:1043-1052) over decoded records. */
double SUF(or_loss_ek)(const or_params* P, const or_layout* L, const uint64_t* words, int64_t n) {
  const int D = P->dim;
  double vals[MAXS];
  R acc = 0;
  for (int64_t p = 0; p < n; ++p) {
    or_decode_record(L, words + p * L->n_words, vals);
    R vv = 0;
    for (int d = 0; d < D; ++d) vv += (R)vals[D + d] * (R)vals[D + d];
    if (D == 3) {
      acc += (R)0.5 * (R)P->p_mass * vv;
      acc += (R)P->g * (R)P->p_mass * (R)vals[1];
    } else {
      acc += vv;
    }
  }
  return (double)acc;
}
