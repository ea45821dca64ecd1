/*
 * ORACLE - test infrastructure only.  CPU restatement of the reference's
 * quantized-state MLS-MPM path.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it, and only as a
 * checker or as the timed CPU baseline; the product (libaq.so) never calls it.
 *
 * What it restates (paths inside the AutoQuantizer repository):
 *   layout      taichi_submission/taichi/struct/struct_llvm.cpp:77-116,
 *               taichi_submission/taichi/program/snode_expr_utils.cpp:30-92
 *   fixed codec codegen_llvm_quant.cpp:44-80 (float_to_custom_int),
 *               :166-184 (custom_type_to_bits), :582-621 (extract by mask),
 *               :624-641 (reconstruct_custom_float), :834-878 (load_split),
 *               runtime.cpp:1732-1762 (rounding_prepare*, dithering)
 *   exp floats  codegen_llvm_quant.cpp:229-305 (own exponent store),
 *               :347-499 (shared exponent store), :660-757 (reconstruct)
 *   bit_pack    codegen_llvm_quant.cpp:884-952 (BitPackAssignStmt)
 *   substep     mpm_exps/engine/mpm_solver.py:590-758, 1012-1031, 1043-1052
 *   polar 2D    taichi_submission/python/taichi/lang/linalg_impl.py:9-26
 *   collider    mpm_exps/engine/mpm_solver.py:1459-1547 (in aq_oracle_mpm.c)
 *   voxelizer   mpm_exps/engine/voxelizer.py:10-105 (aq_oracle_emit.c;
 *               pinned by the reference's shipped letters emission,
 *               tests/golden/letters_voxels.npz, and known-answer meshes)
 * Parity of this restatement is pinned by the reference's own quant tests
 * (taichi_submission/tests/python/test_bit_pack*.py, test_dithering.py,
 * test_custom_float*.py, test_fxp_offset.py) ported in tests/.
 */
#ifndef AQ_ORACLE_H_
#define AQ_ORACLE_H_
#include <stdint.h>

#define OR_MAX_SLOTS 32
#define OR_MAX_GROUPS 4

enum { OR_FIXED = 0, OR_INT = 1, OR_FLOAT_EXP = 2, OR_SHARED_EXP = 3, OR_RAW_F32 = 4, OR_RAW_F64 = 5 };

typedef struct or_layout {
  int n, n_words, total_bits, compute_f64, dither, n_groups;
  int kind[OR_MAX_SLOTS], bits[OR_MAX_SLOTS], sgn[OR_MAX_SLOTS], ebits[OR_MAX_SLOTS];
  int off[OR_MAX_SLOTS], eoff[OR_MAX_SLOTS], group[OR_MAX_SLOTS], efirst[OR_MAX_SLOTS];
  double scale[OR_MAX_SLOTS], offset[OR_MAX_SLOTS];
} or_layout;

typedef struct or_params {
  int dim, precision, res[3], has_F, has_mat, n_mat, friction, bound_clip;
  double dx, dt, p_vol, p_mass, g, lb[3], ub[3];
  int mat_kind[4];
  double mat_mu[4], mat_lam[4];
  uint64_t seed;
  int threads; /* OpenMP threads for the timed baseline; <=1 = serial, deterministic */
  /* rotating SDF collider (mpm_solver.py:1459-1547), 3D; col_on = 0: none.
   * col_c, col_s: cos and sin of this substep's angle (float in the f32
   * simulator), col_yshift = int(height / dx + 0.5) */
  int col_on, col_n, col_dims[3], col_off[3], col_yshift;
  double col_c, col_s, col_omega;
  const float* col_sdf;
  const float* col_nrm;
  /* 1: collider velocity omega x r with r from the node itself
   * (sdf_collision_no_arg, mpm_solver.py:1482-1512); 0: from the rotated
   * index (sdf_collision, :1459-1480) */
  int col_node_cv;
} or_params;

void or_voxelize(const double* tris, int64_t n_tris, const int32_t* res, double dx, int32_t padding,
                 double jitter_scale, int32_t* vox);

#endif
