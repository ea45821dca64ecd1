/*
 * aq.h - C ABI of libaq.so, the B200 (sm_100a) implementation of the quantized
 * MLS-MPM substep (P2G -> grid update -> G2P) over bit_pack particle records.
 *
 * Conventions
 *   - Every entry point returns int: 0 = ok, negative = error (see AQ_E_*).
 *     No entry point aborts the process.
 *   - Pointers named d_* are CUDA device pointers; h_* are host pointers.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Calls are stream-ordered; a handle is not thread-safe.
 *   - Buffers passed in are caller-owned.  An aq_sim owns its particle
 *     records, grids and binning scratch and frees them in aq_sim_destroy.
 *
 * Each declaration names the reference interface it replaces (path inside the
 * AutoQuantizer repository, file:line).
 */
#ifndef AQ_H_
#define AQ_H_

#ifdef __CUDACC_RTC__
/* NVRTC (layout-specialized kernel compilation) has no libc headers */
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#else
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define AQ_ABI_VERSION 1
#define AQ_MAX_SLOTS 32  /* scalars per particle record */
#define AQ_MAX_GROUPS 4  /* shared-exponent groups per record */
#define AQ_MAX_MATERIALS 4

/* error codes */
#define AQ_OK 0
#define AQ_E_ARG (-1)      /* bad argument (null pointer, size, bit width) */
#define AQ_E_LAYOUT (-2)   /* layout does not fit the simulator schema */
#define AQ_E_CUDA (-3)     /* a CUDA runtime call failed */
#define AQ_E_NOMEM (-4)    /* device allocation failed */
#define AQ_E_STATE (-5)    /* call not valid in the current state */
#define AQ_E_LIMIT (-6)    /* size above a documented maximum */

/* device status flags (aq_sim_status) */
#define AQ_ST_OUT_OF_DOMAIN 0x1u  /* a particle stencil left the grid; base clamped */
#define AQ_ST_NAN 0x2u            /* a NaN position was met; base clamped */
#define AQ_ST_FALLBACK 0x4u       /* a particle left its shared-memory tile (informational) */
#define AQ_ST_POOL_FULL 0x8u      /* sparse grid: no free node block; contributions to it were dropped */

/* scalar kinds: quantized types of the reference
 *   AQ_FIXED      ti.quant.fixed(frac=bits, signed, range, offset)
 *                 (taichi_submission/python/taichi/lang/quant_impl.py:28-50)
 *   AQ_INT        ti.quant.int(bits, signed)          (quant_impl.py:12-26)
 *   AQ_FLOAT_EXP  ti.quant.float(exp, frac, signed): own exponent
 *                 (quant_impl.py:52-73, codegen_llvm_quant.cpp:229-305)
 *   AQ_SHARED_EXP custom float whose exponent is shared by its group
 *                 (snode.py place(..., shared_exponent=True), :151-180;
 *                 codegen_llvm_quant.cpp:347-499)
 *   AQ_RAW_F32 / AQ_RAW_F64  unquantized IEEE value stored in the record */
enum {
  AQ_FIXED = 0,
  AQ_INT = 1,
  AQ_FLOAT_EXP = 2,
  AQ_SHARED_EXP = 3,
  AQ_RAW_F32 = 4,
  AQ_RAW_F64 = 5
};

/* One scalar of a particle record, in place order. */
typedef struct aq_scalar_spec {
  int32_t kind;
  int32_t bits;      /* digits incl. sign bit, 1..32 (RAW: ignored) */
  int32_t is_signed;
  int32_t exp_bits;  /* FLOAT_EXP / SHARED_EXP: exponent bits, 1..8 */
  int32_t group;     /* SHARED_EXP: members with equal id share one exponent */
  int32_t _pad;
  double range;      /* FIXED: scale = range/2^(bits-1) (signed) or range/2^bits */
  double offset;     /* FIXED: value = code*scale + offset */
} aq_scalar_spec;

/* Resolved slot: bit positions inside the record and derived constants. */
typedef struct aq_slot {
  int32_t kind, bits, is_signed, exp_bits;
  int32_t bit_offset;  /* first bit of the digits (little-endian bit stream) */
  int32_t exp_offset;  /* first bit of the exponent (FLOAT_EXP, SHARED_EXP) */
  int32_t group;       /* SHARED_EXP: dense group index */
  int32_t exp_first;   /* SHARED_EXP: the group exponent precedes this slot */
  float scale_f32, inv_scale_f32, offset_f32, _pad2;
  double scale_f64, inv_scale_f64, offset_f64, _pad3;
} aq_slot;

typedef struct aq_layout {
  int32_t n_slots, n_words, total_bits, compute_f64, use_dithering, n_groups;
  int32_t _pad[2];
  aq_slot slot[AQ_MAX_SLOTS];
} aq_layout;

#ifndef __CUDACC_RTC__ /* declarations only: NVRTC sees the types */
/* Build a bit_pack record layout: fields are packed in place order into a
 * little-endian stream of 64-bit words; a field may straddle two words; a
 * shared exponent is placed right before the first member of its group.
 * Replaces the bit_pack layout pass taichi_submission/taichi/struct/
 * struct_llvm.cpp:77-116 and place_child in
 * taichi_submission/taichi/program/snode_expr_utils.cpp:30-92. */
int aq_layout_build(int32_t n_scalars, const aq_scalar_spec* h_specs,
                    int32_t compute_f64, int32_t use_dithering,
                    aq_layout* h_out);

/* Encode n records.  d_values is n x n_slots (f32, or f64 if values_f64).
 * Dithering (layout.use_dithering) draws the uniform of slot s of particle
 * d_pid[i] (or i when d_pid is NULL) at substep `step` from the counter-based
 * generator keyed on (seed, step, pid, slot); d_uniforms (n x n_slots, compute
 * type), when non-NULL, supplies the uniforms instead.
 * Replaces ti.bit_pack_assign (taichi_submission/python/taichi/lang/
 * impl.py:753-756) lowered by CodeGenLLVM::visit(BitPackAssignStmt)
 * (codegen_llvm_quant.cpp:884-952), float_to_custom_int (:44-80),
 * custom_type_to_bits (:166-184) and rounding_prepare_f{32,64}[_with_dithering]
 * (taichi_submission/taichi/runtime/llvm/runtime.cpp:1732-1762). */
int aq_encode(const aq_layout* h_layout, const void* d_values, int32_t values_f64,
              uint64_t* d_words, int64_t n, const int32_t* d_pid, uint64_t seed,
              int64_t step, const void* d_uniforms, void* stream);

/* Decode n records into d_values (n x n_slots).
 * Replaces load_custom_float / load_as_custom_int / load_split /
 * reconstruct_custom_float[_with_exponent] (codegen_llvm_quant.cpp:529-878). */
int aq_decode(const aq_layout* h_layout, const uint64_t* d_words, void* d_values,
              int32_t values_f64, int64_t n, void* stream);
#endif

/* ---------------------------------------------------------------- simulator */

enum { AQ_MAT_FLUID = 0, AQ_MAT_ELASTIC = 1, AQ_MAT_COROTATED = 2 };

/* AQ_MAT_FLUID:     cauchy = diag(lam*(J-1))
 * AQ_MAT_ELASTIC:   the reference's elastic law: 2D fixed-corotated
 *                   2mu(F-R)F^T + lam J(J-1) I; 3D mu(FF^T-I) + lam log J
 *                   added to every entry (mpm_solver.py:1012-1031)
 * AQ_MAT_COROTATED: fixed-corotated in 2D and 3D (3D via a 3x3 polar
 *                   decomposition); not a reference material */
typedef struct aq_material {
  int32_t kind, _pad;
  double mu, lam;
} aq_material;

typedef struct aq_params {
  int32_t dim;         /* 2 or 3 */
  int32_t precision;   /* 0: f32 grid and arithmetic, 1: f64 */
  int32_t res[3];      /* grid cells per axis */
  int32_t has_F;       /* record holds F (dim*dim) after C, else J (1) */
  int32_t has_mat;     /* record holds a material-id INT slot last */
  int32_t n_materials;
  int32_t use_friction, use_bound_clip;
  int32_t sort_interval; /* re-bin particles every k substeps (>=1) */
  int32_t jit;           /* 1: compile the substep kernel for this layout with
                            NVRTC (default), 0: nvcc-built generic kernel */
  double dx, dt, p_vol, p_mass, gravity;
  double lb[3], ub[3]; /* grid-index walls, as MPMSolver.lb/ub */
  aq_material mat[AQ_MAX_MATERIALS];
  int64_t n_particles;
  uint64_t seed;
  int32_t sparse;        /* 1: sparse grid (only node blocks near particles are
                            stored, through a table of one int32 per grid
                            block; index spaces up to 2^31 blocks), 0: dense */
  int32_t reserved;
} aq_params;

#ifndef __CUDACC_RTC__
typedef struct aq_sim aq_sim;

/* Create a simulator for n_particles records of `layout`.  Record slots must
 * follow the reference place order x(dim), v(dim), C(dim*dim), F(dim*dim) | J,
 * [material id] (mpm_solver.py:445-452).
 * Replaces MPMSolver.__init__ (mpm_exps/engine/mpm_solver.py:19-122) with its
 * init_quantaichi (:364-455) and init_sparse_grids (:216-253). */
int aq_sim_create(const aq_params* h_params, const aq_layout* h_layout, aq_sim** out);
int aq_sim_destroy(aq_sim* sim);

/* Quantize and store all particle values (d_values: n x n_slots, particle
 * order).  Replaces the per-field initial stores of fill_in_box*
 * (mpm_solver.py:1561-1597) through store_custom_int (codegen_llvm.cpp:1266-1300). */
int aq_sim_set_state(aq_sim* sim, const void* d_values, int32_t values_f64, void* stream);
/* Decode all particle values in particle order.
 * Replaces fetch_data_np / fetch_*_data (mpm_solver.py:1782-1830). */
int aq_sim_get_state(aq_sim* sim, void* d_values, int32_t values_f64, void* stream);
/* Raw packed records in particle order (n x n_words). */
int aq_sim_set_words(aq_sim* sim, const uint64_t* d_words, void* stream);
int aq_sim_get_words(aq_sim* sim, uint64_t* d_words, void* stream);

/* Advance n substeps.  Replaces MPMSolver.substep (mpm_solver.py:624-631):
 * deactivate + build_pid (:578-588) + p2g_bls (:590-622) + grid_op (:633-665)
 * + g2p_bls (:667-758).  Consecutive substeps are fused: G2P of substep k and
 * P2G of substep k+1 run in one kernel. */
int aq_sim_substeps(aq_sim* sim, int32_t n, void* stream);

/* Particles added to a running simulator (the emitters: add_cube, add_ball,
 * emit_water, add_mesh, the letters; mpm_solver.py:1334-1440,1562-1632, which
 * write only the new particles' fields).  A simulator holds up to
 * h_params->n_particles records (its capacity); aq_sim_set_count sets how
 * many of them are active (1..capacity; records beyond are ignored), and
 * aq_sim_append encodes `count` more particles from d_values (count x
 * n_slots, particle ids n, n + 1, ...; dithering keyed on those ids at the
 * initial-state step, as aq_sim_set_state draws) behind the active ones,
 * leaving every stored record as it is.  AQ_E_LIMIT past the capacity;
 * AQ_E_STATE on a streamed simulator.  aq_sim_count reports the active
 * count and the capacity. */
int aq_sim_set_count(aq_sim* sim, int64_t n);
int aq_sim_append(aq_sim* sim, const void* d_values, int32_t values_f64, int64_t count, void* stream);
int aq_sim_count(const aq_sim* sim, int64_t* h_n, int64_t* h_capacity);

/* Streamed (out-of-core) simulator: the packed records of all
 * h_params->n_particles particles live in pinned host memory that the
 * library allocates, and every pass over the particles (aq_sim_substeps,
 * aq_sim_loss) moves them through the device in chunks of at most `chunk`
 * records (upload, binning of the chunk, the substep kernel, download); the
 * grids stay on the device and collect every chunk.  For scenes whose
 * records do not fit in device memory: device memory then holds four
 * chunk buffers and the grids, and the host link bounds the speed, in
 * proportion to the record bytes (the host keeps each chunk in particle
 * order, so no particle ids cross the link).  Dense grids only (sparse = 0).  Records enter and
 * leave through aq_sim_stream_set_words / aq_sim_stream_get_words (host
 * pointers, particle order, n x n_words); aq_sim_set_state, get_state,
 * set_words, get_words and field_stats return AQ_E_STATE on a streamed
 * simulator.  Results equal the in-core simulator's up to the order in which
 * grid sums are added.  No counterpart in the reference, whose particle
 * state is device-resident (mpm_solver.py:190-207). */
int aq_sim_create_streamed(const aq_params* h_params, const aq_layout* h_layout, int64_t chunk, aq_sim** out);
/* Synchronize `stream` (host copies complete on return). */
int aq_sim_stream_set_words(aq_sim* sim, const uint64_t* h_words, void* stream);
int aq_sim_stream_get_words(aq_sim* sim, uint64_t* h_words, void* stream);
/* The chunk size (0: in-core) and the particle count of a simulator. */
int aq_sim_stream_chunks(const aq_sim* sim, int64_t* h_chunk, int64_t* h_n_total);

/* Mesh voxelizer of the emitters (add_mesh: voxelizer.py:53-119): voxel
 * counts of n_tris triangles (d_tris: n_tris x 9 doubles, corners a, b, c)
 * on a res[0] x res[1] x res[2] voxel grid of spacing dx into d_voxels
 * (int32, row-major; voxels > 0 are inside).  Every triangle whose normal
 * has |z| >= 1e-10 adds +1 (normal z > 0) or -1 to the voxels
 * [padding, height) of each column (p, q) in [padding, res - padding) whose
 * centre ((p + 0.5) dx, (q + 0.5) dx) its xy projection covers, height =
 * min(int(-n.(c - a) / n_z / dx + 0.5), res[1] - padding); vertices are
 * first moved by the reference's fixed jitter times jitter_scale (1e-8 at
 * double precision).  Needs 2 padding < res[k]; asynchronous on stream. */
int aq_voxelize(const double* d_tris, int64_t n_tris, const int32_t* res, double dx, int32_t padding,
                double jitter_scale, int32_t* d_voxels, void* stream);

/* Grid masses after the latest substep (the P2G sums grid_op starts from;
 * zeros before the first substep) into d_out, res[0] x res[1] (x res[2])
 * floats, row-major: the grid_m that dump_grid writes
 * (mpm_solver.py:1755-1759). */
int aq_sim_grid_mass(aq_sim* sim, float* d_out, void* stream);

/* Loss of the current state (written to *h_out, synchronizes the stream).
 * kind 0: compute_ek (mpm_solver.py:1043-1052): 3D sum 0.5 m|v|^2 + g m x_y,
 * 2D sum |v|^2. */
int aq_sim_loss(aq_sim* sim, int32_t kind, double* h_out, void* stream);

/* Per-slot statistics of the current decoded state, the inputs of the
 * sensitivity surrogate's features (no counterpart in the reference).
 * h_out receives n_slots x 5 doubles: sum |v|, sum v, sum v^2, max |v|,
 * sum |v - ref|, where d_ref (optional, null skips the last one) holds
 * n x n_slots values in particle order, f64 if ref_f64 else f32.
 * Synchronizes the stream. */
int aq_sim_field_stats(aq_sim* sim, const void* d_ref, int32_t ref_f64, double* h_out, void* stream);

/* Rotating SDF collider of the 3D experiments (init_sdf_collider,
 * init_sdf_value, sdf_collision, rot_scene, step_collider:
 * mpm_solver.py:284-318,1444-1547), applied to the grid velocities after
 * grid_op.  d_sdf: signed distances (float, dims[0] x dims[1] x dims[2],
 * row-major), d_normal: their normals (float x 3), both placed at grid index
 * offset[] and owned by the caller, who keeps them alive while the
 * simulator runs.  The grid index is rotated by -theta about (center, .,
 * center) and lowered by height/dx before the lookup; after every substep
 * theta += omega dt and height += height_rate dt (the reference's
 * step_collider: omega 5, rate 0.1).  d_sdf null switches the collider off.
 * 3D simulators only. */
int aq_sim_set_collider(aq_sim* sim, const float* d_sdf, const float* d_normal, const int32_t* dims,
                        const int32_t* offset, int32_t center, double theta, double height, double omega,
                        double height_rate);
/* Sparse grids (aq_params.sparse): pool slots (node blocks) handed out so
 * far and grid blocks holding particles at the last re-binning.  A dense
 * simulator returns AQ_E_STATE.  Synchronizes `stream`.  Replaces the
 * reference's view of its pointer grid's active blocks (init_sparse_grids,
 * mpm_solver.py:216-253). */
int aq_sim_sparse_blocks(aq_sim* sim, int64_t* h_slots, int64_t* h_occupied, void* stream);

/* Current collider angle and height. */
int aq_sim_collider_get(aq_sim* sim, double* h_theta, double* h_height);
/* Put the collider at angle theta and height `height` for the next substep
 * without touching its volumes or kernel (step_collider_difftaichi,
 * mpm_solver.py:1554-1559, which the autodiff-path drivers call after each
 * substep: theta = omega dt s, height = 0.15 dt s). */
int aq_sim_collider_pose(aq_sim* sim, double theta, double height);
/* Collider velocity omega x r at a node inside the collider: from_node 0
 * takes r from the rotated index (sdf_collision, mpm_solver.py:1459-1480,
 * the forward substep's collider), 1 from the node itself
 * (sdf_collision_no_arg, :1482-1512, the collider of substep_difftaichi and
 * so of nlogn_step_forward).  Default 0. */
int aq_sim_collider_velocity_mode(aq_sim* sim, int32_t from_node);

/* Per-slot running max/min of the state (range detection), accumulated on
 * the device after every substep once enabled.
 * Replaces update_limits_* / get_limits (mpm_solver.py:944-997). */
int aq_sim_ranges_enable(aq_sim* sim, int32_t on, void* stream);
int aq_sim_ranges_get(aq_sim* sim, double* h_max, double* h_min, void* stream);

/* Status flags (AQ_ST_*) and tile-fallback counter; synchronizes the
 * stream.  clear != 0 resets them. */
int aq_sim_status(aq_sim* sim, uint32_t* h_flags, int64_t* h_fallbacks,
                  int32_t clear, void* stream);
int aq_sim_step_count(const aq_sim* sim, int64_t* h_out);
/* Set the substep counter (the dithering generator's step index), e.g. when
 * resuming from saved records so that the continuation draws the same
 * uniforms as an uninterrupted run. */
int aq_sim_set_step_count(aq_sim* sim, int64_t step);
/* 1 if the substep kernel in use was compiled for this layout by NVRTC, 0 if
 * it is the generic nvcc-built kernel.  No reference counterpart (Taichi
 * always JIT-compiles, taichi_submission/taichi/backends/cuda/jit_cuda.cpp). */
int aq_sim_kernel_is_jit(const aq_sim* sim, int32_t* h_out);
/* Launch counters of this simulator's own kernels (for accounting). */
int aq_sim_launches(const aq_sim* sim, int64_t* h_out);

/* Kernel timing with CUDA events recorded around each launch of the fused
 * substep kernel (k_step) and of the grid kernel (k_grid) on the stream they
 * run on.  No reference counterpart (the reference profiles through CUPTI,
 * taichi_submission/taichi/program/kernel_profiler.h:46).  which: 0 = k_step,
 * 1 = the grid clear before each P2G.  profile_get synchronizes and resets
 * the accumulators. */
int aq_sim_profile_enable(aq_sim* sim, int32_t on);
int aq_sim_profile_get(aq_sim* sim, int32_t which, double* h_total_ms, int64_t* h_launches);

/* Per-slot error of a (n x n_slots) against b: h_sq[s] = sum (a-b)^2,
 * h_max[s] = max |a-b|, accumulated in f64.  Used for the error report
 * against the f64 oracle run. */
int aq_state_error(const void* d_a, int32_t a_f64, const void* d_b, int32_t b_f64,
                   int64_t n, int32_t n_slots, double* h_sq, double* h_max,
                   void* stream);

/* ------------------------------------------------------------- adjoint */

/* Hand-written reverse of the substep on unquantized state (n x n_slots,
 * slots x, v, C, F|J; f32 or f64 per params.precision), one material
 * (AQ_MAT_FLUID or the reference's AQ_MAT_ELASTIC), no friction; position
 * clipping is not applied, as in the reference's differentiable g2p.
 * Replaces the reference's autodiff pass: run_forward_with_ad_nlogn with
 * checkpoint / rerun_from / nlogn_loop_forward_grad / accu_grad /
 * get_gradients (mpm_exps/engine/mpm_solver.py:1093-1302) and the Taichi
 * grad kernels of p2g, grid_op and g2p (taichi_submission/taichi/transforms/
 * auto_diff.cpp).  Checkpoints every `every` substeps; a segment is
 * recomputed from its checkpoint during the backward pass. */
typedef struct aq_adjoint aq_adjoint;
int aq_adjoint_create(const aq_params* h_params, aq_adjoint** out);
int aq_adjoint_destroy(aq_adjoint* adj);
/* The rotating SDF collider in the adjoint's substeps (sdf_collision_no_arg
 * and its gradient in the reference's autodiff runs, mpm_solver.py:1491-1516,
 * 1189-1190): same volumes and arguments as aq_sim_set_collider; at substep
 * t the angle is theta + omega dt t and the height height + height_rate dt t
 * (step_collider_difftaichi, :1554-1559).  d_sdf null switches it off.
 * 3D only. */
int aq_adjoint_set_collider(aq_adjoint* adj, const float* d_sdf, const float* d_normal, const int32_t* dims,
                            const int32_t* offset, int32_t center, double theta, double height, double omega,
                            double height_rate);
/* Run n_substeps from d_s0, keeping checkpoints; d_sT receives the final
 * state.  every > 0: a checkpoint every `every` substeps, each segment
 * recomputed once by aq_adjoint_backward (memory n_substeps/every + every
 * states).  every = 0: only the initial state is kept and the backward
 * pass recomputes by bisection, one stashed state per level (the
 * reference's logarithmic stash, run_forward_with_ad_nlogn / rerun_from /
 * cnt_ending_zero, mpm_solver.py:1093-1137,1201-1207; memory ceil(log2 T) + 3
 * states, about T log2(T) / 2 recomputed substeps).  Internally the state is
 * kept sorted by base cell for locality; d_s0, d_sT and the gradients are in
 * the caller's particle order. */
int aq_adjoint_forward(aq_adjoint* adj, const void* d_s0, int32_t n_substeps, int32_t every, void* d_sT,
                       void* stream);
/* Back-propagate d_seed = dL/d(final state) of the last forward run.
 * d_grad_s0 (optional) receives dL/d(initial state); h_sens (optional,
 * n_slots doubles) receives sum over substeps t = 1..T-1 and particles of
 * (dL/d state_t)^2 per slot, the reference's grad_sum. */
int aq_adjoint_backward(aq_adjoint* adj, const void* d_seed, void* d_grad_s0, double* h_sens, void* stream);

/* Same result as aq_state_error, for callers that cannot allocate device
 * memory themselves: hosts that own the device heap (an engine or an in-situ
 * analysis plugin that hands out only its own buffers), or loops that must
 * not take the allocator's locks and latency.  No counterpart in the
 * reference.  It allocates nothing: its per-slot sums live in a fixed
 * library-owned device array of 2 * AQ_NOALLOC_MAX_SLOTS doubles that every
 * GPU loading libaq.so keeps until the process exits; n_slots above
 * AQ_NOALLOC_MAX_SLOTS returns AQ_E_LIMIT, and a current device index at or
 * above AQ_NOALLOC_MAX_DEVICES returns AQ_E_LIMIT.  The first call on a device
 * looks up the array's device address (make that first call before any
 * stream capture starts).  All calls share the one array, each clears its
 * part first, and calls that overlap on the GPU (e.g. from two streams)
 * race on it.  Synchronizes `stream`.  The address looked up on a device is
 * kept for the life of the process, so resetting a device
 * (cudaDeviceReset) while libaq.so is loaded is not supported for this entry
 * point: the kept address would belong to the destroyed context. */
#define AQ_NOALLOC_MAX_SLOTS 256
#define AQ_NOALLOC_MAX_DEVICES 64
int aq_state_error_noalloc(const void* d_a, int32_t a_f64, const void* d_b, int32_t b_f64,
                           int64_t n, int32_t n_slots, double* h_sq, double* h_max,
                           void* stream);

/* ------------------------------------------------ sensitivity surrogate */

/* MLP in -> h -> h -> out (GELU on the hidden layers) predicting per-field
 * log-sensitivities from forward-pass statistics, so that the analytical
 * solver (solvers/analytical_solver.py) can derive a bit-width scheme without
 * a full backward run.  No reference counterpart.  Parameters: one float32
 * vector W1[h][in], b1[h], W2[h][h], b2[h], W3[out][h], b3[out] and its bf16
 * copy (weights are read as bf16, every dot product accumulates in fp32).
 * d_act: B*4*h floats of saved activations (optional for inference). */
int64_t aq_mlp_param_count(int32_t in, int32_t h, int32_t out);
int aq_mlp_to_bf16(const float* d_params, uint16_t* d_params_bf16, int64_t n, void* stream);
int aq_mlp_forward(int32_t in, int32_t h, int32_t out, const float* d_params, const uint16_t* d_params_bf16,
                   const float* d_x, int32_t batch, float* d_y, float* d_act, void* stream);
/* Gradient of the loss w.r.t. all parameters (d_grad, same layout) given
 * d_dy = dL/dy and the activations saved by aq_mlp_forward. */
int aq_mlp_backward(int32_t in, int32_t h, int32_t out, const uint16_t* d_params_bf16, const float* d_x,
                    int32_t batch, const float* d_act, const float* d_dy, float* d_grad, void* stream);
/* Masked mean squared error: d_dy = 2 (y - t) m / count; *d_loss += loss. */
int aq_mlp_mse_grad(const float* d_y, const float* d_target, const float* d_mask, float* d_dy, int64_t n,
                    float count, float* d_loss, void* stream);
/* One Adam step (t >= 1) on the fp32 parameters; refreshes the bf16 copy. */
int aq_mlp_adam(float* d_params, uint16_t* d_params_bf16, float* d_m, float* d_v, const float* d_grad, int64_t n,
                float lr, float beta1, float beta2, float eps, int32_t t, void* stream);

const char* aq_error_string(int32_t code);
int32_t aq_abi_version(void);
#endif /* __CUDACC_RTC__ */

#ifdef __cplusplus
}
#endif
#endif /* AQ_H_ */
