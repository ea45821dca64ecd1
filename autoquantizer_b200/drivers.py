"""The reference's experiment pipeline on libaq: range detection (-r), the
gradient pass (-a), and scheme derivation followed by quantized forward runs
(-f), for the deterministic 2D experiments of mpm_exps/ and a 3D elastic
block.

    python -m autoquantizer_b200.drivers elastic_2d -r            # ranges/elastic_2d/elastic_2d.npy
    python -m autoquantizer_b200.drivers elastic_2d -a            # grads/elastic_2d/elastic_2d.npy
    python -m autoquantizer_b200.drivers elastic_2d -f -m 1 -e 0.1 -N 20

Flags follow the reference drivers (run_mpm_elastic_2d.py:18-50): -a
gradients, -r ranges, -f solve + forward, -e epsilon, -m mode (0 compression
rate, 1 error bound); with -f, --optimality TASK -b S1 -b2 S2 perturbs the
solved widths as run_mpm_optimality_check.py does before the runs.  Additions: --root (folder holding grads/ and ranges/,
default the working directory), -N (forward runs), --timesteps (shorter
horizons), --json (one summary line).

Experiments:
  elastic_2d  run_mpm_elastic_2d.py:54-122 — 80,000 particles in eight
              lattice cubes, 128^2, dt 2e-4, 8193 timesteps, E 50, f64.
  fluid_2d    run_mpm_fluid_2d.py:185-214 — 10,000 particles in one lattice
              cube, 128^2, dt 2e-4, 16385 timesteps, bulk modulus 500, f64;
              compression-rate mode only, with the driver's own solver
              variant (run_mpm_fluid_2d.py:129-145).
  falling_block_3d  the 3D elastic block of the adjoint benchmark (262,144
              particles, 64^3, dt 5e-5, 257 timesteps, f32); scheme recipe of
              run_mpm_elastic_3d.py:331-341 (ranges doubled, CR, bits + 1).
  elastic_3d  run_mpm_elastic_3d.py — the letters mesh emitted frame by
              frame (add_mesh over the mesh voxelizer), 3D reference law.
  fluid_3d    run_mpm_fluid_3d.py — two fluid slabs stirred by the rotating
              SDF propeller collider (init_sdf_value; the autodiff path's
              collider schedule for -a and -r).
  dithering_2d  run_mpm_dithering_exp.py — the 2D elastic material in four
              cubes on a fixed scheme; -f runs it unquantized, quantized with
              dithering and without.
  fluid_3d_scaling  run_mpm_fluid_3d_scaling.py — a fluid block (or, for
              configurations 5 and 6, two water jets) in a walled box, from
              one of the reference's JSON configurations (-c); scheme from
              the SLSQP memory-budget solver.

Each forward run re-seeds the dithering generator (seed = run index), which
plays the role of the reference's per-run random state.
"""
import argparse
import json
import os
import sys

import numpy as np

from .mpm_config import MPMConfig
from .solvers import LagrangianCR, LagrangianEB, ScipySolverMemMode

CR, EB = 0, 1


def lagrangian_cr_fluid_2d(grads, r=0.5, a=None):
    """The compression-rate solver as run_mpm_fluid_2d.py:129-145 defines it
    locally: multiplier 2·ln2 inside the log and bits rounded up, with no
    separate sign bit added afterwards."""
    grads = np.asarray(grads, dtype=np.float64)
    n = len(grads)
    r = r * 32.0 - 1
    a = np.ones(n) if a is None else np.asarray(a, dtype=np.float64)
    b = a / grads
    t = np.log2(b)
    log_la = -r * 2 - t @ a / np.sum(a) + np.log2(2 * np.log(2))
    la = np.power(2, log_la)
    fun = (b * la) @ grads / 12.0
    bits = np.ceil(-(t + log_la) / 2.0).astype(np.int32)
    return bits, fun


class Experiment:
    name = None
    file_name = None
    f64_data = None  # unquantized loss the error-bound mode measures against
    modes = (CR, EB)

    def config(self, kind="forward"):
        """kind: "ad", "ranges" or "forward" (the drivers' set-ups differ)."""
        raise NotImplementedError

    def init(self, mpm):
        raise NotImplementedError

    def scheme(self, grads, ranges, mode, eps):
        raise NotImplementedError


class Elastic2D(Experiment):
    """run_mpm_elastic_2d.py:54-122 (config, init) and :232-250 (solve)."""

    name = "elastic_2d"
    file_name = "elastic_2d.npy"
    f64_data = 6893.409

    def config(self, kind="forward"):
        c = MPMConfig()
        c.dim = 2
        c.E = 5e1
        c.id = "elastic_2d_err_bound"
        c.la = 1e3
        c.bound = [3, 3]
        c.use_friction = False
        c.use_fluid = False
        c.n_particles = 80000
        c.dt = 2e-4
        c.n_grid = 128
        c.n_timesteps = 1024 * 8 + 1
        c.steps = 64
        c.size = 1
        c.p_rho = 1.0
        c.p_vol = (1 / c.n_grid * 0.5) ** c.dim
        c.quantized_properties = {"x": 1, "v": 1, "C": 1, "F": 1}
        c.quant_bits = np.array([32] * 12)
        c.quant_ranges = np.array([2.0] * 12)
        c.precision = "f64"  # ti.init(default_fp=ti.float64)
        return c

    def init(self, mpm):
        mpm.initialize()
        n = mpm.param.n_particles // 8
        for i in range(4):
            mpm.add_cube(((0.2 + i * 0.4) / 4, (0.2 + i * 0.8) / 4), (0.7 / 4, 0.7 / 4), n)
        for i in range(4):
            mpm.add_cube(((3.1 - i * 0.2) / 4, (0.2 + i * 0.8) / 4), (0.7 / 4, 0.7 / 4), n)

    def scheme(self, grads, ranges, mode, eps):
        d = 2
        ranges = np.array(ranges, dtype=np.float64)
        ranges[:d] = 1.0
        ranges[d:] *= 2.0
        if mode == CR:
            bits, _ = LagrangianCR(grads=grads * ranges ** 2, r=eps)
        else:
            bits, _ = LagrangianEB(grads=grads * ranges ** 2, ref=self.f64_data, tol_rel=eps)
        return bits + 1, ranges


class Dithering2D(Elastic2D):
    """run_mpm_dithering_exp.py: the 2D elastic material (E 50, 80,000
    particles, 128^2, 8193 timesteps, f64) in four lattice cubes at
    (0.125 + 0.2 i, 0.75), 0.15 x 0.15, a fixed scheme (widths 19, 19, 13,
    13, 9, 10, 10, 9, 14, 14, 14, 15 on the elastic_2d experiment's ranges,
    positions 1, the others doubled, :119-132); -f runs it unquantized (the
    f64 reference), quantized with dithering and quantized without (the
    driver's three modes, :98-113).  The driver sets config.dt = 5e-5 in
    init_dithering (:79), after the solver has read its time step
    (mpm_solver.py:44): its runs use dt 2e-4, and so do these."""

    name = "dithering_2d"
    file_name = "elastic_2d.npy"  # ranges/elastic_2d: the elastic_2d experiment's
    modes = ()
    BITS = [19, 19, 13, 13, 9, 10, 10, 9, 14, 14, 14, 15]

    def config(self, kind="forward"):
        c = super().config(kind)
        c.id = "dithering"
        c.quant_bits = np.array(self.BITS)
        return c

    def init(self, mpm):
        mpm.initialize()
        n = mpm.param.n_particles // 4
        for i in range(4):
            mpm.add_cube((0.125 + i * 0.2, 0.75), (0.15, 0.15), n)


def dithering_experiment(exp, cfg, root):
    """The three runs of run_mpm_dithering_exp.py on the experiment's fixed
    scheme and the elastic_2d ranges: the loss of each and the relative
    error of the quantized ones against the unquantized run."""
    import copy

    ranges = np.array(np.load(os.path.join(root, "ranges", "elastic_2d", exp.file_name)), dtype=np.float64)
    ranges[:2] = 1.0
    ranges[2:] *= 2.0
    cfg.quant_ranges = ranges
    out = {"bits": list(exp.BITS), "ranges": ranges.tolist()}
    ref = float(run(exp, copy.deepcopy(cfg), 1, quant=False)[0])
    out["loss_f64"] = ref
    for name, dith in (("dithering", True), ("no_dithering", False)):
        c = copy.deepcopy(cfg)
        c.use_dithering = dith
        loss = float(run(exp, c, 1, quant=True)[0])
        out["loss_" + name] = loss
        out["rel_err_" + name] = abs(loss - ref) / abs(ref)
    return out


def perturb_bits(bits, dim, task, s1, s2=None, rng=None):
    """The widths of run_mpm_optimality_check.py's checks (:196-232) from
    solved ones: task 0 takes s1 bits off every field, task 1 off half of
    the fields chosen at random, task 2 moves s1 bits from each position
    component to the velocity's and s2 from each entry of C to F's."""
    b = np.array(bits, dtype=np.int64).copy()
    n = len(b)
    if task in (0, 1):
        order = (rng or np.random.default_rng(0)).permutation(n)
        for k in order[: n if task == 0 else n // 2]:
            b[k] -= s1
    elif task == 2:
        s2 = s1 if s2 is None else s2
        b[:dim] -= s1
        b[dim:2 * dim] += s1
        b[2 * dim:2 * dim + dim * dim] -= s2
        b[2 * dim + dim * dim:2 * dim + 2 * dim * dim] += s2
    else:
        raise ValueError("optimality task %r is not 0, 1 or 2" % (task,))
    return b


class Fluid2D(Experiment):
    """run_mpm_fluid_2d.py:116-127 (init), :162-178 (solve), :185-214 (config)."""

    name = "fluid_2d"
    file_name = "fluid_2d_t16385_dt0.0002_p10000_g128.npy"
    modes = (CR,)

    def config(self, kind="forward"):
        c = MPMConfig()
        c.dim = 2
        c.E = 5e4
        c.id = "fluid_2d_mem_bound"
        c.la = 5e2
        c.bound = [3, 3]
        c.use_friction = False
        c.quant_ranges = np.ones(9)
        c.quantized_properties = {"x": 1, "v": 1, "C": 1, "J": 1}
        c.quant_bits = np.ones(9)
        c.n_particles = 10000
        c.dt = 2e-4
        c.n_grid = 128
        c.n_timesteps = 1024 * 16 + 1
        c.steps = 128
        c.size = 1
        c.precision = "f64"
        return c

    def init(self, mpm):
        mpm.initialize()
        dx = 1 / mpm.param.n_grid
        b = mpm.param.bound
        mpm.add_cube((b[0] * dx, b[1] * dx), (1.5 / 4, 1.5 / 4), mpm.param.n_particles)

    def scheme(self, grads, ranges, mode, eps):
        if mode != CR:
            raise ValueError("fluid_2d runs the compression-rate mode only (run_mpm_fluid_2d.py:182)")
        ranges = np.array(ranges, dtype=np.float64)
        ranges[:2] = 1.0
        ranges[2:] *= 2.0
        g = np.asarray(grads, dtype=np.float64)
        g = g / g.min()
        bits, _ = lagrangian_cr_fluid_2d(g * ranges ** 2, r=eps)
        return bits, ranges


class FallingBlock3D(Experiment):
    """The 3D elastic block of the adjoint benchmark, with the 2D drivers'
    range recipe (positions range 1 on the unit domain, the other ranges
    doubled)."""

    name = "falling_block_3d"
    file_name = "falling_block_3d.npy"

    def config(self, kind="forward"):
        from . import scenes

        c, vals = scenes.falling_block_3d()
        c.n_timesteps = 257
        c.steps = 16
        c.quantized_properties = {"x": 1, "v": 1, "C": 1, "F": 1}
        c.quant_bits = np.array([32] * 24)
        c.quant_ranges = np.array([2.0] * 24)
        c.compute_fp = "f32"
        self._vals = vals
        return c

    def init(self, mpm):
        mpm.initialize()
        mpm.set_particles(self._vals)

    def scheme(self, grads, ranges, mode, eps):
        ranges = np.array(ranges, dtype=np.float64) * 2.0
        ranges[:3] = 1.0
        if mode == CR:
            bits, _ = LagrangianCR(grads * ranges ** 2, r=eps)
        else:
            ref = self.f64_data if self.f64_data is not None else 1.0
            bits, _ = LagrangianEB(grads * ranges ** 2, ref=ref, tol_rel=eps)
        return bits + 1, ranges


class Letters3D(Experiment):
    """The 3D elastic letters experiment (run_mpm_elastic_3d.py): config
    :249-290 (the high-resolution forward run) and, for the gradient and
    range passes, the low-resolution set-up (use_low_res); scheme :323-333;
    the letters mesh inputs/auto_quant.ply (load_mesh with scale (0.1, 0.1,
    2), offset (0.02, 0.02, 0.5), :249), emitted by add_mesh at
    translation (0.90, 1.6, 0.1) and (2.2, 1.6, 0.1) (add_letters, :45-61).
    The range pass and the forward runs follow the driver's frame loop
    (run_forward_only, :87-157): every emit_step frames, while the next batch
    fits, two more sets of letters (emit / add_letters, :45-84)."""

    name = "elastic_3d"
    file_name = "elastic_3d.npy"
    modes = (CR,)
    inputs = "inputs"

    def config(self, kind="forward"):
        c = MPMConfig()
        c.dim = 3
        c.E, c.la, c.nu = 5e5, 5e4, 0.2
        c.g = 9.8 * 2.5
        c.bound = [3, 3, 3]
        c.p_rho = 1000.0
        c.use_fluid = False
        if kind == "ad":  # use_low_res with default_fp f64 (:240-244, :265-271)
            c.n_particles = 100 ** 3
            c.dt = 1e-4
            c.n_grid = 128
            c.n_timesteps = 1024 * 16 + 1
            self.sample_density = 1
            self.emit_step = 5
            c.precision = "f64"
        else:  # high resolution (:272-280); detect_range keeps 500^3 particles, 16k substeps (:307-316)
            c.n_particles = int(3e8) if kind == "forward" else 500 ** 3
            c.dt = 7.5e-5
            c.n_grid = 128 * 2
            c.n_timesteps = 1024 * 40 + 1 if kind == "forward" else 1024 * 16
            self.sample_density = 8
            self.emit_step = 4
        c.steps = 128
        c.p_vol = (1 / c.n_grid * 0.5) ** c.dim
        c.quantized_properties = {"x": 1, "v": 1, "C": 1, "F": 1}
        c.use_dithering = True
        c.use_bitpack = True
        c.use_bound_clip = True
        c.quant_bits = np.array([32] * 24)
        c.quant_ranges = np.array([4.0] * 24)
        c.grid_res = [4 * c.n_grid, 2 * c.n_grid, 2 * c.n_grid]
        return c

    def mesh(self):
        from .mesh_io import load_mesh

        return load_mesh(os.path.join(self.inputs, "auto_quant.ply"), scale=(0.1, 0.1, 2), offset=(0.02, 0.02, 0.5))

    def init(self, mpm):
        """initialize(); the letters come with the frames (emit)."""
        mpm.initialize()
        self.num_emit = 0
        self._tri = self.mesh()

    def emit(self, frame, mpm):
        """emit / add_letters (run_mpm_elastic_3d.py:45-84): at frames that are
        multiples of emit_step, while the batch fits below n_particles, two
        letter meshes at x 0.90 and 2.2, y 1.6, z 0.1 + 0.006 k (k = frame //
        emit_step), falling at 4 m/s; a batch is twice the particle count of
        one mesh and starts at particle k times that."""
        if frame % self.emit_step:
            return
        k = frame // self.emit_step
        z = 0.1 + 0.006 * k
        if self.num_emit == 0:
            self.num_emit = 2 * mpm.cnt_mesh_particles_num(self._tri, translation=(0.90, 1.6, z),
                                                           sample_density=self.sample_density)
        if k * self.num_emit + self.num_emit >= mpm.n_particles:
            return
        mpm.current_idx = k * self.num_emit
        for x0 in (0.90, 2.2):
            mpm.add_mesh(self._tri, velocity=(0.0, -4.0, 0.0), translation=(x0, 1.6, z),
                         sample_density=self.sample_density)

    def run_frames(self, mpm, detect=False):
        """The driver's frame loop (run_forward_only, :87-157): int(n_timestep
        / steps + 1) frames, each emit() then `steps` substeps; with detect,
        the state at the end of every frame is folded into the ranges
        (detect_bound_kernel, get_limits), which are returned."""
        max_frame = int(mpm.n_timestep / mpm.steps + 1.0)
        for frame in range(max_frame):
            self.emit(frame, mpm)
            if mpm.current_idx == 0:
                continue
            mpm.substeps(mpm.steps)
            if detect:
                mpm.detect_bound_kernel(0)
        if detect:
            mpm.detect_bound()
            return mpm.get_limits()
        return None

    def scheme(self, grads, ranges, mode, eps):
        if mode != CR:
            raise ValueError("elastic_3d runs the compression-rate mode only")
        ranges = np.array(ranges, dtype=np.float64) * 2.0
        ranges[:3] = 4.0
        bits, _ = LagrangianCR(np.asarray(grads) * ranges ** 2, r=eps)
        return bits + 1, ranges


class Propeller3D(Experiment):
    """The 3D fluid-and-propeller experiment (run_mpm_fluid_3d.py): the
    gradient and range set-up ad_or_ranges :101-146 (1e6 particles, 64
    grid, domain 2 x 1 x 2, two slabs, collider inputs/propeller_higher*.npz
    on the autodiff schedule: height rate 0.15), the forward set-up :164-227
    (4e8 particles, 256 grid, domain 4 x 1 x 4, one slab, collider
    inputs/propeller_2x2_larger*.npz, height rate 0.1) and the scheme of
    solve() :149-161 (quantized ranges :203-209)."""

    name = "fluid_3d"
    file_name = "fluid_3d.npy"
    modes = (CR,)
    inputs = "inputs"

    def config(self, kind="forward"):
        c = MPMConfig()
        c.dim = 3
        c.use_fluid = True
        c.use_friction = False
        c.p_rho = 1000.0
        c.la = 5e5
        c.E = 5e4
        c.bound = [3, 3, 3]
        c.quantized_properties = {"x": 1, "v": 1, "C": 1, "J": 1}
        if kind in ("ad", "ranges"):
            c.n_particles = 100 ** 3
            c.dt = 4e-4
            c.n_grid = 64
            c.n_timesteps = 1024 * 8 + 1
            c.p_vol = (1 / c.n_grid) ** 3
            c.ub = [c.n_grid * 2 - 3, c.n_grid - 3, c.n_grid * 2 - 3]
            # the slabs reach x, z = 1.984 (node 128 in the stencil) and the
            # reference's grid is a 4096^3 index space: nodes beyond the
            # walls must exist here too
            c.grid_res = [2 * c.n_grid + 4, c.n_grid + 4, 2 * c.n_grid + 4]
            c.precision = "f64" if kind == "ad" else "f32"
            self.kind = "ad"
        else:
            c.n_particles = int(4e8)
            c.dt = 1e-4
            c.n_grid = 128 * 2
            c.n_timesteps = 1024 * 32 + 1
            c.p_vol = (4 * 4 * 0.3) / c.n_particles
            c.g = 9.8
            c.lb = [3, 3, 3]
            c.ub = [c.n_grid * 4 - 3, c.n_grid - 3, c.n_grid * 4 - 3]
            c.grid_res = [4 * c.n_grid, c.n_grid, 4 * c.n_grid]
            c.use_dithering = True
            c.use_bitpack = True
            c.use_bound_clip = True
            self.kind = "forward"
        c.quant_bits = np.array([32] * 16)
        c.quant_ranges = np.array([2.0] * 16)
        return c

    def collider(self):
        stem = "propeller_higher" if getattr(self, "kind", "forward") == "ad" else "propeller_2x2_larger"
        sdf = np.load(os.path.join(self.inputs, stem + ".npz"))["sdf"]
        normal = np.load(os.path.join(self.inputs, stem + "_normal.npz"))["sdf"]
        return sdf, normal

    def init(self, mpm):
        mpm.initialize()
        c = mpm.param
        sdf, normal = self.collider()
        rate = 0.15 if self.kind == "ad" else 0.1
        mpm.init_sdf_value(sdf, normal, offset=[0, 0, 0], omega=5.0, height_rate=rate)
        dx = 1 / c.n_grid
        b = c.bound
        if self.kind == "ad":
            ub = [c.n_grid * 2 - b[0] - 1, c.n_grid - b[1], c.n_grid * 2 - b[2] - 1]
            for y0 in (b[1] * dx, b[1] * dx + 0.2):
                mpm.add_cube((b[0] * dx, y0, b[2] * dx), (ub[0] * dx, 0.2, ub[2] * dx), c.n_particles // 2)
        else:
            lb, ub = c.lb, c.ub
            mpm.add_cube(((lb[0] + 0.5) * dx, (lb[1] + 0.5) * dx, (lb[2] + 0.5) * dx),
                         ((ub[0] - lb[0] - 0.5) * dx, 0.3, (ub[0] - lb[0] - 0.5) * dx), c.n_particles)

    def scheme(self, grads, ranges, mode, eps):
        """Bits from the solve() recipe (positions range 2 there), returned
        with the quantized ranges of the forward run (positions 4, y 1)."""
        if mode != CR:
            raise ValueError("fluid_3d runs the compression-rate mode only")
        r = np.array(ranges, dtype=np.float64)
        r[6:15] *= 24
        r[3:6] *= 1.5
        r[-1] *= 1.5
        rs = r.copy()
        rs[:3] = 2.0
        bits, _ = LagrangianCR(np.asarray(grads) * rs ** 2, r=eps)
        r[:3] = 4.0
        r[1] = 1.0
        return bits + 1, r


class Fluid3DScaling(Experiment):
    """The 3D fluid scaling and initial-condition experiments
    (run_mpm_fluid_3d_scaling.py): a weakly compressible fluid block (bulk
    modulus 5e5, 2e6 for configurations 4 and 7; rho 1000) in a walled box,
    set up from one of the reference's JSON configurations (parse_json,
    :60-73: particle count, dt, timesteps = steps * 1024 + 1, grid, walls
    lb / ub, id, frame length steps // 16 * 128, task 0 scaling or 1 initial
    condition; --config), the initial blocks of init() (:222-275) and, for
    configurations 5 and 6, two water jets emitted every 30 substeps
    (emit_water, :126-131).  solve() (:324-346) reads the gradients of the
    reference's 200,000-particle run and the ranges of its 5,000,000-particle
    run and derives the scheme with the SLSQP memory-budget solver for
    configurations 0-5, the compression-rate closed form (bits + 1) for 6
    and 7; compression-rate mode only."""

    name = "fluid_3d_scaling"
    file_name = "fluid_3d_t16385_dt0.0002_p200000_g64.npy"
    solve_range_file = "fluid_3d_t65537_dt5e-05_p5000000_g256.npy"
    f64_data = 0.06709209246760206
    modes = (CR,)
    config_file = None
    emit_step = 30
    SCALING, INIT_CONDITION = 0, 1

    def config(self, kind="forward"):
        c = MPMConfig()
        c.dim = 3
        c.bound = [3, 3, 3]
        c.lb = [15, 3, 3]
        c.ub = [48, 60, 60]
        c.use_friction = False
        c.use_fluid = True
        if self.config_file is not None:
            with open(self.config_file) as f:
                data = json.load(f)
            c.n_particles = data["n_particles"]
            c.dt = data["dt"]
            c.n_timesteps = data["steps"] * 1024 + 1
            c.n_grid = data["grids"]
            c.lb = data["lb"]
            c.ub = data["ub"]
            c.id = data["id"]
            c.steps = data["steps"] // 16 * 128
            c.task = data.get("task", self.SCALING)
        c.la = 2e6 if c.id in (4, 7) else 5e5
        c.E = 5e4
        c.p_rho = 1000.0
        c.p_vol = (1 / c.n_grid * 0.5) ** c.dim
        c.size = 1.0
        c.g = 9.8
        c.quantized_properties = {"x": 1, "v": 1, "C": 1, "J": 1}
        c.quant_bits = np.array([32] * 16)
        c.quant_ranges = np.array([2.0] * 16)
        c.precision = "f64"  # ti.init(default_fp=ti.float64)
        self.cid, self.task = c.id, c.task
        return c

    def init(self, mpm):
        """init() (:222-275): blocks at the walls lb, sized from lb / ub."""
        mpm.initialize()
        c = mpm.param
        dx = 1 / c.n_grid
        lb, ub, n = c.lb, c.ub, c.n_particles
        low = ((lb[0] + 0.5) * dx, (lb[1] + 0.5) * dx, (lb[2] + 0.5) * dx)
        full = ((ub[0] - lb[0] + 1) * dx, 0.2, 0.3)
        if self.task == self.SCALING:
            mpm.add_cube(low, full, n)
        elif self.task == self.INIT_CONDITION:
            if self.cid == 0:
                mpm.add_cube(low, ((ub[0] - lb[0] + 1) * 0.5 * dx, 0.2, 0.3), n)
            elif self.cid == 1:
                mpm.add_cube((((lb[0] + ub[0]) * 0.5) * dx, low[1], low[2]),
                             ((ub[0] - lb[0] + 1) * 0.5 * dx, 0.2, 0.3), n)
            elif self.cid == 2:
                mpm.add_cube(low, ((ub[0] - lb[0] + 1) * dx, 0.3, 0.3), n)
            elif self.cid == 3:
                mpm.add_cube(low, full, n // 2)
                mpm.add_cube((low[0], low[1], (ub[2] - 0.3 * c.n_grid - 0.5) * dx), full, n // 2)
            elif self.cid in (4, 7):
                mpm.add_cube(low, full, n)
            elif self.cid not in (5, 6):  # 5 and 6 start empty: the jets fill them
                raise ValueError("no initial condition %d" % self.cid)
        else:
            raise ValueError("task %r is neither scaling (0) nor initial condition (1)" % (self.task,))

    def emit(self, s, mpm):
        """The jets of configurations 5 and 6 (:126-131), at substeps that are
        multiples of emit_step."""
        if s % self.emit_step:
            return
        if self.cid == 5:
            mpm.emit_water([0.5, 0.3, 0.2], 0.04, [0.0, 0.0, 2.0], 1000)
            mpm.emit_water([0.5, 0.3, 0.8], 0.04, [0.0, 0.0, -2.0], 1000)
        elif self.cid == 6:
            mpm.emit_water([0.5, 0.3, 0.3], 0.04, [0.0, 0.0, 3.0], 1000)
            mpm.emit_water([0.5, 0.3, 0.7], 0.04, [0.0, 0.0, -3.0], 1000)

    def run_frames(self, mpm, detect=False):
        """run_forward_only (:77-152): n_timestep - 1 substeps, the jets
        emitted on their substeps; with detect, the range pass of
        run_forward_detect_ranges (:292-302), which emits nothing."""
        if detect:
            return mpm.run_forward_detect_ranges()
        total = mpm.n_timestep - 1
        s = 0
        while s < total:
            nxt = total
            if self.cid in (5, 6):
                self.emit(s, mpm)
                nxt = min(total, (s // self.emit_step + 1) * self.emit_step)
            if mpm.current_idx > 0:
                mpm.substeps(nxt - s)
            s = nxt
        return None

    def scheme(self, grads, ranges, mode, eps):
        if mode != CR:
            raise ValueError("fluid_3d_scaling runs the compression-rate mode only")
        ranges = np.array(ranges, dtype=np.float64)
        ranges[:3] = 1.0
        ranges[3:] *= 2.0
        grads = np.asarray(grads, dtype=np.float64)
        if self.cid < 6:
            s = ScipySolverMemMode(len(grads), a=[1], eps=eps, grad=grads / grads.min())
            s.set_range(ranges)
            s.run()
            return np.array(s.get_bits()).astype(np.int32), ranges
        bits, _ = LagrangianCR(grads=grads * ranges ** 2, r=eps)
        return bits + 1, ranges


EXPERIMENTS = {e.name: e for e in (Elastic2D, Dithering2D, Fluid2D, FallingBlock3D, Letters3D, Propeller3D,
                                    Fluid3DScaling)}


def _paths(exp, root):
    g = os.path.join(root, "grads", exp.name)
    r = os.path.join(root, "ranges", exp.name)
    return os.path.join(g, exp.file_name), os.path.join(r, exp.file_name)


def _solver(exp, cfg):
    from .mpm_solver import MPMSolver

    mpm = MPMSolver(cfg)
    exp.init(mpm)
    return mpm


def ad(exp, cfg, root, every=64):
    """The drivers' ad(): the gradient pass, saved as grads/<exp>/<file>."""
    cfg.use_difftaichi = True
    cfg.use_quantaichi = False
    mpm = _solver(exp, cfg)
    loss = mpm.run_forward_with_ad_nlogn(every=every)
    g = mpm.get_gradients()
    fn, _ = _paths(exp, root)
    os.makedirs(os.path.dirname(fn), exist_ok=True)
    np.save(fn, g)
    return {"loss": float(loss), "grads": g.tolist(), "file": fn}


def detect_range(exp, cfg, root):
    """The drivers' detect_range(): unquantized forward with running
    max/min, saved as ranges/<exp>/<file>."""
    cfg.use_quantaichi = False
    mpm = _solver(exp, cfg)
    if hasattr(exp, "run_frames"):  # experiments that emit particles frame by frame
        ranges = exp.run_frames(mpm, detect=True)
    else:
        ranges = mpm.run_forward_detect_ranges()
    _, fn = _paths(exp, root)
    os.makedirs(os.path.dirname(fn), exist_ok=True)
    np.save(fn, ranges)
    return {"ranges": ranges.tolist(), "file": fn, "max": mpm._rmax.tolist(), "min": mpm._rmin.tolist()}


def solve(exp, cfg, root, mode, eps):
    """The drivers' solve(): bits and ranges from the saved gradients and
    ranges, written into the config."""
    gfn, rfn = _paths(exp, root)
    if getattr(exp, "solve_range_file", None):  # a range file of another run (fluid_3d_scaling)
        rfn = os.path.join(os.path.dirname(rfn), exp.solve_range_file)
    grads, ranges = np.load(gfn), np.load(rfn)
    bits, ranges = exp.scheme(grads, ranges, mode, eps)
    if np.any(np.asarray(bits) < 1) or np.any(np.asarray(bits) > 32):
        # the reference passes these to ti.quant.fixed, which rejects them
        raise ValueError("solved bit widths %s fall outside [1, 32]; choose another epsilon" % list(bits))
    cfg.quant_bits = np.asarray(bits)
    cfg.quant_ranges = np.asarray(ranges)
    return {"bits": [int(b) for b in bits], "ranges": ranges.tolist(),
            "compression_rate": float(np.sum(bits) / (32 * len(bits)))}


def run(exp, cfg, n_runs, quant=True):
    """The drivers' run(N, quant=True): N forward runs, loss of each."""
    if quant:
        cfg.use_difftaichi = False
        cfg.use_bls = True
        cfg.use_bitpack = True
        cfg.use_quantaichi = True
    losses = []
    for i in range(n_runs):
        cfg.seed = i
        mpm = _solver(exp, cfg)
        if hasattr(exp, "run_frames"):  # particles emitted frame by frame
            exp.run_frames(mpm)
            losses.append(float(mpm.compute_loss()))
        else:
            losses.append(float(mpm.run_forward_only()))
        if mpm.status()[0] != 0:
            raise RuntimeError("simulator status flags 0x%x in run %d" % (mpm.status()[0], i))
        mpm._drop_sim()
    return np.array(losses)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("experiment", choices=sorted(EXPERIMENTS))
    ap.add_argument("-a", "--ad", action="store_true", help="compute gradients")
    ap.add_argument("-r", "--ranges", action="store_true", help="detect ranges")
    ap.add_argument("-f", "--forward", action="store_true", help="solve the scheme and run quantized")
    ap.add_argument("-e", "--epsilon", type=float, default=0.1)
    ap.add_argument("-m", "--mode", type=int, default=CR, help="0 compression rate, 1 error bound")
    ap.add_argument("-N", "--runs", type=int, default=20)
    ap.add_argument("--root", default=".")
    ap.add_argument("--inputs", default="inputs", help="folder of the 3D experiments' meshes and collider volumes")
    ap.add_argument("-c", "--config", default=None,
                    help="fluid_3d_scaling: one of the reference's JSON configurations (mpm_exps/configs/...)")
    ap.add_argument("--optimality", type=int, default=None, metavar="TASK",
                    help="with -f: perturb the solved widths as run_mpm_optimality_check.py does "
                         "(0: -b bits off every field, 1: off half of them, 2: move -b bits x->v, -b2 bits C->F)")
    ap.add_argument("-b", "--search-bits", type=int, default=1)
    ap.add_argument("-b2", "--search-bits-2", type=int, default=1)
    ap.add_argument("--seed", type=int, default=0, help="fields chosen by --optimality 1")
    ap.add_argument("--timesteps", type=int, default=None)
    ap.add_argument("--json", action="store_true")
    args = ap.parse_args(argv)

    exp = EXPERIMENTS[args.experiment]()
    exp.inputs = args.inputs
    exp.config_file = args.config
    cfg = exp.config("ad" if args.ad else "ranges" if args.ranges else "forward")
    if args.timesteps:
        cfg.n_timesteps = args.timesteps
    if args.ad:
        out = ad(exp, cfg, args.root)
    elif args.ranges:
        out = detect_range(exp, cfg, args.root)
    elif args.forward and isinstance(exp, Dithering2D):
        out = dithering_experiment(exp, cfg, args.root)
    elif args.forward:
        if args.mode not in exp.modes:
            ap.error("%s has no mode %d" % (exp.name, args.mode))
        out = solve(exp, cfg, args.root, args.mode, args.epsilon)
        if args.optimality is not None:
            b = perturb_bits(out["bits"], cfg.dim, args.optimality, args.search_bits, args.search_bits_2,
                             np.random.default_rng(args.seed))
            if np.any(b < 1) or np.any(b > 32):
                ap.error("perturbed widths %s fall outside [1, 32]" % b.tolist())
            cfg.quant_bits = b
            out["bits_solved"], out["bits"] = out["bits"], b.tolist()
        loss = run(exp, cfg, args.runs)
        out.update({"loss_mean": float(loss.mean()), "loss_std": float(loss.std()),
                    "loss_max": float(loss.max()), "loss_min": float(loss.min()), "losses": loss.tolist()})
        if args.mode == EB and exp.f64_data is not None:
            tar = args.epsilon * exp.f64_data
            out["succeed"] = float(np.mean(np.abs(loss - exp.f64_data) < tar * 3))
    else:
        ap.error("one of -a, -r, -f")
    out["experiment"] = exp.name
    if args.json:
        print(json.dumps(out))
    else:
        for k, v in out.items():
            print("%s: %s" % (k, v))
    return out


if __name__ == "__main__":
    main(sys.argv[1:])
