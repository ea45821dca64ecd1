"""MPMConfig: the simulator's parameter bag.

Same fields and defaults as the reference's mpm_exps/mpm_config.py:1-53, so
drivers written against it run unchanged; fields after the marked line are
additions of this implementation.
"""


class MPMConfig(object):
    def __init__(self):
        self.id = 0
        self.n_grid = 128
        self.res = 512
        self.n_particles = 9000
        self.dim = 2
        self.dt = 1e-4
        self.p_rho = 1
        self.p_vol = (1 / self.n_grid * 0.5) ** self.dim
        self.E, self.nu = 0.1e4, 0.2
        self.la = 100000
        self.output_folder = None
        self.benchmark_path = None
        self.material = 1
        self.save_end_state = False
        self.n_timesteps = 2048
        self.quantized_properties = None
        self.n_vec2_vars = 0
        self.n_mat2_vars = 0
        self.use_quantaichi = False
        self.use_hand_scheme = False
        self.use_difftaichi = False
        self.forward_only_mode = False
        self.nlogn_mode = False
        self.pos_output_folder = None
        self.quant_bits = None
        self.quant_ranges = None
        self.use_g2p2g = False
        self.use_sdf_collider = False
        self.use_bls = False
        self.use_bitpack = False
        self.use_fluid = True
        self.use_friction = True
        self.use_dithering = True
        self.use_grad_clip = False
        self.use_height_loss = False
        self.use_bound_clip = False
        self.bound = None
        self.lb = None
        self.ub = None
        self.g = 9.8
        self.steps = 128
        self.compute_fp = 'f64'
        self.size = 4.0
        self.task = -1
        self.softer = False
        self.refine_ranges = False
        self.hand_scheme_exp = False
        # ---- additions -------------------------------------------------
        # arithmetic and grid precision of the simulator ('f32' | 'f64'); the
        # reference takes it from ti.init(default_fp=...)
        self.precision = 'f32'
        # grid cells per axis; None = round(n_grid * size) per axis
        self.grid_res = None
        # v stored as floats with one shared exponent of this many bits
        # (None = fixed point, as init_quantaichi builds it)
        self.v_exp_bits = None
        # per-particle materials: list of (kind, E, nu, la) and an id slot
        self.materials = None
        # re-bin particles every k substeps
        self.sort_interval = 16
        # seed of the dithering generator and of the random scene seeding
        self.seed = 0
        # compile the substep kernel for the record layout with NVRTC
        # (False: the generic kernel built into libaq.so)
        self.jit = True
        # sparse grid: store only the grid blocks around particles (the
        # reference's pointer grid over a 4096^dim index space,
        # mpm_solver.py:216-253), for domains whose dense grid is too large
        self.sparse_grid = False
