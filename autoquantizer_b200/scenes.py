"""Seeded synthetic scenes of the benchmark configurations.

Each builder returns an MPMConfig and the initial particle values (n x
n_slots, float64, record slot order x, v, C, F|J[, material id]).  All
randomness comes from numpy default_rng(seed).

  elastic_block_2d   2D elastic block, plain FP32 state: 128^2 grid,
                     8192 particles jittered in a 0.2 box at (0.4, 0.6),
                     E 1e4, nu 0.2, rho 1, dt 1e-4, walls 3 cells.
  dam_break_2d       2D weakly compressible fluid, quantized: 256^2,
                     65,536 particles in [0.05,0.45]x[0.05,0.65], bulk
                     modulus 400, dt 5e-5; x 2x20-bit fixed on range 1,
                     v 2x13-bit digits + shared 6-bit exponent, C 4x16 on
                     range 64, J 16-bit on [0.5, 1.5]; dithering on.
  mixed_boxes_3d     3D throughput scene: 128^3, 2,097,152 particles in 4
                     random boxes (2 fixed-corotated elastic, E log-uniform
                     in [1e3,1e5], nu in [0.2,0.4]; 2 fluid), dt 2e-5;
                     x 3x21 fixed, v 3x12 digits + shared 6-bit exponent,
                     C 9x16 fixed, F 9x16 fixed on range 2.
  falling_block_3d   3D elastic block falling on the floor: 64^3, 262,144
                     particles, E 5e3, nu 0.3, dt 5e-5.
"""
import numpy as np

from . import _lib
from .mpm_config import MPMConfig


def _base(dim, n_grid, n, dt):
    c = MPMConfig()
    c.dim, c.n_grid, c.n_particles, c.dt = dim, n_grid, n, dt
    c.p_rho = 1.0
    c.p_vol = (1.0 / n_grid * 0.5) ** dim
    c.size = 1.0
    c.bound = [3] * dim
    c.use_friction = False
    c.use_bls = True
    c.precision = "f32"
    c.compute_fp = "f32"
    c.grid_res = [n_grid] * dim
    return c


def _values(cfg, x, mat=None):
    d = cfg.dim
    n = x.shape[0]
    has_F = not cfg.use_fluid
    ns = 2 * d + d * d + (d * d if has_F else 1) + (1 if cfg.materials else 0)
    v = np.zeros((n, ns), dtype=np.float64)
    v[:, :d] = x
    if has_F:
        v[:, 2 * d + d * d:2 * d + 2 * d * d] = np.eye(d).ravel()
    else:
        v[:, 2 * d + d * d] = 1.0
    if cfg.materials:
        v[:, -1] = mat
    return v


def elastic_block_2d(seed=0, n=8192, n_grid=128):
    c = _base(2, n_grid, n, 1e-4)
    c.use_fluid = False
    c.E, c.nu = 1e4, 0.2
    c.n_timesteps = 2001
    rng = np.random.default_rng(seed)
    m = int(round(np.sqrt(n)))
    i, j = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    cell = 0.2 / m
    x = np.stack([0.4 + (i.ravel() + rng.random(m * m)) * cell, 0.6 + (j.ravel() + rng.random(m * m)) * cell], 1)
    return c, _values(c, x[:n])


def dam_break_2d(seed=0, n=65536, n_grid=256, quantized=True):
    c = _base(2, n_grid, n, 5e-5)
    c.use_fluid = True
    c.la = 400.0
    c.n_timesteps = 4001
    if quantized:
        c.use_quantaichi = c.use_bitpack = True
        c.use_dithering = True
        c.quantized_properties = {"x": 1, "v": 1, "C": 1, "J": 1}
        c.quant_bits = np.array([20, 20, 13, 13, 16, 16, 16, 16, 16])
        c.quant_ranges = np.array([1.0, 1.0, 1.0, 1.0, 64.0, 64.0, 64.0, 64.0, 0.5])
        c.v_exp_bits = 6
    rng = np.random.default_rng(seed)
    x = np.stack([0.05 + 0.4 * rng.random(n), 0.05 + 0.6 * rng.random(n)], 1)
    return c, _values(c, x)


C3_BITS = [21] * 3 + [12] * 3 + [16] * 9 + [16] * 9
C3_RANGES = [1.0] * 3 + [1.0] * 3 + [64.0] * 9 + [2.0] * 9


def mixed_boxes_3d(seed=0, n=2097152, n_grid=128, quantized=True, precision="f32", c_range=64.0):
    c = _base(3, n_grid, n, 2e-5)
    c.use_fluid = False
    c.n_timesteps = 1001
    c.precision = precision
    rng = np.random.default_rng(seed)
    E = 10 ** rng.uniform(3, 5, 2)
    nu = rng.uniform(0.2, 0.4, 2)
    c.materials = [(_lib.AQ_MAT_COROTATED, E[0], nu[0], 0.0), (_lib.AQ_MAT_COROTATED, E[1], nu[1], 0.0),
                   (_lib.AQ_MAT_FLUID, 0.0, 0.0, 1e4), (_lib.AQ_MAT_FLUID, 0.0, 0.0, 1e4)]
    if quantized:
        c.use_quantaichi = c.use_bitpack = True
        c.use_dithering = True
        c.quantized_properties = {"x": 1, "v": 1, "C": 1, "F": 1}
        c.quant_bits = np.array(C3_BITS)
        r = list(C3_RANGES)
        r[6:15] = [c_range] * 9
        c.quant_ranges = np.array(r)
        c.v_exp_bits = 6
    # four boxes with edges in [0.25, 0.4], inside [0.08, 0.92]^3, particles
    # split by volume
    sizes = rng.uniform(0.25, 0.4, (4, 3))
    lows = np.array([rng.uniform(0.08, 0.92 - s) for s in sizes.ravel()]).reshape(4, 3)
    vol = sizes.prod(1)
    counts = np.floor(n * vol / vol.sum()).astype(np.int64)
    counts[-1] = n - counts[:-1].sum()
    xs, ms = [], []
    for b in range(4):
        xs.append(lows[b] + rng.random((counts[b], 3)) * sizes[b])
        ms.append(np.full(counts[b], b, dtype=np.float64))
    x = np.concatenate(xs)
    return c, _values(c, x, np.concatenate(ms))


def mixed_boxes_3d_device(seed=0, n=2097152, n_grid=128):
    """The 3D throughput scene generated on the GPU (for sizes whose
    n x n_slots values would not fit host memory): the same configuration,
    box layout and materials as mixed_boxes_3d (numpy default_rng(seed)),
    particle positions drawn with torch's CUDA generator (seeded with seed),
    dt scaled with the cell size (2e-5 at 128 cells).  Returns the config and
    a CUDA float32 tensor (n x n_slots) for MPMSolver.set_particles."""
    import torch

    c, _ = mixed_boxes_3d(seed=seed, n=4, n_grid=n_grid)
    c.n_particles = n
    c.dt = 2e-5 * 128.0 / n_grid
    rng = np.random.default_rng(seed)
    rng.uniform(3, 5, 2), rng.uniform(0.2, 0.4, 2)  # the draws mixed_boxes_3d spends on the materials
    sizes = rng.uniform(0.25, 0.4, (4, 3))
    lows = np.array([rng.uniform(0.08, 0.92 - s) for s in sizes.ravel()]).reshape(4, 3)
    vol = sizes.prod(1)
    counts = np.floor(n * vol / vol.sum()).astype(np.int64)
    counts[-1] = n - counts[:-1].sum()
    ns = 2 * 3 + 9 + 9 + 1
    gen = torch.Generator(device="cuda")
    gen.manual_seed(int(seed))
    vals = torch.zeros((n, ns), dtype=torch.float32, device="cuda")
    vals[:, 15] = vals[:, 19] = vals[:, 23] = 1.0  # F = I
    at = 0
    for b in range(4):
        k = int(counts[b])
        lo = torch.tensor(lows[b], dtype=torch.float32, device="cuda")
        sz = torch.tensor(sizes[b], dtype=torch.float32, device="cuda")
        vals[at:at + k, :3] = lo + torch.rand((k, 3), generator=gen, device="cuda") * sz
        vals[at:at + k, 24] = float(b)
        at += k
    return c, vals


def falling_block_3d(seed=0, n=262144, n_grid=64):
    c = _base(3, n_grid, n, 5e-5)
    c.use_fluid = False
    c.E, c.nu = 5e3, 0.3
    c.n_timesteps = 257
    rng = np.random.default_rng(seed)
    side = (n / (8 * n_grid ** 3)) ** (1 / 3)
    x = np.array([0.5 - side / 2, 0.3, 0.5 - side / 2]) + rng.random((n, 3)) * side
    return c, _values(c, x)
