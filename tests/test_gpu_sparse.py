"""Sparse grids (MPMConfig.sparse_grid; aq_params.sparse): only the grid
blocks around particles are stored, in node pools reached through a block
table, as the reference's pointer grid over a 4096^dim index space keeps
only active blocks (mpm_solver.py:216-253).

The sparse simulator must give the dense simulator's results: against the
oracle with the substep parity tolerance (2e-5 relative plus one
quantization step; 1e-8 in f64), including the out-of-tile path whose
writes hand out pool slots on touch, and against the dense simulator on a
1024^3 index space where the particles occupy well under 10 % of the blocks.
"""
import numpy as np
import pytest

from autoquantizer_b200 import _lib, scenes
from helpers import compare_states, twin

pytestmark = pytest.mark.gpu


def _sparse(cfg):
    cfg.sparse_grid = True
    return cfg


@pytest.mark.parametrize("jit", [True, False])
def test_sparse_mixed_boxes_3d_quantized_matches_oracle(jit):
    cfg, vals = scenes.mixed_boxes_3d(n=40000, n_grid=32)
    cfg.jit = jit
    s, o = twin(_sparse(cfg), vals)
    assert s.kernel_is_jit() == jit
    for k in (1, 3):
        s.substeps(k)
        o.substeps(k)
        compare_states(s, o, 2e-5)
    fl, _ = s.status()
    assert fl == o.flags == 0


def test_sparse_dam_break_2d_matches_oracle():
    cfg, vals = scenes.dam_break_2d(n=8192, n_grid=128)
    s, o = twin(_sparse(cfg), vals)
    s.substeps(4)
    o.substeps(4)
    compare_states(s, o, 2e-5)
    assert s.status()[0] == 0


def test_sparse_out_of_tile_writes_claim_slots():
    # fast rigid motion without re-binning: particles leave the blocks the
    # last binning activated, so their writes hand out pool slots on touch
    cfg, vals = scenes.falling_block_3d(n=20000, n_grid=32)
    cfg.precision = "f64"
    cfg.sort_interval = 1000
    vals[:, 3] = 60.0
    vals[:, 5] = -60.0
    s, o = twin(_sparse(cfg), vals)
    s.substeps(1)
    o.substeps(1)
    slots0, occupied = s.sparse_blocks()
    s.substeps(49)
    o.substeps(49)
    compare_states(s, o, 1e-8)
    fl, fb = s.status()
    assert fl == 0 and fb > 0
    slots, occ2 = s.sparse_blocks()
    assert occ2 == occupied and slots > slots0  # handed out on touch, no re-binning


def test_sparse_grid_mass_matches_dense():
    import torch

    cfg, vals = scenes.mixed_boxes_3d(n=40000, n_grid=32)
    out = []
    for sparse in (False, True):
        c, v = scenes.mixed_boxes_3d(n=40000, n_grid=32)
        c.sparse_grid = sparse
        s, _ = twin(c, v)
        s.substeps(3)
        m = torch.zeros(32 ** 3, dtype=torch.float32, device="cuda")
        import ctypes as C

        _lib.check(_lib.lib().aq_sim_grid_mass(s._sim, C.c_void_p(m.data_ptr()), _lib.stream_ptr()))
        out.append(m.cpu().numpy())
    assert np.allclose(out[0], out[1], rtol=1e-5, atol=1e-12)
    assert out[0].sum() > 0


def test_sparse_1024_index_space_matches_dense():
    """500,000 particles in a block of 40 cells a side inside a 1024^3 grid:
    occupied blocks are about 0.1 % of the 256^3 blocks.  The dense run
    (69 GB of f64 grids) and the sparse one agree to 1e-8 relative (in f32
    the stiff block amplifies the different summation orders of the two
    into differences of C far above rounding, as any two runs would)."""
    from autoquantizer_b200.mpm_solver import MPMSolver

    def run(sparse):
        cfg, vals = scenes.falling_block_3d(n=500000, n_grid=1024)
        cfg.dt = 5e-6
        cfg.precision = "f64"
        cfg.sparse_grid = sparse
        s = MPMSolver(cfg)
        s.set_particles(vals)
        s.substeps(10)
        fl, _ = s.status()
        assert fl == 0
        return s.state_values(), (s.sparse_blocks() if sparse else None)

    dense, _ = run(False)
    sparse, (slots, occupied) = run(True)
    assert 0 < occupied <= slots < 0.1 * 256 ** 3
    for k in range(dense.shape[1]):
        scale = max(1.0, float(np.abs(dense[:, k]).max()))
        assert np.max(np.abs(sparse[:, k] - dense[:, k])) <= 1e-8 * scale, k
