"""GPU parity at the benchmark configurations' full sizes, and on the
out-of-tile path of the fused substep.

The CUDA substep runs from the same packed records as the oracle (the CPU
restatement of mpm_solver.py's p2g/grid_op/g2p, OpenMP on every host core
for the full-size scenes) and every slot of every particle is compared:

  elastic block 2D    8,192 particles, 128^2 grid, plain f32 state
  dam break 2D        65,536 particles, 256^2 grid, quantized (x 2x20
                      fixed, v 2x13 + shared 6-bit exponent, C 4x16, J 16),
                      dithering on
  mixed boxes 3D      2,097,152 particles, 128^3 grid, quantized (x 3x21,
                      v 3x12 + shared exponent, C 9x16, F 9x16, material id)
                      and FP32 state

The two add the grid sums in different orders, so agreement is to rounding,
not bit for bit.  Per substep (compare_states): f32 state within 2e-5
relative to max(1, max |value|) of the slot, plus one quantization step of
fixed-point slots where a dithered rounding lands on the neighbouring code.
Quantized runs are checked two ways.  Substep by substep, with the
oracle re-started from the GPU's records after every substep, every slot of
every particle must meet that bound.  Run freely over many substeps, the
last-bit differences of the grid sums flip roundings (dithered fixed point,
round-to-nearest shared-exponent digits) here and there, and a flipped v or
x code moves its neighbours' next C by several C steps (C varies with the
grid velocity as 4 inv_dx times its difference across a cell), so free runs
are held to compare_states_stats: every position within two codes, at most
2e-3 of the particles beyond the per-slot bound, mean errors below a tenth
of it.

The out-of-tile tests move the particles fast with re-binning switched off,
so that particles leave the grid tile staged for their block: G2P then
gathers from the global grid and P2G scatters with global vector reductions
(aq_kernels.cuh, the !in_tile branches).  They assert that the branch ran
(status fallbacks > 0) and still matches the oracle.  Fast rigid motion
makes C a difference of large products (C of a uniform velocity field is
zero), whose f32 rounding the elastic response then amplifies, so the
unquantized variants run in f64 (1e-8 relative) where that noise is 1e-12.
"""
import pytest

from autoquantizer_b200 import scenes
from helpers import compare_states, compare_states_stats, host_threads, twin

pytestmark = pytest.mark.gpu


def _twin(cfg, vals, threads=1, sort_interval=16):
    cfg.sort_interval = sort_interval
    s, o = twin(cfg, vals, threads=threads)
    assert s.kernel_is_jit()
    return s, o


def _resynced(s, o, k, rel=2e-5):
    """k single substeps; after each, every slot of every particle against
    the oracle's substep from the same records, then the oracle continues
    from the GPU's records."""
    for _ in range(k):
        s.substeps(1)
        o.substeps(1)
        compare_states(s, o, rel)
        o.set_words(s.words())


def _clean(s, o):
    fl, fb = s.status()
    assert fl == o.flags == 0
    return fb


def test_elastic_block_2d_full_size_f32():
    cfg, vals = scenes.elastic_block_2d()
    assert vals.shape[0] == 8192 and cfg.n_grid == 128
    s, o = _twin(cfg, vals, threads=host_threads())
    s.substeps(32)
    o.substeps(32)
    compare_states(s, o, 2e-5)
    _clean(s, o)


def test_dam_break_2d_full_size_quantized_dithered():
    cfg, vals = scenes.dam_break_2d()
    assert vals.shape[0] == 65536 and cfg.n_grid == 256 and cfg.use_dithering
    s, o = _twin(cfg, vals, threads=host_threads())
    _resynced(s, o, 8)
    s, o = _twin(cfg, vals, threads=host_threads())
    s.substeps(16)  # fused, free-running
    o.substeps(16)
    compare_states_stats(s, o, max_frac=2e-3)
    _clean(s, o)


@pytest.mark.parametrize("quantized", [True, False], ids=["quantized", "fp32_state"])
def test_mixed_boxes_3d_full_size(quantized):
    cfg, vals = scenes.mixed_boxes_3d(quantized=quantized)
    assert vals.shape[0] == 2097152 and cfg.n_grid == 128
    s, o = _twin(cfg, vals, threads=host_threads())
    if quantized:
        _resynced(s, o, 8)
        s, o = _twin(cfg, vals, threads=host_threads())
        s.substeps(8)  # fused, free-running
        o.substeps(8)
        compare_states_stats(s, o, max_frac=2e-3)
    else:
        s.substeps(8)
        o.substeps(8)
        compare_states(s, o, 2e-5)
    _clean(s, o)


def test_out_of_tile_path_3d_matches_oracle():
    # a block moving 2.3 cells in +x and -z over the run, never re-binned:
    # a +1 cell drift already leaves the 3D tile
    cfg, vals = scenes.falling_block_3d(n=20000, n_grid=32)
    cfg.precision = "f64"
    vals[:, 3] = 60.0
    vals[:, 5] = -60.0
    s, o = _twin(cfg, vals, sort_interval=1000)
    s.substeps(24)
    o.substeps(24)
    compare_states(s, o, 1e-8)
    assert _clean(s, o) > 0


def test_out_of_tile_path_2d_matches_oracle():
    # the 2D tile keeps one cell of slack: move 4 cells in +x and -y
    cfg, vals = scenes.elastic_block_2d(n=4096)
    cfg.precision = "f64"
    vals[:, 2] = 40.0
    vals[:, 3] = -40.0
    s, o = _twin(cfg, vals, sort_interval=1000)
    s.substeps(8)
    o.substeps(8)
    compare_states(s, o, 1e-8)
    assert _clean(s, o) > 0


def test_out_of_tile_path_quantized_matches_oracle():
    # quantized, dithered fluid moving 3 cells (f64 compute and grid, so
    # that C is free of the f32 cancellation of fast motion): substep by
    # substep from the same records, every slot of every particle
    cfg, vals = scenes.dam_break_2d(n=8192, n_grid=128)
    cfg.dt = 1e-4
    cfg.precision = cfg.compute_fp = "f64"
    vals[:, 2] = 20.0
    vals[:, 3] = -20.0
    s, o = _twin(cfg, vals, sort_interval=1000)
    _resynced(s, o, 12, rel=1e-8)
    assert _clean(s, o) > 0
