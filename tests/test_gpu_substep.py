"""GPU substep parity: libaq's fused P2G/grid/G2P against the oracle's scalar
restatement of mpm_solver.py, from identical packed records.

Atomic accumulation order differs between the two, so values agree to
floating-point tolerance, not bit for bit: f32 state within 2e-5 relative
(plus one quantization step of the slot for fixed-point slots, since a
dithered rounding can land on the neighbouring code), f64 state within 1e-8
(relative to max(1, max |value|) of the slot).
"""
import numpy as np
import pytest

from autoquantizer_b200 import _lib, scenes
from helpers import quant_steps, twin

pytestmark = pytest.mark.gpu


def _compare(s, o, rel, steps_slack=1.0):
    g = s.state_values()
    r = o.get_state()
    assert g.shape == r.shape
    q = quant_steps(s)
    for k in range(g.shape[1]):
        scale = max(1.0, float(np.max(np.abs(r[:, k]))))
        tol = rel * scale
        if q[k] > 0:
            tol += steps_slack * q[k]
        elif np.isnan(q[k]):  # float with exponent: relative to the value
            tol += 2.0 ** -10 * scale
        err = float(np.max(np.abs(g[:, k] - r[:, k])))
        assert err <= tol, "slot %d: max err %g > tol %g" % (k, err, tol)


def _run(cfg, vals, k, rel, sort_interval=16, jit=True):
    cfg.sort_interval = sort_interval
    cfg.jit = jit
    s, o = twin(cfg, vals)
    assert s.kernel_is_jit() == jit
    s.substeps(k)
    o.substeps(k)
    _compare(s, o, rel)
    fl, _ = s.status()
    assert fl == o.flags == 0
    return s, o


def test_elastic_2d_f32_raw():
    cfg, vals = scenes.elastic_block_2d(n=4096)
    _run(cfg, vals, 5, 2e-5)


def test_elastic_2d_f64_raw():
    cfg, vals = scenes.elastic_block_2d(n=4096)
    cfg.precision = "f64"
    _run(cfg, vals, 5, 1e-8)


@pytest.mark.parametrize("jit", [True, False])
def test_dam_break_2d_quantized(jit):
    cfg, vals = scenes.dam_break_2d(n=8192, n_grid=128)
    _run(cfg, vals, 4, 2e-5, jit=jit)


def test_dam_break_2d_quantized_unfused_matches_fused():
    # substep() one at a time runs P2G / grid / G2P as separate launches
    cfg, vals = scenes.dam_break_2d(n=4096, n_grid=128)
    s, o = twin(cfg, vals)
    for _ in range(3):
        s.substep()
    o.substeps(3)
    _compare(s, o, 2e-5)


def test_falling_block_3d_reference_law_f32():
    cfg, vals = scenes.falling_block_3d(n=20000, n_grid=32)
    _run(cfg, vals, 4, 2e-5)


def test_falling_block_3d_reference_law_f64():
    cfg, vals = scenes.falling_block_3d(n=20000, n_grid=32)
    cfg.precision = "f64"
    _run(cfg, vals, 4, 1e-8)


@pytest.mark.parametrize("jit", [True, False])
def test_mixed_boxes_3d_quantized(jit):
    cfg, vals = scenes.mixed_boxes_3d(n=40000, n_grid=32)
    _run(cfg, vals, 3, 2e-5, jit=jit)


def test_mixed_boxes_3d_fp32_state():
    cfg, vals = scenes.mixed_boxes_3d(n=40000, n_grid=32, quantized=False)
    _run(cfg, vals, 3, 2e-5)


@pytest.mark.parametrize("interval", [1, 3, 1000])
def test_rebinning_interval_does_not_change_results(interval):
    cfg, vals = scenes.falling_block_3d(n=8000, n_grid=32)
    _run(cfg, vals, 6, 2e-5, sort_interval=interval)


def test_fluid_3d_quantized_with_J():
    cfg, vals = scenes.falling_block_3d(n=12000, n_grid=32)
    cfg.use_fluid = True
    cfg.la = 1e3
    cfg.use_quantaichi = True
    cfg.use_dithering = True
    cfg.compute_fp = "f32"
    cfg.quantized_properties = {"x": 1, "v": 1, "C": 1, "J": 1}
    cfg.quant_bits = np.array([21] * 3 + [16] * 3 + [16] * 9 + [16])
    cfg.quant_ranges = np.array([1.0] * 3 + [4.0] * 3 + [64.0] * 9 + [0.5])
    d = 3
    v2 = np.zeros((vals.shape[0], 2 * d + d * d + 1))
    v2[:, :d] = vals[:, :d]
    v2[:, -1] = 1.0
    _run(cfg, v2, 4, 2e-5)


def test_loss_matches_oracle():
    cfg, vals = scenes.elastic_block_2d(n=4096)
    cfg.precision = "f64"
    s, o = _run(cfg, vals, 8, 1e-8)
    assert s.compute_loss() == pytest.approx(o.loss(), rel=1e-9)


def test_out_of_domain_sets_status_without_fault():
    # host-side fault injection: a particle outside the grid is clamped and
    # reported, never dereferenced out of bounds
    cfg, vals = scenes.falling_block_3d(n=4000, n_grid=32)
    vals[17, 0] = 1.7
    vals[18, 1] = -0.4
    s, o = twin(cfg, vals)
    s.substeps(2)
    fl, _ = s.status(clear=True)
    assert fl & _lib.AQ_ST_OUT_OF_DOMAIN
    assert s.status()[0] == 0


def test_nan_particle_sets_status():
    cfg, vals = scenes.falling_block_3d(n=4000, n_grid=32)
    vals[5, 2] = np.nan
    s, _ = twin(cfg, vals)
    s.substeps(1)
    fl, _ = s.status(clear=True)
    assert fl & _lib.AQ_ST_NAN


@pytest.mark.parametrize("jit", [True, False])
@pytest.mark.parametrize("n", [1001, 20037])
def test_partial_record_group_matches_oracle(jit, n):
    """Records are stored in groups of 32 with interleaved word pairs; a
    particle count that is not a multiple of 32 leaves the last group
    partial.  The substeps (re-binning included) still match the oracle, and
    words written through the C ABI come back unchanged."""
    cfg, vals = scenes.mixed_boxes_3d(n=n, n_grid=32)
    s, o = _run(cfg, vals, 3, 2e-5, sort_interval=2, jit=jit)
    w = s.words()
    assert w.shape == (n, s.layout().n_words)
    s.set_words(w)
    assert np.array_equal(s.words(), w)
    s.substeps(2)
    o.substeps(2)
    _compare(s, o, 2e-5)
