"""aq_sim_field_stats (the surrogate's feature statistics) against numpy on
the decoded state, and device-tensor initial values against host ones."""
import numpy as np
import pytest
import torch

from autoquantizer_b200 import scenes
from autoquantizer_b200.mpm_solver import MPMSolver

pytestmark = pytest.mark.gpu


def _scene():
    cfg, vals = scenes.mixed_boxes_3d(n=20000, n_grid=32)
    return cfg, vals


def test_field_stats_match_numpy():
    cfg, vals = _scene()
    s = MPMSolver(cfg)
    s.set_particles(vals)
    s.substeps(4)
    ref = torch.from_numpy(vals).cuda()
    st = s.field_stats(reference=ref)
    b = s.state_values()
    assert st.shape == (b.shape[1], 5)
    assert st[:, 0] == pytest.approx(np.abs(b).sum(0), rel=1e-12, abs=1e-12)
    assert st[:, 1] == pytest.approx(b.sum(0), rel=1e-9, abs=1e-9)
    assert st[:, 2] == pytest.approx((b * b).sum(0), rel=1e-12, abs=1e-12)
    assert np.array_equal(st[:, 3], np.abs(b).max(0))
    assert st[:, 4] == pytest.approx(np.abs(b - vals).sum(0), rel=1e-12, abs=1e-12)
    st32 = s.field_stats(reference=ref.float())
    assert st32[:, 4] == pytest.approx(np.abs(b - vals.astype(np.float32)).sum(0), rel=1e-9, abs=1e-9)
    no_ref = s.field_stats()
    assert np.array_equal(no_ref[:, :4], st[:, :4]) and not no_ref[:, 4].any()


def test_field_stats_rejects_bad_reference():
    cfg, vals = _scene()
    s = MPMSolver(cfg)
    s.set_particles(vals)
    with pytest.raises(ValueError):
        s.field_stats(reference=torch.zeros((3, 3), device="cuda"))


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_device_initial_values_match_host(dtype):
    cfg, vals = _scene()
    a = MPMSolver(cfg)
    a.set_particles(vals.astype(np.float32).astype(np.float64) if dtype == torch.float32 else vals)
    b = MPMSolver(cfg)
    b.set_particles(torch.from_numpy(vals).to("cuda", dtype))
    assert np.array_equal(a.words(), b.words())
    a.substeps(3)
    b.substeps(3)
    # P2G sums with float atomics in no fixed order: equal up to rounding,
    # except where a dithered code lands on its neighbour (one quantization
    # step, up to 64 / 2^15 for C and 2^-11 of the shared exponent's scale
    # for v)
    sa, sb = a.state_values(), b.state_values()
    assert np.allclose(sa[:, :3], sb[:, :3], rtol=0, atol=1e-5)
    assert np.mean(np.abs(sa - sb) > 5e-3) < 1e-3


def test_device_generated_scene_matches_the_host_scene_layout():
    """mixed_boxes_3d_device: same boxes, materials and counts as the host
    generator, positions from the GPU generator; it runs clean."""
    cfg_h, vals_h = scenes.mixed_boxes_3d(seed=3, n=30000, n_grid=32)
    cfg_d, vals_d = scenes.mixed_boxes_3d_device(seed=3, n=30000, n_grid=32)
    v = vals_d.cpu().numpy()
    assert v.shape == vals_h.shape and cfg_d.n_particles == 30000 and cfg_d.dt == pytest.approx(2e-5 * 4)
    assert cfg_d.materials == cfg_h.materials and list(cfg_d.quant_bits) == list(cfg_h.quant_bits)
    for b in range(4):
        mh, md = vals_h[:, 24] == b, v[:, 24] == b
        assert mh.sum() == md.sum()
        lo, hi = vals_h[mh, :3].min(0), vals_h[mh, :3].max(0)
        assert np.all(v[md, :3] >= lo - 1e-3) and np.all(v[md, :3] <= hi + 1e-3)
    assert np.array_equal(v[:, 3:24], vals_h[:, 3:24].astype(np.float32))
    s = MPMSolver(cfg_d)
    s.set_particles(vals_d)
    s.substeps(4)
    assert s.status()[0] == 0
