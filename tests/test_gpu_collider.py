"""The rotating SDF collider (sdf_collision / rot_scene / step_collider,
mpm_solver.py:1459-1547) on the GPU against the oracle's restatement: an
elastic block dropped onto a rotating bar, FP32 state, same tolerance as the
substep parity tests."""
import numpy as np
import pytest

from autoquantizer_b200 import scenes
from helpers import compare_states, twin

pytestmark = pytest.mark.gpu


def bar_sdf(nx=64, ny=32, nz=64):
    """A bar along x through the rotation centre, 4 cells thick in y at
    height 8..12 and 8 cells wide in z; normals point up."""
    sdf = np.full((nx, ny, nz), 0.02)
    sdf[:, 8:12, nz // 2 - 4:nz // 2 + 4] = -0.01
    normal = np.zeros((nx, ny, nz, 3))
    normal[..., 1] = 1.0
    return sdf, normal


def _scene():
    cfg, vals = scenes.falling_block_3d(n=20000, n_grid=32)
    # a domain 2 n_grid wide in x and z with the rotation centre (32, ., 32)
    # in the middle, as in the reference's collider experiments
    cfg.grid_res = [64, 32, 64]
    cfg.ub = [61, 29, 61]
    vals = vals.copy()
    vals[:, 0] += 0.5
    vals[:, 2] += 0.5
    return cfg, vals


@pytest.mark.parametrize("steps,jit", [(1, True), (6, True), (6, False)])
def test_collider_matches_oracle(steps, jit):
    """jit False: the library's own nvcc-built kernel (collider always
    compiled in) instead of the layout-specialized one."""
    cfg, vals = _scene()
    cfg.jit = jit
    s, o = twin(cfg, vals)
    sdf, normal = bar_sdf()
    kw = dict(theta=0.3, height=0.0, omega=5.0, height_rate=0.1)
    s.init_sdf_value(sdf, normal, **kw)
    o.set_collider(sdf, normal, offset=(0, 0, 0), center=32, **kw)
    s.substeps(steps)
    o.substeps(steps)
    assert s.kernel_is_jit() == jit
    assert s.status()[0] == 0
    compare_states(s, o, 2e-5)
    th, hh = s.collider_state()
    assert th == pytest.approx(0.3 + 5.0 * cfg.dt * steps, rel=1e-12)
    assert hh == pytest.approx(0.1 * cfg.dt * steps, rel=1e-12)


def test_collider_changes_the_motion():
    cfg, vals = _scene()
    s_free, _ = twin(cfg, vals)
    s_col, _ = twin(cfg, vals)
    sdf, normal = bar_sdf()
    s_col.init_sdf_value(sdf, normal, theta=0.0, omega=5.0)
    s_free.substeps(20)
    s_col.substeps(20)
    a, b = s_free.state_values(), s_col.state_values()
    # particles over the bar keep their height, the others fall freely
    assert np.max(np.abs(a[:, 4] - b[:, 4])) > 1e-3


def test_autodiff_pass_runs_with_a_collider():
    """run_forward_with_ad_nlogn hands the collider (at its current angle and
    height) to the adjoint: finite sensitivities that differ from the run
    without it."""
    def grads(col):
        cfg, vals = _scene()
        cfg.precision, cfg.use_quantaichi, cfg.materials = "f64", False, None
        cfg.n_timesteps = 9
        from autoquantizer_b200.mpm_solver import MPMSolver

        s = MPMSolver(cfg)
        s.set_particles(vals[:, :s.n_slots()])
        if col:
            sdf, normal = bar_sdf()
            s.init_sdf_value(sdf, normal, theta=0.3)
        s.run_forward_with_ad_nlogn(every=4)
        return np.asarray(s.get_gradients(), dtype=np.float64).ravel()

    a, b = grads(True), grads(False)
    assert np.all(np.isfinite(a)) and np.all(a >= 0)
    assert not np.allclose(a, b, rtol=1e-6, atol=0)


def test_nlogn_step_forward_follows_the_autodiff_collider_schedule():
    """nlogn_step_forward(s) (mpm_solver.py:1161-1167) runs the autodiff
    path's substep, whose collider takes its velocity from the node itself
    (sdf_collision_no_arg), then puts the collider at step_collider_difftaichi
    (s): angle omega dt s, height 0.15 dt s.  Checked against the oracle run
    through the same schedule, and the pose after every call."""
    cfg, vals = _scene()
    s, o = twin(cfg, vals)
    sdf, normal = bar_sdf()
    s.init_sdf_value(sdf, normal, theta=0.3, omega=5.0)
    o.set_collider(sdf, normal, offset=(0, 0, 0), center=32, theta=0.3, omega=5.0, node_velocity=True)
    emitted = []
    for k in range(5):
        s.nlogn_step_forward(k, emit_func=lambda step, mpm: emitted.append(step))
        o.substeps(1)
        o.col_theta, o.col_height = 5.0 * cfg.dt * k, 0.15 * cfg.dt * k
        th, hh = s.collider_state()
        assert th == pytest.approx(5.0 * cfg.dt * k, abs=1e-15)
        assert hh == pytest.approx(0.15 * cfg.dt * k, abs=1e-15)
    assert emitted == list(range(5))
    assert s.status()[0] == 0
    compare_states(s, o, 2e-5)
    # the node-velocity form really differs from the forward substep's
    s2, _ = twin(cfg, vals)
    s2.init_sdf_value(sdf, normal, theta=0.3, omega=5.0)
    for k in range(5):
        s2.substep(k)
        s2.step_collider_difftaichi(k)
    assert not np.array_equal(s.words(), s2.words())


def test_substep_difftaichi_keeps_the_collider_pose():
    cfg, vals = _scene()
    s, _ = twin(cfg, vals)
    sdf, normal = bar_sdf()
    s.init_sdf_value(sdf, normal, theta=0.3, height=0.01, omega=5.0)
    s.substep_difftaichi(0, 1)
    assert s.collider_state() == pytest.approx((0.3, 0.01), abs=1e-15)
