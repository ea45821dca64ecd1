"""The hand-written adjoint (aq_adjoint_*) against central finite
differences of the forward substep, in f64.

Perturbations are small (h = 1e-7 relative) so that no particle's B-spline
base cell changes between the two evaluations; the directional derivative
from the adjoint must then agree with the difference quotient to 1e-5
relative.  The sensitivity sum is checked against its definition
(sum over t = 1..T-1 of |dL/ds_t|^2, t split out with the autograd
Function)."""
import numpy as np
import pytest

from autoquantizer_b200 import _lib, scenes
from autoquantizer_b200.adjoint import Adjoint, ek_loss, ek_seed, rollout
from autoquantizer_b200.mpm_solver import MPMSolver

pytestmark = pytest.mark.gpu


def _setup(cfg, vals, n_grid=None):
    import torch

    cfg.precision = "f64"
    cfg.use_quantaichi = False
    cfg.materials = None
    s = MPMSolver(cfg)
    s.set_particles(vals[:, : s.n_slots()])
    P = s._params()
    adj = Adjoint(P)
    s0 = torch.from_numpy(np.ascontiguousarray(vals[:, : s.n_slots()])).cuda().double()
    return s, adj, s0


def _fd_check(cfg, vals, T, every, seed=0, h=1e-7, prep=None):
    import torch

    s, adj, s0 = _setup(cfg, vals)
    if prep is not None:
        prep(s, adj)
    rng = np.random.default_rng(seed)
    ns = s0.shape[1]
    r = torch.from_numpy(rng.normal(size=(s0.shape[0], cfg.dim))).cuda()

    def loss(st):
        return float((r * st[:, : cfg.dim]).sum() + (st[:, cfg.dim:2 * cfg.dim] ** 2).sum())

    sT = adj.forward(s0, T, every)
    seed_t = torch.zeros_like(sT)
    seed_t[:, : cfg.dim] = r
    seed_t[:, cfg.dim:2 * cfg.dim] = 2 * sT[:, cfg.dim:2 * cfg.dim]
    g0, sens = adj.backward(seed_t)
    # direction: per slot scaled to the slot's magnitude
    scale = torch.clamp(s0.abs().max(0).values, min=1e-3)
    scale[: cfg.dim] = 1.0 / s.n_grid  # positions: a fraction of a cell
    dirn = torch.from_numpy(rng.normal(size=s0.shape)).cuda() * scale
    lp = loss(adj.forward(s0 + h * dirn, T, every))
    lm = loss(adj.forward(s0 - h * dirn, T, every))
    fd = (lp - lm) / (2 * h)
    an = float((g0 * dirn).sum())
    assert an == pytest.approx(fd, rel=1e-5, abs=1e-9 * max(1.0, abs(fd))), (an, fd)
    assert np.all(np.isfinite(sens)) and np.all(sens >= 0)
    adj.close()
    return sens


def test_fd_elastic_2d_corotated():
    cfg, vals = scenes.elastic_block_2d(n=1024, n_grid=32)
    cfg.dt = 2e-4
    _fd_check(cfg, vals, T=12, every=5)


def test_fd_elastic_3d_reference_law():
    cfg, vals = scenes.falling_block_3d(n=2000, n_grid=16)
    _fd_check(cfg, vals, T=8, every=3)


def test_fd_fluid_2d_J():
    # away from the walls: at a wall node whose velocity component is exactly
    # 0 (particles at rest) the wall mask v_k < 0 has a kink that central
    # differences straddle
    cfg, vals = scenes.dam_break_2d(n=1024, n_grid=32, quantized=False)
    vals[:, 0] += 0.25
    vals[:, 1] += 0.2
    _fd_check(cfg, vals, T=10, every=4)


def test_fd_fluid_3d_with_F():
    cfg, vals = scenes.falling_block_3d(n=2000, n_grid=16)
    cfg.materials = None
    cfg.use_fluid = False
    s = MPMSolver(cfg)
    P = s._params()
    P.mat[0].kind = _lib.AQ_MAT_FLUID
    P.mat[0].lam = 1e3
    import torch

    cfg.precision = "f64"
    P.precision = 1
    P.n_particles = vals.shape[0]
    adj = Adjoint(P)
    s0 = torch.from_numpy(np.ascontiguousarray(vals)).cuda().double()
    sT = adj.forward(s0, 6, 2)
    seed = torch.zeros_like(sT)
    seed[:, 3:6] = 2 * sT[:, 3:6]
    g0, _ = adj.backward(seed)
    rng = np.random.default_rng(3)
    dirn = torch.from_numpy(rng.normal(size=s0.shape)).cuda() * 1e-2
    dirn[:, :3] /= 16
    h = 1e-7
    f = lambda st: float((st[:, 3:6] ** 2).sum())  # noqa: E731
    fd = (f(adj.forward(s0 + h * dirn, 6, 2)) - f(adj.forward(s0 - h * dirn, 6, 2))) / (2 * h)
    assert float((g0 * dirn).sum()) == pytest.approx(fd, rel=1e-5)


def test_sensitivity_is_sum_of_squared_state_gradients():
    import torch

    cfg, vals = scenes.elastic_block_2d(n=512, n_grid=32)
    s, adj, s0 = _setup(cfg, vals)
    T = 6
    sT = adj.forward(s0, T, 2)
    seed = ek_seed(sT, 2, s.p_mass, s.g)
    _, sens = adj.backward(seed)
    # dL/ds_t for each t = 1..T-1 via split rollouts
    total = np.zeros_like(sens)
    for t in range(1, T):
        a1 = Adjoint(s._params())
        a2 = Adjoint(s._params())
        st = a1.forward(s0, t, 2).requires_grad_(True)
        sT2 = rollout(st, a2, T - t, 2)
        assert torch.allclose(sT2, sT, rtol=1e-12, atol=1e-14)
        L = (sT2[:, 2:4] ** 2).sum()
        (g,) = torch.autograd.grad(L, st)
        total += (g ** 2).sum(0).cpu().numpy()
        a1.close()
        a2.close()
    assert sens == pytest.approx(total, rel=1e-9)


def test_rollout_autograd_matches_backward():
    import torch

    cfg, vals = scenes.dam_break_2d(n=512, n_grid=32, quantized=False)
    s, adj, s0 = _setup(cfg, vals)
    x = s0.clone().requires_grad_(True)
    sT = rollout(x, adj, 5, 2)
    L = (sT[:, 2:4] ** 2).sum() + sT[:, 1].sum()
    L.backward()
    assert x.grad is not None and torch.isfinite(x.grad).all()
    assert adj.sens is not None and (adj.sens >= 0).all()


def test_mpmsolver_ad_entry_points():
    cfg, vals = scenes.elastic_block_2d(n=1024, n_grid=32)
    cfg.precision = "f64"
    cfg.n_timesteps = 33
    s = MPMSolver(cfg)
    s.set_particles(vals)
    loss = s.run_forward_with_ad_nlogn(every=8)
    g = s.get_gradients()
    assert g.shape == (12,) and np.all(g > 0)
    # forward loss agrees with the main simulator on the same scene
    s2 = MPMSolver(cfg)
    s2.set_particles(vals)
    assert s2.run_forward_only() == pytest.approx(loss, rel=1e-8)
    assert ek_loss(s._ad_final, 2, s.p_mass, s.g) == pytest.approx(loss)


def test_fd_elastic_3d_with_collider():
    """The rotating SDF collider in the adjoint (sdf_collision_no_arg and its
    gradient): a block resting on a rotating bar, FD-checked; the collider
    changes the gradient."""
    import torch

    from test_gpu_collider import _scene, bar_sdf

    cfg, vals = _scene()
    sdf, normal = bar_sdf()
    t_sdf = torch.from_numpy(sdf.astype(np.float32)).cuda()
    t_nrm = torch.from_numpy(normal.astype(np.float32)).cuda()

    def prep(s, adj):
        adj.set_collider(t_sdf, t_nrm, (0, 0, 0), 32, theta=0.3, height=0.0, omega=5.0, height_rate=0.1)

    with_col = _fd_check(cfg, vals, T=8, every=3, prep=prep)
    cfg2, vals2 = _scene()
    without = _fd_check(cfg2, vals2, T=8, every=3)
    assert np.max(np.abs(with_col - without) / (np.abs(without) + 1e-30)) > 1e-3


@pytest.mark.parametrize("T", [1, 7, 16, 37])
def test_bisection_checkpointing_matches_segments(T):
    """every = 0 selects the logarithmic-memory scheme (the reference's
    nlogn stash, restated as bisection): the same final state, gradient of
    the initial state and sensitivity sums as checkpoints every 4 substeps
    (f64; both recompute the same substeps, so they agree to rounding of the
    grid sums' order)."""
    import torch

    cfg, vals = scenes.falling_block_3d(n=6000, n_grid=32)
    _, adj, s0 = _setup(cfg, vals)
    rng = np.random.default_rng(T)
    sT_a = adj.forward(s0, T, 4)
    seed = torch.from_numpy(rng.normal(size=sT_a.shape)).cuda()
    g_a, sens_a = adj.backward(seed)
    g_a = g_a.clone()
    sens_a = np.array(sens_a)
    sT_b = adj.forward(s0, T, 0)
    g_b, sens_b = adj.backward(seed)
    assert torch.allclose(sT_a, sT_b, rtol=1e-12, atol=1e-12)
    assert torch.allclose(g_a, g_b, rtol=1e-9, atol=1e-9 * float(g_a.abs().max()))
    np.testing.assert_allclose(sens_b, sens_a, rtol=1e-9, atol=0)
    adj.close()


def test_run_forward_with_ad_nlogn_bisection_matches_segments():
    """MPMSolver.run_forward_with_ad_nlogn with every=0 (logarithmic stash)
    and with segments of 8 substeps: same loss and sensitivities."""
    cfg, vals = scenes.falling_block_3d(n=6000, n_grid=32)
    cfg.precision = "f64"
    cfg.n_timesteps = 25
    out = []
    for every in (8, 0):
        s = MPMSolver(cfg)
        s.set_particles(vals[:, : s.n_slots()])
        loss = s.run_forward_with_ad_nlogn(every=every)
        out.append((loss, np.asarray(s.get_gradients(), dtype=np.float64).ravel()))
    assert out[0][0] == pytest.approx(out[1][0], rel=1e-12)
    np.testing.assert_allclose(out[1][1], out[0][1], rtol=1e-9)


def test_fp32_adjoint_matches_fp64_on_every_slot():
    """The FP32 adjoint against the FP64 adjoint, which the difference tests
    above pin, on the 3D falling block (32,768 particles, 32^3, 64 substeps,
    checkpoints every 16), for every slot, v and C included (FP32 central
    differences cannot resolve those).  The slots' sensitivities span 19
    decades (x_y 3e-3, v_y 1e-8, F 1e-12..1e-14, x_x and v_x 1e-17, C
    1e-21), and FP32 resolves the small ones only relative to the large
    ones: the dominant slots (x, v_y) agree to 1e-2 relative, the others
    to a factor of 4.  What the solver takes from them is a width,
    log2(S R^2) / 2 up to constants: the error-bound scheme from the FP32
    sensitivities is the FP64 one's within one bit in every slot."""
    import copy

    import torch

    cfg, vals = scenes.falling_block_3d(n=32768, n_grid=32)
    cfg.use_quantaichi = False
    cfg.materials = None
    out = {}
    for prec in ("f32", "f64"):
        c = copy.deepcopy(cfg)
        c.precision = prec
        s = MPMSolver(c)
        ns = s.n_slots()
        s.set_particles(vals[:, :ns])
        adj = Adjoint(s._params())
        s0 = torch.from_numpy(np.ascontiguousarray(vals[:, :ns])).cuda()
        sT = adj.forward(s0, 64, 16)
        _, sens = adj.backward(ek_seed(sT, 3, s.p_mass, s.g))
        out[prec] = np.asarray(sens, dtype=np.float64)
        adj.close()
    s32, s64 = out["f32"], out["f64"]
    print("sensitivities f64:", np.array2string(s64, precision=3))
    print("sensitivities f32/f64:", np.array2string(s32 / s64, precision=4))
    assert s32.shape == s64.shape == (24,)
    assert np.all(s64 > 0) and np.all(s32 > 0)
    dominant = [0, 1, 2, 4]
    np.testing.assert_allclose(s32[dominant], s64[dominant], rtol=1e-2)
    assert np.all(np.abs(np.log2(s32 / s64)) < 2.0)
    from autoquantizer_b200.solvers import LagrangianEB

    ranges = np.array([1.0] * 3 + [2.0] * 3 + [64.0] * 9 + [2.0] * 9)
    b32, _ = LagrangianEB(s32 * ranges ** 2, ref=1.0, tol_rel=1e-3)
    b64, _ = LagrangianEB(s64 * ranges ** 2, ref=1.0, tol_rel=1e-3)
    print("error-bound widths f64:", b64.tolist(), "f32:", b32.tolist())
    assert np.all(np.abs(b32 - b64) <= 1), (b32, b64)
