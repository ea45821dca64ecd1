"""The experiment pipeline (-r, -a, -f) on the GPU.

Range detection is pinned to the ranges the reference shipped for its
deterministic 2D experiments (mpm_exps/ranges/elastic_2d/*.npy,
mpm_exps/ranges/fluid_2d/*.npy; values in tests/golden/reference_data.json).
The error-bound forward runs of the 2D elastic experiment, on the schemes
solved from the reference's shipped sensitivities and ranges, must meet the
success criterion of run_mpm_elastic_2d.py:190-205 (|loss - f64 loss| <
3 * eps * f64 loss).
"""
import json
import os

import numpy as np
import pytest

from autoquantizer_b200 import drivers as D

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_data.json")))


def test_elastic_2d_ranges_match_reference(tmp_path):
    exp = D.Elastic2D()
    out = D.detect_range(exp, exp.config(), str(tmp_path))
    ours = np.array(out["ranges"])
    a = np.array(GOLD["ranges"]["elastic_2d/elastic_2d.npy"])
    b = np.array(GOLD["ranges"]["elastic_2d/elastic_2d_t8193_dt0.0002_p80000_g128.npy"])
    print("elastic_2d ranges ours/reference:", np.array2string(ours / a, precision=6))
    assert np.array_equal(np.load(out["file"]), ours)
    # the two shipped files differ only in C_01 (549.96 vs 593.46); ours must
    # match one of them there and both elsewhere
    close = lambda x, y: np.abs(x - y) <= 1e-3 * np.abs(y)  # noqa: E731
    assert np.all(close(ours, a) | close(ours, b)), (ours, a, b)


def test_fluid_2d_ranges_match_reference(tmp_path):
    """The shipped fluid_2d file holds max|J - 1| for J (the offset of J's
    fixed-point type), not max|J| as the reference's current get_limits
    returns; the test compares J that way and the rest directly."""
    exp = D.Fluid2D()
    out = D.detect_range(exp, exp.config(), str(tmp_path))
    ours = np.array(out["ranges"])
    ref = np.array(GOLD["ranges"]["fluid_2d/fluid_2d_t16385_dt0.0002_p10000_g128.npy"])
    j_dev = max(abs(out["max"][-1] - 1.0), abs(out["min"][-1] - 1.0))
    cmp = np.concatenate([ours[:-1], [j_dev]])
    print("fluid_2d ranges ours/reference:", np.array2string(cmp / ref, precision=4))
    assert ours[-1] == pytest.approx(max(abs(out["max"][-1]), abs(out["min"][-1])))
    assert cmp == pytest.approx(ref, rel=0.05)


def test_elastic_2d_error_bound_runs_meet_the_drivers_criterion(tmp_path):
    """The reference driver reports the fraction of its N runs with
    |loss - f64 loss| < 3 eps f64 loss (run_mpm_elastic_2d.py:190-207).  The
    scene is chaotic over 8192 substeps (and P2G sums in no fixed order), so
    single runs can miss; 20 runs measured on a B200 succeeded 18 times.
    Here 10 runs must succeed at least 6 times (a 90 % rate fails that with
    probability 0.2 %)."""
    exp = D.Elastic2D()
    cfg = exp.config()
    gfn, rfn = D._paths(exp, str(tmp_path))
    os.makedirs(os.path.dirname(gfn))
    os.makedirs(os.path.dirname(rfn))
    np.save(gfn, np.array(GOLD["grads"]["elastic_2d/elastic_2d.npy"]))
    np.save(rfn, np.array(GOLD["ranges"]["elastic_2d/elastic_2d.npy"]))
    eps = 0.1
    sol = D.solve(exp, cfg, str(tmp_path), D.EB, eps)
    loss = D.run(exp, cfg, 10)
    ok = np.abs(loss - exp.f64_data) < 3 * eps * exp.f64_data
    print("elastic_2d EB eps %g bits %s losses %s (f64 %.3f) succeed %.2f" % (eps, sol["bits"], loss, exp.f64_data,
                                                                              ok.mean()))
    assert sol["compression_rate"] < 0.5
    assert ok.mean() >= 0.6
    assert len(set(loss.tolist())) > 1  # dithering seeds differ between runs


def test_pipeline_end_to_end_reproduces_reference_scheme(tmp_path):
    """-r, -a and -f chained through the CLI on the full experiment: the
    solved compression-rate scheme must be the one the reference's own
    gradients and ranges give, to within one bit per scalar."""
    root = str(tmp_path)
    common = ["elastic_2d", "--root", root, "--json"]
    r = D.main(common + ["-r"])
    a = D.main(common + ["-a"])
    f = D.main(common + ["-f", "-m", "0", "-e", "0.5", "-N", "2"])
    assert os.path.exists(r["file"]) and os.path.exists(a["file"])
    assert a["loss"] == pytest.approx(D.Elastic2D.f64_data, abs=5e-3)
    case = [c for c in GOLD["solver"] if c["key"] == "elastic_2d/elastic_2d.npy" and c["mode"] == "CR"
            and c["eps"] == 0.5][0]
    want = np.array(case["bits"]) + 1
    print("solved bits", f["bits"], "from reference data", want.tolist(), "losses", f["losses"])
    assert np.max(np.abs(np.array(f["bits"]) - want)) <= 1
    assert f["compression_rate"] == pytest.approx(0.5, abs=0.05)
    assert np.all(np.isfinite(f["losses"]))



def test_detect_bound_kernel_folds_only_the_states_it_is_called_on():
    """detect_bound_kernel (update_limits_*, mpm_solver.py:943-979) folds the
    state at the call and nothing in between: called twice, three substeps
    apart, the limits are the max |q| of exactly those two states."""
    from autoquantizer_b200 import scenes
    from autoquantizer_b200.mpm_solver import MPMSolver

    cfg, vals = scenes.falling_block_3d(n=8000, n_grid=32)
    vals[:, 3] = 2.0
    s = MPMSolver(cfg)
    s.set_particles(vals)
    s.substeps(2)
    s.detect_bound_kernel(0)
    a = s.state_values()
    s.substeps(3)
    s.detect_bound_kernel(1)
    b = s.state_values()
    s.substeps(4)  # not folded
    s.detect_bound()
    d = cfg.dim
    expect = np.maximum(np.abs(a), np.abs(b)).max(0)[d:]
    lim = s.get_limits()
    assert np.array_equal(lim[:d], [2.0] * d)
    np.testing.assert_allclose(lim[d:], expect, rtol=1e-12, atol=0)
    c = s.state_values()
    assert np.any(np.abs(c).max(0)[d:] > expect)  # the later state would have widened them


def test_fluid_3d_ranges_match_reference_statistically(tmp_path):
    """The -r pass of the 3D fluid experiment (run_mpm_fluid_3d.py:101-146:
    1e6 particles in two slabs, 64 grid over 2 x 1 x 2, 8192 substeps of
    4e-4, the propeller collider on the autodiff schedule), against the
    reference's shipped ranges/fluid_3d/fluid_3d.npy.  add_cube seeds with
    random positions (ti.random in the reference), so the extremes agree as
    statistics: positions exactly 2, max |J| within 0.1 (J near 1), and v_x,
    v_z and every C range within a factor of 2.  Max |v_y| is the exception:
    the shipped value, 29.8, is ten times what the scene allows (slabs at most
    0.45 high fall at most 3 m/s; the propeller moves the fluid sideways, and
    the horizontal maxima, 3.4 and 3.3, match the propeller's tip speed), so
    it records a few extreme particles of that run; here max |v_y| must lie
    between 1 m/s and the shipped value."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "propeller_higher.npz"))
    np.savez(tmp_path / "propeller_higher.npz", sdf=z["sdf"])
    np.savez(tmp_path / "propeller_higher_normal.npz", sdf=z["normal"])
    exp = D.Propeller3D()
    exp.inputs = str(tmp_path)
    out = D.detect_range(exp, exp.config("ranges"), str(tmp_path))
    ours = np.array(out["ranges"])
    ref = np.array(GOLD["ranges"]["fluid_3d/fluid_3d.npy"])
    print("fluid_3d ranges ours/reference:", np.array2string(ours / ref, precision=3))
    assert ours.shape == ref.shape == (16,)
    assert np.array_equal(ours[:3], [2.0, 2.0, 2.0])
    ratio = ours[3:15] / ref[3:15]
    keep = np.ones(12, dtype=bool)
    keep[1] = False  # v_y, below
    assert np.all((ratio[keep] > 0.5) & (ratio[keep] < 2.0)), ratio
    assert 1.0 < ours[4] < ref[4], (ours[4], ref[4])
    assert abs(ours[15] - ref[15]) < 0.1, (ours[15], ref[15])


def _scaling(tmp_path, **kw):
    data = {"id": 0, "n_particles": 20000, "dt": 2e-4, "steps": 1, "grids": 64, "lb": [15, 3, 3], "ub": [48, 60, 60]}
    data.update(kw)
    fn = tmp_path / ("config%d.json" % data["id"])
    fn.write_text(json.dumps(data))
    exp = D.Fluid3DScaling()
    exp.config_file = str(fn)
    return exp


def test_fluid_3d_scaling_pipeline(tmp_path):
    """The scaling experiment's -r and -f passes on a small configuration of
    the reference's format (20,000 particles, 64 grid, 1025 substeps):
    ranges of the fluid block, then the SLSQP scheme from the shipped
    sensitivities and ranges and one quantized forward run with a clean
    status."""
    exp = _scaling(tmp_path)
    out = D.detect_range(exp, exp.config("ranges"), str(tmp_path))
    r = np.array(out["ranges"])
    assert r.shape == (16,) and np.all(np.isfinite(r))
    assert np.all(r[:3] == 2.0)
    assert 0.0 < r[4] < 10.0  # max |v_y|: a 0.2-high block falls well below 10 m/s
    assert 0.9 < r[15] < 1.5  # max |J| of a weakly compressible fluid
    os.makedirs(tmp_path / "grads" / "fluid_3d_scaling", exist_ok=True)
    np.save(tmp_path / "grads" / "fluid_3d_scaling" / exp.file_name,
            np.array(GOLD["grads"]["fluid_3d_scaling/" + exp.file_name]))
    np.save(tmp_path / "ranges" / "fluid_3d_scaling" / exp.solve_range_file,
            np.array(GOLD["ranges"]["fluid_3d_scaling/" + exp.solve_range_file]))
    cfg = exp.config()
    sol = D.solve(exp, cfg, str(tmp_path), D.CR, 0.5)
    assert 0.45 < sol["compression_rate"] < 0.55
    loss = D.run(exp, cfg, 1)
    assert np.all(np.isfinite(loss)) and loss[0] > 0


def test_fluid_3d_scaling_jets_fill_the_box(tmp_path):
    """Configurations 5 and 6 start empty and emit two jets of 1000
    particles every 30 substeps while they fit (emit_water only adds while
    current_idx + num < n_particles)."""
    from autoquantizer_b200.mpm_solver import MPMSolver

    exp = _scaling(tmp_path, id=6, task=1)
    cfg = exp.config()
    cfg.n_timesteps = 301
    mpm = MPMSolver(cfg)
    exp.init(mpm)
    assert mpm.current_idx == 0
    exp.run_frames(mpm)
    # 9 pairs of jets, then at substep 270 one more jet: a second would reach n_particles
    assert mpm.current_idx == 19000
    assert mpm.status()[0] == 0
    x = mpm.state_values()[: mpm.current_idx, :3]
    assert np.all((x > 0) & (x < 1))


def test_dithering_experiment_runs_all_three_modes(tmp_path):
    """run_mpm_dithering_exp.py's three runs on its fixed scheme (the
    elastic_2d ranges from the shipped file), over 512 substeps: the
    unquantized f64 run, quantized with and without dithering.  With
    dithering the loss stays within 1 % of the unquantized one (measured:
    2.3e-4); without it, rounding every velocity update the same way
    (gravity adds about one velocity step per substep) biases the motion,
    and the loss is off by far more (measured: 162 %)."""
    os.makedirs(tmp_path / "ranges" / "elastic_2d")
    np.save(tmp_path / "ranges" / "elastic_2d" / "elastic_2d.npy",
            np.array(GOLD["ranges"]["elastic_2d/elastic_2d.npy"]))
    exp = D.Dithering2D()
    cfg = exp.config()
    cfg.n_timesteps = 513
    out = D.dithering_experiment(exp, cfg, str(tmp_path))
    print("dithering experiment:", out["loss_f64"], out["rel_err_dithering"], out["rel_err_no_dithering"])
    assert out["loss_f64"] > 0
    assert out["rel_err_dithering"] < 1e-2
    assert out["rel_err_no_dithering"] > 10 * out["rel_err_dithering"]
