"""Host side of the experiment pipeline (autoquantizer_b200.drivers): the
solve() recipes against the reference's own solver outputs on its shipped
sensitivities and ranges (tests/golden/reference_data.json), the scene
set-up against the reference driver's constants, and the file plumbing."""
import json
import os

import numpy as np
import pytest

from autoquantizer_b200 import drivers as D

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_data.json")))
E2 = "elastic_2d/elastic_2d.npy"
F2 = "fluid_2d/fluid_2d_t16385_dt0.0002_p10000_g128.npy"
E3 = "elastic_3d/elastic_3d.npy"


def _cases(key, mode):
    return [c for c in GOLD["solver"] if c["key"] == key and c["mode"] == mode]


@pytest.mark.parametrize("mode", ["EB", "CR"])
def test_elastic_2d_solve_matches_reference_solver(mode):
    exp = D.Elastic2D()
    g, r = np.array(GOLD["grads"][E2]), np.array(GOLD["ranges"][E2])
    for c in _cases(E2, mode):
        bits, ranges = exp.scheme(g, r, D.EB if mode == "EB" else D.CR, c["eps"])
        # run_mpm_elastic_2d.py:232-250: solver bits + 1 sign bit
        assert bits.tolist() == [b + 1 for b in c["bits"]], c["eps"]
        assert ranges[:2].tolist() == [1.0, 1.0]
        assert np.allclose(ranges[2:], 2 * r[2:], rtol=0, atol=0)
        assert np.array_equal(g * ranges ** 2, np.array(c["grads_weighted"]))


def test_fluid_2d_solve_matches_the_drivers_own_solver():
    exp = D.Fluid2D()
    g, r = np.array(GOLD["grads"][F2]), np.array(GOLD["ranges"][F2])
    cases = [c for c in GOLD["driver_solver"] if c["driver"] == "fluid_2d"]
    assert cases
    for c in cases:
        bits, ranges = exp.scheme(g, r, D.CR, c["eps"])
        assert bits.tolist() == c["bits"], c["eps"]
        assert ranges.tolist() == c["ranges"]
        _, fun = D.lagrangian_cr_fluid_2d(g / g.min() * ranges ** 2, r=c["eps"])
        assert fun == pytest.approx(c["fun"], rel=1e-12)


def test_fluid_2d_has_no_error_bound_mode():
    with pytest.raises(ValueError):
        D.Fluid2D().scheme(np.ones(9), np.ones(9), D.EB, 0.1)


def test_3d_recipe_matches_reference_solver():
    exp = D.FallingBlock3D()
    g, r = np.array(GOLD["grads"][E3]), np.array(GOLD["ranges"][E3])
    for c in _cases(E3, "CR"):
        bits, ranges = exp.scheme(g, r, D.CR, c["eps"])
        assert bits.tolist() == [b + 1 for b in c["bits"]]
        assert np.array_equal(g * ranges ** 2, np.array(c["grads_weighted"]))


class _FakeSolver:
    def __init__(self, cfg):
        self.param = cfg
        self.cubes = []

    def initialize(self):
        self.cubes = []

    def add_cube(self, low, size, n):
        self.cubes.append((list(low), list(size), n))


def test_elastic_2d_scene_matches_reference_driver():
    exp = D.Elastic2D()
    cfg = exp.config()
    ref = GOLD["elastic_2d"]
    assert (cfg.n_particles, cfg.dt, cfg.n_grid, cfg.n_timesteps, cfg.E, cfg.size) == (
        ref["n_particles"], ref["dt"], ref["n_grid"], ref["n_timesteps"], ref["E"], ref["size"])
    assert cfg.precision == "f64" and not cfg.use_fluid and not cfg.use_friction
    m = _FakeSolver(cfg)
    exp.init(m)
    assert [c[0] for c in m.cubes] == ref["cubes_low"]
    assert all(c[1] == ref["cube_size"] and c[2] == ref["per_cube"] for c in m.cubes)


def test_fluid_2d_scene_matches_reference_driver():
    exp = D.Fluid2D()
    cfg = exp.config()
    # run_mpm_fluid_2d.py:185-214 and the shipped file name built from them
    assert "fluid_2d_t%d_dt%s_p%d_g%d.npy" % (cfg.n_timesteps, cfg.dt, cfg.n_particles, cfg.n_grid) == exp.file_name
    assert cfg.use_fluid and cfg.la == 5e2 and cfg.precision == "f64"
    m = _FakeSolver(cfg)
    exp.init(m)
    assert m.cubes == [([3 / 128, 3 / 128], [1.5 / 4, 1.5 / 4], 10000)]


def test_solve_reads_saved_files(tmp_path):
    exp = D.Elastic2D()
    cfg = exp.config()
    gfn, rfn = D._paths(exp, str(tmp_path))
    os.makedirs(os.path.dirname(gfn))
    os.makedirs(os.path.dirname(rfn))
    np.save(gfn, np.array(GOLD["grads"][E2]))
    np.save(rfn, np.array(GOLD["ranges"][E2]))
    out = D.solve(exp, cfg, str(tmp_path), D.EB, 0.1)
    want = [b + 1 for b in _cases(E2, "EB")[0]["bits"]]
    assert out["bits"] == want
    assert cfg.quant_bits.tolist() == want
    assert cfg.quant_ranges[0] == 1.0
    assert out["compression_rate"] == pytest.approx(sum(want) / (32 * 12))


def test_cli_needs_one_action():
    with pytest.raises(SystemExit):
        D.main(["elastic_2d"])
    with pytest.raises(SystemExit):
        D.main(["fluid_2d", "-f", "-m", "1", "--root", "/nonexistent"])


def test_solve_rejects_unusable_widths(tmp_path):
    exp = D.Elastic2D()
    cfg = exp.config()
    gfn, rfn = D._paths(exp, str(tmp_path))
    os.makedirs(os.path.dirname(gfn))
    os.makedirs(os.path.dirname(rfn))
    np.save(gfn, np.array(GOLD["grads"]["elastic_2d/elastic_2d.npy"]))
    np.save(rfn, np.array(GOLD["ranges"]["elastic_2d/elastic_2d.npy"]))
    with pytest.raises(ValueError):
        D.solve(exp, cfg, str(tmp_path), D.CR, 0.05)


def test_adjoint_report_groups_partition_the_3d_record():
    from autoquantizer_b200 import adjoint_report as AR
    from autoquantizer_b200.adjoint import group_fields_3d

    g = AR.group_slots()
    assert sorted(sum(g, [])) == list(range(24)) and len(g) == len(AR.GROUP_NAMES) == 12
    v = np.arange(24, dtype=np.float64)
    assert np.array_equal([v[s].sum() for s in g], group_fields_3d(v))


@pytest.mark.parametrize("driver,cls", [("elastic_3d", D.Letters3D), ("fluid_3d", D.Propeller3D)])
def test_3d_drivers_solve_matches_reference_solver(driver, cls):
    """The 3D drivers' solve() recipes (run_mpm_elastic_3d.py:323-333,
    run_mpm_fluid_3d.py:149-161) against the reference's LagrangianCR on
    its shipped gradients and ranges."""
    exp = cls()
    key = "%s/%s.npy" % (driver, driver)
    g, r = np.array(GOLD["grads"][key]), np.array(GOLD["ranges"][key])
    cases = [c for c in GOLD["driver_solver"] if c["driver"] == driver]
    assert len(cases) == 3
    for c in cases:
        bits, ranges = exp.scheme(g, r, D.CR, c["eps"])
        assert bits.tolist() == [b + 1 for b in c["bits"]], c["eps"]
        if driver == "elastic_3d":
            assert ranges.tolist() == c["ranges"]
        else:  # solved with positions at 2, run with positions at 4 and y at 1
            want = np.array(c["ranges"])
            want[:3] = [4.0, 1.0, 4.0]
            assert ranges.tolist() == want.tolist()
    with pytest.raises(ValueError):
        exp.scheme(g, r, D.EB, 0.1)


def test_fluid_3d_scheme_reproduces_the_drivers_recorded_bits():
    """run_mpm_fluid_3d.py:201 records the bits its solve() gave at a 0.5
    compression target: [21, 22, 21, 15, 18, 15, 12, 16, 13, 14, 13, 14, 14,
    15, 13, 17]; the scheme at eps 0.512 (the value solve() uses) gives
    them."""
    key = "fluid_3d/fluid_3d.npy"
    bits, _ = D.Propeller3D().scheme(np.array(GOLD["grads"][key]), np.array(GOLD["ranges"][key]), D.CR, 0.512)
    assert bits.tolist() == [21, 22, 21, 15, 18, 15, 12, 16, 13, 14, 13, 14, 14, 15, 13, 17]


class _Recorder(_FakeSolver):
    PER_MESH = 100  # particles a stand-in mesh seeds

    def __init__(self, cfg):
        super().__init__(cfg)
        self.calls = []
        self.current_idx = 0
        self.n_particles = cfg.n_particles

    def add_mesh(self, tri, **kw):
        self.calls.append(("add_mesh", tri.shape, kw, self.current_idx))
        self.current_idx += self.PER_MESH

    def cnt_mesh_particles_num(self, tri, **kw):
        return self.PER_MESH

    def init_sdf_value(self, sdf, normal, **kw):
        self.calls.append(("init_sdf_value", sdf.shape, normal.shape, kw))


def test_3d_experiment_setups(tmp_path):
    """Scene set-up of the 3D drivers with stand-in input files: the meshes
    and collider volumes are read from --inputs, the letters are emitted at
    the reference's translations, the propeller scene gets the collider on
    the autodiff schedule and the reference's slabs."""
    from autoquantizer_b200 import mesh_io

    inp = tmp_path / "inputs"
    inp.mkdir()
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], dtype=np.float32)
    with open(inp / "auto_quant.ply", "wb") as f:
        f.write(b"ply\nformat binary_little_endian 1.0\nelement vertex 3\nproperty float x\nproperty float y\n"
                b"property float z\nelement face 1\nproperty list uchar uint vertex_indices\nend_header\n")
        f.write(v.tobytes() + np.uint8(3).tobytes() + np.array([0, 1, 2], "<u4").tobytes())
    for stem in ("propeller_higher", "propeller_2x2_larger"):
        np.savez(inp / (stem + ".npz"), sdf=np.zeros((4, 5, 6), np.float32))
        np.savez(inp / (stem + "_normal.npz"), sdf=np.zeros((4, 5, 6, 3), np.float32))
    assert mesh_io.load_mesh(str(inp / "auto_quant.ply")).shape == (1, 9)

    le = D.Letters3D()
    le.inputs = str(inp)
    cfg = le.config("forward")
    assert (cfg.n_particles, cfg.n_grid, cfg.dt, cfg.E, cfg.la, cfg.nu) == (int(3e8), 256, 7.5e-5, 5e5, 5e4, 0.2)
    m = _Recorder(cfg)
    le.init(m)
    assert m.calls == []  # the letters come with the frames
    for frame in range(9):
        le.emit(frame, m)
    # frames 0, 4, 8 (emit_step 4): two meshes each, z 0.1 + 0.006 k, each
    # batch starting at k * (2 x the particles of one mesh)
    zs = [0.1, 0.1 + 0.006, 0.1 + 0.012]
    assert [c[2]["translation"] for c in m.calls] == [(x, 1.6, z) for z in zs for x in (0.90, 2.2)]
    assert [c[3] for c in m.calls] == [0, 100, 200, 300, 400, 500]
    assert all(c[2]["sample_density"] == 8 and c[2]["velocity"] == (0.0, -4.0, 0.0) for c in m.calls)
    m.n_particles = 700  # the next batch would not fit: no more letters
    le.emit(12, m)
    assert len(m.calls) == 6

    pr = D.Propeller3D()
    pr.inputs = str(inp)
    cfg = pr.config("ad")
    assert (cfg.n_particles, cfg.n_grid, cfg.dt, cfg.la) == (100 ** 3, 64, 4e-4, 5e5)
    assert cfg.ub == [125, 61, 125] and cfg.grid_res == [132, 68, 132]
    m = _Recorder(cfg)
    pr.init(m)
    assert m.calls[0][0] == "init_sdf_value" and m.calls[0][3]["height_rate"] == 0.15
    dx = 1 / 64
    assert m.calls[0][1] == (4, 5, 6)
    assert [c[0] for c in m.cubes] == [[3 * dx, 3 * dx, 3 * dx], [3 * dx, 3 * dx + 0.2, 3 * dx]]
    assert all(c[2] == 100 ** 3 // 2 for c in m.cubes)
    cfg = pr.config("forward")
    assert (cfg.n_particles, cfg.n_grid, cfg.ub) == (int(4e8), 256, [1021, 253, 1021])
    m = _Recorder(cfg)
    pr.init(m)
    assert m.calls[0][3]["height_rate"] == 0.1 and len(m.cubes) == 1 and m.cubes[0][2] == int(4e8)


def test_mpm_config_defaults_match_the_reference():
    """Every field of the reference's MPMConfig (mpm_exps/mpm_config.py)
    exists here with the same default, so drivers run unchanged."""
    from autoquantizer_b200.mpm_config import MPMConfig

    ours = vars(MPMConfig())
    for k, v in GOLD["mpm_config_defaults"].items():
        assert k in ours, k
        assert ours[k] == pytest.approx(v) if isinstance(v, float) else ours[k] == v, k


def test_checkpoint_file_round_trip(tmp_path):
    """save_checkpoint / load_checkpoint plumbing on CPU (the device calls
    replaced by recorders): words, particle count, substep count and the
    layout check."""
    from autoquantizer_b200 import scenes
    from autoquantizer_b200.mpm_solver import MPMSolver

    cfg, vals = scenes.falling_block_3d(n=500, n_grid=16)
    a = MPMSolver(cfg)
    a.set_particles(vals[:300])
    W = a.layout().n_words
    words = np.arange(300 * W, dtype=np.uint64).reshape(300, W) * np.uint64(0x9E3779B97F4A7C15)
    a.words = lambda: words
    a.step_count = lambda: 77
    fn = a.save_checkpoint(str(tmp_path / "ck.npz"))

    b = MPMSolver(cfg)
    got = {}
    b.set_words = lambda w: got.setdefault("words", np.array(w))
    b.set_step_count = lambda st: got.setdefault("step", st)
    b.load_checkpoint(fn)
    assert b.current_idx == 300 and got["step"] == 77 and np.array_equal(got["words"], words)

    other, _ = scenes.dam_break_2d(n=100, n_grid=16)
    with pytest.raises(ValueError):
        MPMSolver(other).load_checkpoint(fn)


def test_driver_loop_helpers_on_the_host():
    """The small methods the reference drivers call in their own loops."""
    from autoquantizer_b200 import scenes
    from autoquantizer_b200.mpm_solver import MPMSolver

    assert [MPMSolver.cnt_ending_zero(s) for s in range(8)] == [0, 1, 0, 2, 0, 1, 0, 3]
    cfg, vals = scenes.falling_block_3d(n=100, n_grid=16)
    s = MPMSolver(cfg)
    s.step_collider()  # nothing to do: the simulator advances the collider itself
    s._grads = [np.arange(3.0), np.arange(3.0, 6.0)]
    assert s.dump_grad(0).tolist() == [0, 1, 2, 3, 4, 5]
    import torch

    s._col = {"sdf": torch.zeros((2, 2, 2)), "normal": torch.zeros((2, 2, 2, 3)), "offset": [0, 0, 0],
              "theta": 0.0, "height": 0.0, "omega": 5.0, "rate": 0.1}
    s.step_collider_difftaichi(10)
    assert s.collider_state() == (pytest.approx(5.0 * cfg.dt * 10), pytest.approx(0.15 * cfg.dt * 10))


SCIPY_GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "scipy_solver.json")))
FS = "fluid_3d_scaling/fluid_3d_t16385_dt0.0002_p200000_g64.npy"
FS_R = "fluid_3d_scaling/fluid_3d_t65537_dt5e-05_p5000000_g256.npy"


def _scaling_config(tmp_path, **kw):
    data = {"id": 0, "n_particles": 200000, "dt": 2e-4, "steps": 16, "grids": 64, "lb": [15, 3, 3], "ub": [48, 60, 60]}
    data.update(kw)
    fn = tmp_path / "config.json"
    fn.write_text(json.dumps(data))
    exp = D.Fluid3DScaling()
    exp.config_file = str(fn)
    return exp, exp.config()


def test_fluid_3d_scaling_reads_the_reference_config_format(tmp_path):
    """parse_json (run_mpm_fluid_3d_scaling.py:60-73) and the driver's fixed
    settings (:362-401)."""
    exp, c = _scaling_config(tmp_path, id=4, task=1, steps=32, grids=128, dt=1e-4, lb=[30, 3, 3], ub=[97, 124, 124])
    assert (c.n_timesteps, c.steps, c.n_grid, c.dt) == (32 * 1024 + 1, 32 // 16 * 128, 128, 1e-4)
    assert c.lb == [30, 3, 3] and c.ub == [97, 124, 124]
    assert (c.la, c.E, c.p_rho, c.size) == (2e6, 5e4, 1000.0, 1.0)
    assert c.p_vol == pytest.approx((0.5 / 128) ** 3)
    assert exp.task == 1 and exp.cid == 4
    _, c0 = _scaling_config(tmp_path)
    assert c0.la == 5e5 and c0.task == D.Fluid3DScaling.SCALING


def test_fluid_3d_scaling_solve_matches_the_reference_slsqp_solver(tmp_path):
    """solve() for configurations 0-5: the SLSQP memory-budget solver on the
    shipped gradients (divided by their minimum) and ranges (positions 1,
    the rest doubled); its widths are the reference solver's."""
    exp, _ = _scaling_config(tmp_path)
    g, r = np.array(GOLD["grads"][FS]), np.array(GOLD["ranges"][FS_R])
    cases = [c for c in SCIPY_GOLD["cases"] if c["key"] == FS and c["form"] == "mem"]
    assert cases
    for case in cases:
        bits, ranges = exp.scheme(g, r, D.CR, case["eps"])
        assert bits.tolist() == case["bits"]
        assert ranges.tolist() == case["ranges"]


def test_fluid_3d_scaling_solve_uses_the_closed_form_for_configs_6_and_7(tmp_path):
    exp, _ = _scaling_config(tmp_path, id=7, task=1)
    g, r = np.array(GOLD["grads"][FS]), np.array(GOLD["ranges"][FS_R])
    bits, ranges = exp.scheme(g, r, D.CR, 0.3)
    ref, _ = D.LagrangianCR(g * ranges ** 2, r=0.3)
    assert bits.tolist() == (ref + 1).tolist()
    with pytest.raises(ValueError):
        exp.scheme(g, r, D.EB, 0.3)


def test_fluid_3d_scaling_solve_reads_the_fixed_range_file(tmp_path):
    """The scaling driver's solve() reads the ranges of the 5M-particle run,
    not those of the run the gradients come from."""
    exp, c = _scaling_config(tmp_path)
    os.makedirs(tmp_path / "grads" / "fluid_3d_scaling")
    os.makedirs(tmp_path / "ranges" / "fluid_3d_scaling")
    np.save(tmp_path / "grads" / FS, np.array(GOLD["grads"][FS]))
    np.save(tmp_path / "ranges" / FS_R, np.array(GOLD["ranges"][FS_R]))
    out = D.solve(exp, c, str(tmp_path), D.CR, 0.5)
    case = [k for k in SCIPY_GOLD["cases"] if k["key"] == FS and k["form"] == "mem" and k["eps"] == 0.5][0]
    assert out["bits"] == case["bits"]


@pytest.mark.parametrize("task,cid", [(0, 0), (1, 0), (1, 1), (1, 2), (1, 3), (1, 4), (1, 5), (1, 6), (1, 7)])
def test_fluid_3d_scaling_initial_conditions(tmp_path, task, cid):
    """init() of run_mpm_fluid_3d_scaling.py:222-275 for the scaling task and
    every initial-condition configuration: the blocks start at the walls lb
    (configurations 5 and 6 start empty), inside the domain, with the
    configuration's particle count (split in two for configuration 3)."""
    from autoquantizer_b200.mpm_solver import MPMSolver

    exp, c = _scaling_config(tmp_path, id=cid, task=task, n_particles=4000)
    mpm = MPMSolver(c)
    exp.init(mpm)
    if cid in (5, 6) and task == 1:
        assert mpm.current_idx == 0
        return
    assert mpm.current_idx == 4000
    x = mpm._staging()[:4000, :3]
    dx = 1.0 / c.n_grid
    assert np.all(x >= (np.array(c.lb) + 0.5) * dx - 1e-12)
    assert np.all(x < 1.0)
    if cid == 1 and task == 1:  # the block starts at the middle of the walls in x
        assert x[:, 0].min() >= (c.lb[0] + c.ub[0]) * 0.5 * dx - 1e-12
    if cid == 3 and task == 1:  # two blocks, one against each z wall
        assert (x[:, 2] < 0.5).sum() == 2000 and (x[:, 2] > 0.5).sum() == 2000


def test_optimality_check_perturbations():
    """run_mpm_optimality_check.py:196-232: task 0 takes S bits off every
    field, task 1 off half of them (chosen at random), task 2 moves S1 bits
    from x to v and S2 from C to F (totals kept)."""
    bits = np.array([22, 22, 16, 16, 9, 11, 11, 9, 18, 17, 17, 18])
    b0 = D.perturb_bits(bits, 2, 0, 2)
    assert (bits - b0).tolist() == [2] * 12
    b1 = D.perturb_bits(bits, 2, 1, 3, rng=np.random.default_rng(5))
    d = bits - b1
    assert sorted(d.tolist()) == [0] * 6 + [3] * 6
    assert not np.array_equal(d, bits - D.perturb_bits(bits, 2, 1, 3, rng=np.random.default_rng(6)))
    b2 = D.perturb_bits(bits, 2, 2, 2, 1)
    assert (b2 - bits).tolist() == [-2, -2, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1]
    assert b2.sum() == bits.sum()
    with pytest.raises(ValueError):
        D.perturb_bits(bits, 2, 3, 1)


def test_dithering_experiment_scene():
    """run_mpm_dithering_exp.py's scene: four 0.15-wide lattice cubes at
    (0.125 + 0.2 i, 0.75) of n/4 particles each, on its fixed scheme."""
    from autoquantizer_b200.mpm_solver import MPMSolver

    exp = D.Dithering2D()
    c = exp.config()
    assert c.quant_bits.tolist() == D.Dithering2D.BITS and c.dt == 2e-4 and c.precision == "f64"
    c.n_particles = 4 * 400
    mpm = MPMSolver(c)
    exp.init(mpm)
    assert mpm.current_idx == 1600
    x = mpm._staging()[:1600, :2]
    for i in range(4):
        blk = x[400 * i:400 * (i + 1)]
        assert blk[:, 0].min() >= 0.125 + 0.2 * i - 1e-12 and blk[:, 0].max() < 0.125 + 0.2 * i + 0.15
        assert blk[:, 1].min() >= 0.75 - 1e-12 and blk[:, 1].max() < 0.9
