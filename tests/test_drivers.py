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
    assert GOLD["driver_solver"]
    for c in GOLD["driver_solver"]:
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
