"""End-to-end pins against numbers the reference itself produced on its 2D
elastic experiment (mpm_exps/run_mpm_elastic_2d.py:54-122; values in
tests/golden/reference_data.json):

  * the f64 reference loss 6893.409 (sum |v|^2 after 8192 substeps of 80,000
    particles in eight lattice cubes, 128^2 grid, dt 2e-4), from its
    unquantized Taichi run;
  * the per-scalar autodiff sensitivities of that loss that the reference
    shipped (mpm_exps/grads/elastic_2d/elastic_2d.npy).

The reference prints the loss to three decimals; it is pinned to that
(5e-3 absolute, i.e. 7e-7 relative).  The sensitivities span 1e4..1e18 and
come out of 8192 substeps whose f64 sums are accumulated in a different
order than Taichi's, so each is pinned to 1% relative.
"""
import json
import os

import numpy as np
import pytest

from autoquantizer_b200.mpm_config import MPMConfig
from autoquantizer_b200.mpm_solver import MPMSolver

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_data.json")))
E2 = GOLD["elastic_2d"]


def _elastic_2d():
    c = MPMConfig()
    c.dim = 2
    c.E, c.nu = E2["E"], E2["nu"]
    c.la = 1e3
    c.bound = E2["bound"]
    c.use_friction = False
    c.use_fluid = False
    c.n_particles = E2["n_particles"]
    c.dt = E2["dt"]
    c.n_grid = E2["n_grid"]
    c.n_timesteps = E2["n_timesteps"]
    c.size = E2["size"]
    c.p_rho = E2["p_rho"]
    c.p_vol = (1.0 / c.n_grid * 0.5) ** 2
    c.g = E2["g"]
    c.precision = "f64"
    c.use_quantaichi = False
    s = MPMSolver(c)
    s.initialize()
    for low in E2["cubes_low"]:
        s.add_cube(low, E2["cube_size"], E2["per_cube"])
    return s


def test_elastic_2d_f64_loss_matches_reference():
    s = _elastic_2d()
    assert s.current_idx == 80000
    loss = s.run_forward_only()
    print("elastic_2d f64 loss %.4f (reference %.3f)" % (loss, E2["f64_loss"]))
    assert s.status()[0] == 0
    assert loss == pytest.approx(E2["f64_loss"], abs=5e-3)


def test_elastic_2d_sensitivities_match_reference_autodiff():
    s = _elastic_2d()
    loss = s.run_forward_with_ad_nlogn(every=64)
    assert loss == pytest.approx(E2["f64_loss"], abs=5e-3)
    ours = s.get_gradients()
    ref = np.array(GOLD["grads"]["elastic_2d/elastic_2d.npy"])
    ratio = ours / ref
    print("sensitivity ratio ours/reference per scalar:", np.array2string(ratio, precision=3))
    assert ours == pytest.approx(ref, rel=1e-2), ratio
