"""Resuming from save_checkpoint / load_checkpoint on the GPU.

What is guaranteed: the resumed run continues with the same dithering draws
(the substep count that keys them is restored) and the same records, and it
agrees with the uninterrupted run to the substep parity tolerance.  What is
not: bit identity.  The order of the records inside a cell after re-binning
comes from atomic counters, so the grid sums of two runs - two uninterrupted
ones included - are added in different orders.
"""
import numpy as np
import pytest

from autoquantizer_b200 import scenes
from autoquantizer_b200.mpm_solver import MPMSolver
from helpers import quant_steps

pytestmark = pytest.mark.gpu


def _close(a, b, s, rel=2e-5, steps=2.0):
    q = quant_steps(s)
    for k in range(a.shape[1]):
        scale = max(1.0, float(np.max(np.abs(b[:, k]))))
        tol = rel * scale + (steps * q[k] if q[k] > 0 else 2.0 ** -10 * scale if np.isnan(q[k]) else 0.0)
        err = float(np.max(np.abs(a[:, k] - b[:, k])))
        assert err <= tol, (k, err, tol)


def test_resume_matches_uninterrupted_run(tmp_path):
    cfg, vals = scenes.dam_break_2d(n=8192, n_grid=128)
    k = 6
    straight = MPMSolver(cfg)
    straight.set_particles(vals)
    straight.substeps(2 * k)

    first = MPMSolver(cfg)
    first.set_particles(vals)
    first.substeps(k)
    fn = first.save_checkpoint(str(tmp_path / "ck.npz"))
    mid = first.words()
    del first

    resumed = MPMSolver(cfg)
    resumed.set_particles(vals)  # overwritten by the checkpoint
    resumed.load_checkpoint(fn)
    assert resumed.step_count() == k
    assert np.array_equal(resumed.words(), mid)
    resumed.substeps(k)
    assert resumed.step_count() == 2 * k
    assert resumed.status()[0] == 0
    _close(resumed.state_values(), straight.state_values(), straight)
