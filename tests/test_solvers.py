"""The analytical bit-width solvers against the reference's own solver
outputs on its shipped sensitivities (tests/golden/reference_data.json,
generated by tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

from autoquantizer_b200 import solvers

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_data.json")))


@pytest.mark.parametrize("case", GOLD["solver"], ids=lambda c: "%s-%s-%g" % (c["key"].split("/")[0], c["mode"], c["eps"]))
def test_solver_matches_reference(case):
    g = np.array(case["grads_weighted"])
    if case["mode"] == "EB":
        bits, rel = solvers.LagrangianEB(g, ref=case["ref"], tol_rel=case["eps"])
        assert bits.tolist() == case["bits"]
        assert rel == pytest.approx(case["rel"], rel=1e-12)
    else:
        bits, fun = solvers.LagrangianCR(g, r=case["eps"])
        assert bits.tolist() == case["bits"]
        assert fun == pytest.approx(case["fun"], rel=1e-12)


def test_scheme_from_sensitivities_matches_driver_solve():
    g = np.array(GOLD["grads"]["elastic_2d/elastic_2d.npy"])
    r = np.array(GOLD["ranges"]["elastic_2d/elastic_2d.npy"])
    bits, ranges = solvers.scheme_from_sensitivities(g, r, dim=2, mode="EB", eps=1e-2, ref=6893.409)
    case = [c for c in GOLD["solver"] if c["key"] == "elastic_2d/elastic_2d.npy" and c["mode"] == "EB"
            and c["eps"] == 1e-2][0]
    assert (bits - 1).tolist() == case["bits"]
    assert ranges[:2].tolist() == [1.0, 1.0]


def test_error_model_step_gradient():
    from autoquantizer_b200.adjoint import step_gradient

    sens = np.array([4.0, 9.0])
    g = step_gradient(sens, bits=[9, 5], ranges=[2.0, 1.0])
    assert g == pytest.approx([4.0 * (2.0 / 256) / 6, 9.0 * (1.0 / 16) / 6])


SCIPY_GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "scipy_solver.json")))


@pytest.mark.parametrize("case", SCIPY_GOLD["cases"],
                         ids=lambda c: "%s-%s-%g" % (c["key"].split("/")[0], c["form"], c["eps"]))
def test_slsqp_solvers_match_reference(case):
    """The SLSQP solvers give the reference's bit widths (and stop where it
    stops) on the reference's shipped sensitivities and ranges."""
    g = np.array(case["grad"])
    n = len(g)
    if case["form"] == "mem":
        s = solvers.ScipySolverMemMode(n, a=[1], eps=case["eps"], grad=g)
    else:
        s = solvers.ScipySolver(n, a=np.ones(n), eps=case["eps"], grad=g)
    s.set_range(case["ranges"])
    res = s.run()
    assert int(res.status) == case["status"]
    assert [int(b) for b in s.get_bits()] == case["bits"]


def test_slsqp_memory_form_meets_its_budget():
    """Where SLSQP converges, the memory form's widths stay within the
    budget it was given (sum of -log2(sqrt(3) x / R) <= 32 eps n, up to the
    rounding up of each width) and spend more bits on more sensitive scalars."""
    case = [c for c in SCIPY_GOLD["cases"] if c["form"] == "mem" and c["status"] == 0][0]
    g = np.array(case["grad"])
    n = len(g)
    s = solvers.ScipySolverMemMode(n, a=[1], eps=case["eps"], grad=g)
    s.set_range(case["ranges"])
    assert s.run().status == 0
    bits = np.array(s.get_bits())
    assert bits.sum() <= 32 * case["eps"] * n + n
    cont = -np.log2(np.sqrt(3.0) * np.abs(s.sol) / np.array(case["ranges"]))
    assert cont.sum() == pytest.approx(32 * case["eps"] * n, rel=1e-6)
