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
