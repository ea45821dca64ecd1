"""Golden bit widths of the reference's SLSQP solvers (solvers/scipy_solver.py),
imported from a reference checkout and run on the sensitivities and ranges
the reference ships (mpm_exps/grads, mpm_exps/ranges), with the range recipe
of the drivers' solve() steps (position ranges 1, other ranges doubled).

    python tests/golden/make_scipy_golden.py <path of the AutoQuantizer reference checkout>

writes tests/golden/scipy_solver.json.  The memory-budget form gets the
sensitivities divided by their minimum, as run_mpm_fluid_3d_scaling.py:333
does; the error-bound form gets g R^2 divided by its maximum and unit
weights.  SLSQP stops early on some inputs (status 4 or 8); those cases are
kept, with their status, since a faithful restatement stops the same way.
"""
import contextlib
import importlib.util
import io
import json
import os
import sys

import numpy as np

CASES = [  # (grads file, ranges file, dim), under mpm_exps/grads and mpm_exps/ranges
    ("fluid_3d_scaling/fluid_3d_t16385_dt0.0002_p200000_g64.npy", "fluid_3d_scaling/fluid_3d_t65537_dt5e-05_p5000000_g256.npy", 3),
    ("fluid_3d/fluid_3d.npy", "fluid_3d/fluid_3d.npy", 3),
    ("elastic_3d/elastic_3d.npy", "elastic_3d/elastic_3d.npy", 3),
    ("elastic_2d/elastic_2d.npy", "elastic_2d/elastic_2d.npy", 2),
    ("fluid_2d/fluid_2d_t16385_dt0.0002_p10000_g128.npy", "fluid_2d/fluid_2d_t16385_dt0.0002_p10000_g128.npy", 2),
]
MEM_EPS = (0.25, 0.3, 0.4, 0.5)
EB_EPS = (1e-3, 1e-2, 1e-1)


def main(ref):
    spec = importlib.util.spec_from_file_location("ref_scipy_solver", os.path.join(ref, "solvers", "scipy_solver.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    out = {"source": "AutoQuantizer reference checkout, solvers/scipy_solver.py", "cases": []}
    for gk, rk, dim in CASES:
        g = np.load(os.path.join(ref, "mpm_exps", "grads", gk))
        r = np.load(os.path.join(ref, "mpm_exps", "ranges", rk)).astype(np.float64)
        r[:dim] = 1.0
        r[dim:] *= 2.0
        n = len(g)
        for eps in MEM_EPS:
            gg = g / g.min()
            s = m.ScipySolverMemMode(n, a=[1], eps=eps, grad=gg)
            s.set_range(r)
            with contextlib.redirect_stdout(io.StringIO()):
                res = s.run()
            out["cases"].append({"key": gk, "form": "mem", "eps": eps, "grad": gg.tolist(), "ranges": r.tolist(),
                                 "status": int(res.status), "bits": [int(b) for b in s.get_bits()]})
        for eps in EB_EPS:
            gw = g * r ** 2
            gg = gw / gw.max()
            s = m.ScipySolver(n, a=np.ones(n), eps=eps, grad=gg)
            s.set_range(r)
            with contextlib.redirect_stdout(io.StringIO()):
                res = s.run()
            out["cases"].append({"key": gk, "form": "eb", "eps": eps, "grad": gg.tolist(), "ranges": r.tolist(),
                                 "status": int(res.status), "bits": [int(b) for b in s.get_bits()]})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scipy_solver.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", path, len(out["cases"]), "cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path of the AutoQuantizer reference checkout>" % sys.argv[0])
    main(sys.argv[1])
