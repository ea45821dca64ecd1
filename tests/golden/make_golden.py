"""Regenerate the golden fixtures of this folder from the AutoQuantizer
reference checkout (read-only), given as the one argument:

    python tests/golden/make_golden.py <reference checkout>

Writes reference_data.json and propeller_higher.npz:
  * the reference's shipped autodiff sensitivities and detected ranges
    (mpm_exps/grads/*/*.npy, mpm_exps/ranges/*/*.npy);
  * the scene constants and the f64 reference loss of the 2D elastic
    experiment (mpm_exps/run_mpm_elastic_2d.py:54-80);
  * outputs of the reference's own analytical bit-width solvers
    (solvers/analytical_solver.py, imported from the checkout) on those
    sensitivities, as the drivers' solve() calls them
    (run_mpm_elastic_2d.py:227-242), for several error bounds and
    compression rates;
  * outputs of the compression-rate solver that run_mpm_fluid_2d.py
    defines locally (:129-145; only that function is taken out of the
    script with ast and run, since the script itself imports Taichi), with
    that driver's solve() recipe (:162-178);
  * outputs of the reference's LagrangianCR with the range recipes of the
    3D drivers' solve() (run_mpm_elastic_3d.py:323-333,
    run_mpm_fluid_3d.py:149-161);
  * the reference's MPMConfig defaults (mpm_exps/mpm_config.py).
Nothing at test time reads the reference checkout; tests read the JSON.
"""
import ast
import glob
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    spec = importlib.util.spec_from_file_location("ref_analytical", os.path.join(ref, "solvers", "analytical_solver.py"))
    ana = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ana)
    out = {"source": "AutoQuantizer reference checkout", "grads": {}, "ranges": {}, "solver": []}
    for kind in ("grads", "ranges"):
        for f in sorted(glob.glob(os.path.join(ref, "mpm_exps", kind, "*", "*.npy"))):
            key = os.path.relpath(f, os.path.join(ref, "mpm_exps", kind))
            out[kind][key] = np.load(f).tolist()
    out["elastic_2d"] = {
        "f64_loss": 6893.409, "n_particles": 80000, "dt": 2e-4, "n_grid": 128, "n_timesteps": 1024 * 8 + 1,
        "E": 5e1, "nu": 0.2, "bound": [3, 3], "size": 1, "p_rho": 1.0, "g": 9.8,
        "cubes_low": [[(0.2 + i * 0.4) / 4, (0.2 + i * 0.8) / 4] for i in range(4)] +
                     [[(3.1 - i * 0.2) / 4, (0.2 + i * 0.8) / 4] for i in range(4)],
        "cube_size": [0.7 / 4, 0.7 / 4], "per_cube": 80000 // 8,
    }
    # solve() of the 2D drivers on the shipped data
    dims = {"elastic_2d/elastic_2d.npy": 2, "fluid_2d/fluid_2d_t16385_dt0.0002_p10000_g128.npy": 2,
            "elastic_3d/elastic_3d.npy": 3, "fluid_3d/fluid_3d.npy": 3}
    for key, dim in dims.items():
        g = np.array(out["grads"][key])
        r = np.array(out["ranges"][key], dtype=np.float64)
        r[:dim] = 1.0
        r[dim:] *= 2.0
        gw = g * r ** 2
        for eps in (1e-1, 1e-2, 1e-3):
            bits, rel = ana.LagrangianEB(grads=gw, ref=6893.409, tol_rel=eps)
            out["solver"].append({"key": key, "mode": "EB", "eps": eps, "ref": 6893.409,
                                  "grads_weighted": gw.tolist(), "bits": bits.tolist(), "rel": float(rel)})
        for rate in (0.3, 0.5, 0.7):
            bits, fun = ana.LagrangianCR(grads=gw, r=rate)
            out["solver"].append({"key": key, "mode": "CR", "eps": rate, "grads_weighted": gw.tolist(),
                                  "bits": bits.tolist(), "fun": float(fun)})
    # solve() of run_mpm_fluid_2d.py with its own LagrangianCR
    src = open(os.path.join(ref, "mpm_exps", "run_mpm_fluid_2d.py")).read()
    fn = [n for n in ast.parse(src).body if isinstance(n, ast.FunctionDef) and n.name == "LagrangianCR"][0]
    ns = {"np": np}
    exec(compile(ast.Module(body=[fn], type_ignores=[]), "run_mpm_fluid_2d.py", "exec"), ns)
    key = "fluid_2d/fluid_2d_t16385_dt0.0002_p10000_g128.npy"
    out["driver_solver"] = []
    for rate in (0.3, 0.5, 0.7):
        g = np.array(out["grads"][key])
        r = np.array(out["ranges"][key], dtype=np.float64)
        r[:2] = 1.0
        r[2:] *= 2.0
        g = g / g.min()
        bits, fun = ns["LagrangianCR"](g * r ** 2, r=rate)
        out["driver_solver"].append({"driver": "fluid_2d", "key": key, "mode": "CR", "eps": rate,
                                     "ranges": r.tolist(), "bits": bits.tolist(), "fun": float(fun)})
    # solve() of run_mpm_elastic_3d.py (:323-333) and run_mpm_fluid_3d.py
    # (:149-161): their own range recipes, the reference's LagrangianCR
    for driver, key in (("elastic_3d", "elastic_3d/elastic_3d.npy"), ("fluid_3d", "fluid_3d/fluid_3d.npy")):
        for rate in (0.3, 0.512, 0.7):
            g = np.array(out["grads"][key])
            r = np.array(out["ranges"][key], dtype=np.float64)
            if driver == "elastic_3d":
                r[:] *= 2.0
                r[:3] = 4.0
            else:
                r[6:15] *= 24
                r[3:6] *= 1.5
                r[-1] *= 1.5
                r[:3] = 2.0
            bits, fun = ana.LagrangianCR(g * (r ** 2), r=rate)
            out["driver_solver"].append({"driver": driver, "key": key, "mode": "CR", "eps": rate,
                                         "ranges": r.tolist(), "bits": bits.tolist(), "fun": float(fun)})
    # MPMConfig defaults (mpm_exps/mpm_config.py, imported from the checkout)
    spec = importlib.util.spec_from_file_location("ref_mpm_config", os.path.join(ref, "mpm_exps", "mpm_config.py"))
    cfg_mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cfg_mod)
    out["mpm_config_defaults"] = dict(vars(cfg_mod.MPMConfig()))
    with open(os.path.join(HERE, "reference_data.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "reference_data.json"))
    # the propeller collider of the 3D fluid experiment's gradient and range
    # passes (run_mpm_fluid_3d.py:101-146 with init_sdf_value,
    # mpm_solver.py:284-318), as float32 volumes, the precision the
    # simulator reads them in
    inp = os.path.join(ref, "mpm_exps", "inputs")
    sdf = np.load(os.path.join(inp, "propeller_higher.npz"))["sdf"].astype(np.float32)
    nrm = np.load(os.path.join(inp, "propeller_higher_normal.npz"))["sdf"].astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "propeller_higher.npz"), sdf=sdf, normal=nrm)
    print("wrote", os.path.join(HERE, "propeller_higher.npz"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path of the AutoQuantizer reference checkout>" % sys.argv[0])
    main(sys.argv[1])
