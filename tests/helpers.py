"""Shared test helpers: product-side objects built next to their oracle twins."""
import numpy as np

import oracle as O
from autoquantizer_b200 import _lib


def oracle_layout_from(bitpack):
    f64, dith = bitpack.compute_and_dithering()
    return O.build_layout(bitpack.spec_tuples(), f64, dith)


def oracle_params_from(P):
    d = P.dim
    mats = [(P.mat[i].kind, P.mat[i].mu, P.mat[i].lam) for i in range(max(1, P.n_materials))]
    return {"dim": d, "precision": P.precision, "res": [P.res[k] for k in range(d)],
            "lb": [P.lb[k] for k in range(d)], "ub": [P.ub[k] for k in range(d)], "has_F": P.has_F,
            "has_mat": P.has_mat, "materials": mats, "use_friction": P.use_friction,
            "use_bound_clip": P.use_bound_clip, "dx": P.dx, "dt": P.dt, "p_vol": P.p_vol, "p_mass": P.p_mass,
            "gravity": P.gravity, "seed": P.seed}


def twin(cfg, values):
    """GPU MPMSolver and oracle Sim holding identical packed records."""
    from autoquantizer_b200.mpm_solver import MPMSolver

    s = MPMSolver(cfg)
    s.set_particles(values)
    L = oracle_layout_from(s.record())
    o = O.Sim(oracle_params_from(s._params()), L)
    o.set_state(values)
    s.set_words(o.words)
    return s, o


def quant_steps(solver):
    """Per-slot quantization step of a layout (0 for raw slots)."""
    L = solver.layout()
    out = []
    for i in range(L.n_slots):
        S = L.slot[i]
        if S.kind == _lib.AQ_FIXED:
            out.append(S.scale_f64)
        elif S.kind in (_lib.AQ_FLOAT_EXP, _lib.AQ_SHARED_EXP):
            out.append(np.nan)  # relative: handled by the caller
        else:
            out.append(0.0)
    return np.array(out)
