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


def _orient_outward(tris, centre):
    """Swap b and c of every triangle whose normal points towards centre."""
    t = np.array(tris, dtype=np.float64).reshape(-1, 3, 3)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    flip = ((t.mean(1) - np.asarray(centre)) * n).sum(1) < 0
    t[flip, 1], t[flip, 2] = t[flip, 2].copy(), t[flip, 1].copy()
    return t.reshape(-1, 9)


def box_mesh(lo, hi):
    """12 triangles of the box [lo, hi], normals outward."""
    lo, hi = np.asarray(lo, dtype=np.float64), np.asarray(hi, dtype=np.float64)
    c = [[lo[0] if i & 1 == 0 else hi[0], lo[1] if i & 2 == 0 else hi[1], lo[2] if i & 4 == 0 else hi[2]]
         for i in range(8)]
    quads = [(0, 1, 3, 2), (4, 5, 7, 6), (0, 1, 5, 4), (2, 3, 7, 6), (0, 2, 6, 4), (1, 3, 7, 5)]
    tris = []
    for a, b, d, e in quads:
        tris += [c[a] + c[b] + c[d], c[a] + c[d] + c[e]]
    return _orient_outward(tris, (lo + hi) / 2)


def sphere_mesh(centre, radius, n_lat=12, n_lon=16):
    """UV sphere (normals outward)."""
    centre = np.asarray(centre, dtype=np.float64)

    def pt(i, j):
        th, ph = np.pi * i / n_lat, 2 * np.pi * j / n_lon
        return list(centre + radius * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)]))

    tris = []
    for i in range(n_lat):
        for j in range(n_lon):
            a, b, c, d = pt(i, j), pt(i + 1, j), pt(i + 1, j + 1), pt(i, j + 1)
            if i > 0:
                tris.append(a + b + d)
            if i < n_lat - 1:
                tris.append(b + c + d)
    return _orient_outward(tris, centre)
