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


def host_threads():
    try:
        import os

        return max(1, len(os.sched_getaffinity(0)))
    except Exception:
        return 1


def twin(cfg, values, threads=1):
    """GPU MPMSolver and oracle Sim holding identical packed records
    (threads > 1: the oracle's OpenMP substep, for full-size scenes)."""
    from autoquantizer_b200.mpm_solver import MPMSolver

    s = MPMSolver(cfg)
    s.set_particles(values)
    L = oracle_layout_from(s.record())
    o = O.Sim(oracle_params_from(s._params()), L, threads=threads)
    o.set_state(values)
    s.set_words(o.words)
    return s, o


def compare_states(s, o, rel, steps_slack=1.0):
    """Slot by slot, max |GPU - oracle| within rel * max(1, max |value|),
    plus steps_slack quantization steps for fixed-point slots (a dithered
    rounding can land on the neighbouring code) or 2^-10 relative for
    floats with exponents.  Returns per-slot (max error, tolerance)."""
    g = s.state_values()
    r = o.get_state()
    assert g.shape == r.shape
    q = quant_steps(s)
    out = []
    for k in range(g.shape[1]):
        scale = max(1.0, float(np.max(np.abs(r[:, k]))))
        tol = rel * scale
        if q[k] > 0:
            tol += steps_slack * q[k]
        elif np.isnan(q[k]):
            tol += 2.0 ** -10 * scale
        err = float(np.max(np.abs(g[:, k] - r[:, k])))
        out.append((err, tol))
    bad = [(k, e, t) for k, (e, t) in enumerate(out) if not e <= t]
    assert not bad, "slots over tolerance (slot, max err, tol): %s" % bad
    return out


def compare_states_stats(s, o, rel=2e-5, steps_slack=2.0, max_frac=1e-4, x_codes=2.0):
    """Statistical agreement for runs long enough that a dithered rounding of
    x can land on the neighbouring code in one implementation and not the
    other (the GPU and the oracle add the grid sums in different orders, so
    x before rounding differs in its last bits).  One x code changes the
    particle's next C by about 4 inv_dx^2 |dv| dx_code, many C steps, so the
    per-slot bound of compare_states cannot hold for every particle.
    Required: every position within x_codes quantization steps (or rel for
    raw slots), at most max_frac of the particles with any slot beyond the
    compare_states tolerance, and a mean error below a tenth of that
    tolerance in every slot.  Returns the fraction of particles beyond."""
    g = s.state_values()
    r = o.get_state()
    assert g.shape == r.shape
    q = quant_steps(s)
    d = s.dim
    tol = np.empty(g.shape[1])
    for k in range(g.shape[1]):
        scale = max(1.0, float(np.max(np.abs(r[:, k]))))
        tol[k] = rel * scale + (steps_slack * q[k] if q[k] > 0 else 2.0 ** -10 * scale if np.isnan(q[k]) else 0.0)
    err = np.abs(g - r)
    xt = np.where(q[:d] > 0, x_codes * q[:d], tol[:d])
    assert np.all(err[:, :d] <= xt), ("positions", err[:, :d].max(0), xt)
    frac = float(np.mean(np.any(err > tol, axis=1)))
    assert frac <= max_frac, ("particles beyond tolerance", frac, err.max(0) / tol)
    mean = err.mean(0)
    assert np.all(mean <= 0.1 * tol), ("mean error", mean / tol)
    return frac


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
