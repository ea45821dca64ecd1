"""Error gradients of the 3D falling block (the adjoint benchmark scene) and
their finite-difference check.

    python -m autoquantizer_b200.adjoint_report [--n 262144] [--grid 64]
        [--substeps 256] [--every 16] [--projections 4] [--out report.json]

Scene: 262,144 elastic particles (E 5e3, nu 0.3) dropped onto the floor of a
64^3 grid, dt 5e-5, 256 substeps, FP32 forward with checkpoints every 16.

Quantity: the expected squared final-position error E|x_T - x_T*|^2 under
the reference's error model (quantization noise of variance Delta_f^2 / 12
added to every scalar of field f at every substep, mpm_solver.py:461-470)
is sum_f Delta_f^2 / 12 * S_f with S_f = sum_{t,p, scalars of f}
|d x_T / d s_t|^2.  S_f is estimated with random projections: for r with
independent +-1 entries, L_r = r . x_T has E_r[(dL_r/ds)^2] = |dx_T/ds|^2,
so the mean over projections of the adjoint's per-slot sums
(aq_adjoint_backward) estimates S.  Fields are the 12 groups x, v
components and rows of C and F; dE/dDelta_f = S_f Delta_f / 6.

Check: for each group, the adjoint's directional derivative of L_r along a
perturbation of that group's scalars at t = 0 against central finite
differences with h = 1e-3 (relative to each scalar's magnitude; positions
relative to a cell), in the FP32 forward and in an FP64 forward.
"""
import argparse
import json
import time

import numpy as np

GROUP_NAMES = ["x0", "x1", "x2", "v0", "v1", "v2", "C_row0", "C_row1", "C_row2", "F_row0", "F_row1", "F_row2"]


def group_slots():
    g = [[0], [1], [2], [3], [4], [5]]
    g += [[6 + 3 * r + c for c in range(3)] for r in range(3)]
    g += [[15 + 3 * r + c for c in range(3)] for r in range(3)]
    return g


def _setup(n, grid, precision):
    import torch

    from . import scenes
    from .adjoint import Adjoint
    from .mpm_solver import MPMSolver

    cfg, vals = scenes.falling_block_3d(n=n, n_grid=grid)
    cfg.precision = precision
    s = MPMSolver(cfg)
    s.set_particles(vals)
    adj = Adjoint(s._params())
    dt = torch.float64 if precision == "f64" else torch.float32
    s0 = torch.from_numpy(vals).to("cuda", dt)
    return cfg, adj, s0


def sensitivities(n=262144, grid=64, substeps=256, every=16, projections=4, seed=0):
    """Group sensitivities S_f (mean over projections) and timings."""
    import torch

    cfg, adj, s0 = _setup(n, grid, "f32")
    gen = torch.Generator(device="cuda").manual_seed(seed)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    ev[0].record()
    sT = adj.forward(s0, substeps, every)
    ev[1].record()
    sens = np.zeros(s0.shape[1])
    t_bwd = 0.0
    for k in range(projections):
        r = torch.randint(0, 2, (s0.shape[0], 3), generator=gen, device="cuda").to(s0.dtype) * 2 - 1
        seed_t = torch.zeros_like(sT)
        seed_t[:, :3] = r
        ev[2].record()
        _, sk = adj.backward(seed_t)
        ev[3].record()
        torch.cuda.synchronize()
        t_bwd += ev[2].elapsed_time(ev[3])
        sens += sk / projections
    t_fwd = ev[0].elapsed_time(ev[1])
    adj.close()
    S = np.array([sens[g].sum() for g in group_slots()])
    return S, sens, t_fwd, t_bwd / projections


def fd_check(precision, n=262144, grid=64, substeps=256, every=16, h=1e-3, seed=1):
    """Adjoint vs central differences of L_r, per group."""
    import torch

    cfg, adj, s0 = _setup(n, grid, precision)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    r = torch.randint(0, 2, (s0.shape[0], 3), generator=gen, device="cuda").to(s0.dtype) * 2 - 1

    def L(st):
        return float((r.double() * st[:, :3].double()).sum())

    sT = adj.forward(s0, substeps, every)
    seed_t = torch.zeros_like(sT)
    seed_t[:, :3] = r
    g0, _ = adj.backward(seed_t)
    scale = torch.clamp(s0.abs().max(0).values, min=1e-3)
    scale[:3] = 1.0 / grid
    out = []
    rng = np.random.default_rng(seed)
    for name, slots in zip(GROUP_NAMES, group_slots()):
        u = torch.zeros_like(s0)
        for sl in slots:
            u[:, sl] = torch.from_numpy(rng.normal(size=s0.shape[0])).to("cuda", s0.dtype) * scale[sl]
        fd = (L(adj.forward(s0 + h * u, substeps, every)) - L(adj.forward(s0 - h * u, substeps, every))) / (2 * h)
        an = float((g0.double() * u.double()).sum())
        out.append({"group": name, "adjoint": an, "fd": fd, "rel_err": abs(an - fd) / max(abs(fd), 1e-30)})
    adj.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--grid", type=int, default=64)
    ap.add_argument("--substeps", type=int, default=256)
    ap.add_argument("--every", type=int, default=16)
    ap.add_argument("--projections", type=int, default=4)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    S, sens, t_fwd, t_bwd = sensitivities(a.n, a.grid, a.substeps, a.every, a.projections)
    # example scheme: the 3D throughput scene's widths (x 21 bits on range 1,
    # v 12 bits, C 16 bits on 64, F 16 bits on 2) as fixed point
    delta = np.array([1 / 2 ** 20] * 3 + [2.0 / 2 ** 11] * 3 + [64 / 2 ** 15] * 3 + [2 / 2 ** 15] * 3)
    rep = {"scene": "falling_block_3d", "particles": a.n, "grid": a.grid, "substeps": a.substeps,
           "checkpoint_every": a.every, "projections": a.projections,
           "forward_ms": t_fwd, "backward_ms_per_projection": t_bwd,
           "groups": GROUP_NAMES, "S": S.tolist(), "per_slot_S": sens.tolist(),
           "example_delta": delta.tolist(), "dE_dDelta": (S * delta / 6).tolist(),
           "E_final_pos_err2": float((S * delta ** 2 / 12).sum()),
           "fd_f32": fd_check("f32", a.n, a.grid, a.substeps, a.every),
           "fd_f64": fd_check("f64", a.n, a.grid, a.substeps, a.every),
           "wall_seconds": time.perf_counter() - t0}
    print(json.dumps(rep, indent=1))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rep, f, indent=1)
    return rep


if __name__ == "__main__":
    main()
