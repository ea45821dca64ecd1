"""Closed-form bit-width allocation for quantized fields.

Same interface and results as the reference's solvers/analytical_solver.py
(LagrangianCR :3-47, LagrangianEB :50-84).  The error model (mpm_solver.py:
461-470) gives each quantized scalar i a quantization step
Delta_i = R_i / 2^b_i with uniform error variance Delta_i^2 / 12, so the
simulation error is approximated by E = sum_i g_i 4^-b_i / 12 with
g_i = (sum of squared sensitivities) * R_i^2.

  * LagrangianCR: minimise E under a memory budget sum_i a_i (b_i + 1)
    = 32 r sum_i a_i (one sign bit per scalar).  Stationarity gives
    b_i = r' + (tbar - t_i)/2 with t_i = log2(a_i / g_i), tbar the a-weighted
    mean of t, r' = 32 r - 1; bits are rounded down.
  * LagrangianEB: minimise memory under E <= (ref * tol_rel)^2.  Equal
    marginal cost gives (Delta_i/R_i)^2 = x_i = 12 tol a_i / (g_i sum a),
    b_i = ceil(-log2(x_i) / 2).
Both return fraction bits; callers add the sign bit.
"""
import numpy as np

LOG2_LN2 = np.log2(np.log(2.0))


def LagrangianCR(grads, r=0.5, a=None, debug=False):
    g = np.asarray(grads, dtype=np.float64)
    n = len(g)
    w = np.ones(n, dtype=np.float64) if a is None else np.asarray(a, dtype=np.float64)
    assert len(w) == n
    rp = 32.0 * r - 1.0
    t = np.log2(w / g)
    tbar = t @ w / np.sum(w)
    log_lambda = -2.0 * rp - tbar + LOG2_LN2  # log2 of the Lagrange multiplier
    frac = -(t + log_lambda - LOG2_LN2) / 2.0
    est = (w / g * np.power(2.0, log_lambda) / np.log(2.0)) @ g / 12.0
    if debug:
        print((frac + 1).sum() / 32 / w.sum())
    return np.floor(frac).astype(np.int32), est


def LagrangianEB(grads, ref, tol_rel=1e-3, a=None):
    g = np.asarray(grads, dtype=np.float64)
    n = len(g)
    w = np.ones(n, dtype=np.float64) if a is None else np.asarray(a, dtype=np.float64)
    assert len(w) == n
    tol = (ref * tol_rel) ** 2
    x = 12.0 / np.sum(w) * tol * (w / g)
    bits = np.ceil(-np.log2(x) / 2.0).astype(np.int32)
    rel = np.sqrt(x @ g / (12.0 * ref ** 2))
    return bits, rel


def scheme_from_sensitivities(grads, ranges, dim, mode="EB", eps=1e-3, ref=1.0):
    """The drivers' solve() step (mpm_exps/run_mpm_elastic_2d.py:227-242):
    position ranges fixed to 1, other ranges doubled, then bits + 1 sign bit."""
    ranges = np.array(ranges, dtype=np.float64)
    ranges[:dim] = 1.0
    ranges[dim:] *= 2.0
    g = np.asarray(grads, dtype=np.float64) * ranges ** 2
    if mode == "CR":
        bits, _ = LagrangianCR(g, r=eps)
    else:
        bits, _ = LagrangianEB(g, ref=ref, tol_rel=eps)
    return bits + 1, ranges
