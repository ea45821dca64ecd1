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


# ------------------------------------------------------------------ SLSQP
# The reference's numerical alternative to the closed forms
# (solvers/scipy_solver.py): the same allocation problems, posed in the RMS
# rounding errors x_i = Delta_i / sqrt(12) of the scalars, handed to SciPy's
# SLSQP.
# The objective, constraint, bounds, starting point and options are the
# reference's, expression for expression, because SLSQP's path (and, where it
# stops early, its answer) depends on every value it is given; only the
# printing is left out.  Bits are the reference's ceil(-log2(sqrt(3) x / R)).

class _SlsqpBase:
    """n_vars quantized scalars, weights a, bound eps, sensitivities grad
    (scipy_solver.py:9-22); set_range gives the scalars' ranges R_i."""

    def __init__(self, n_vars, a=None, eps=None, grad=None):
        self.n_vars = n_vars
        self.a = a
        self.eps = eps
        self.grad = grad
        self.sol = None
        self.r = [1.0] * len(self.a)

    def set_range(self, _range):
        # list slice assignment: the list takes the given ranges' length
        self.r[:] = _range[:]


class ScipySolver(_SlsqpBase):
    """Error-bound form (scipy_solver.py:26-78): minimise the bits
    sum_i a_i (-log2 x_i) subject to sum_i g_i x_i^2 <= eps^2, x_i in
    [1e-23, 1]; the objective's gradient is left to SLSQP's differences."""

    def __init__(self, n_vars, a=None, eps=None, grad=None):
        super().__init__(n_vars, a, eps, grad)
        self.lb = 1e-32
        self.bounds = [(1e-23, 1) for _ in range(self.n_vars)]

    def run(self):
        from scipy.optimize import NonlinearConstraint, minimize

        con = NonlinearConstraint(fun=self.con, lb=0.0, ub=self.eps ** 2, jac=self.con_jac)
        x0 = np.sqrt(np.ones(self.n_vars) * (self.eps ** 2 / self.n_vars) / self.grad)
        res = minimize(self.obj, x0, method="SLSQP", constraints=con, bounds=self.bounds,
                       options={"maxiter": 10000})
        self.sol = np.array(res.x)
        return res

    def con(self, x):
        return np.dot(self.grad.reshape(1, self.n_vars), x * x)

    def con_jac(self, x):
        return 2 * self.grad * x

    def obj(self, x):
        return np.dot(-np.log2(np.abs(x)), self.a)

    def jac(self, x):
        return ((x + self.lb) ** -1) * (-1.0 / np.log(2.0)) * self.a

    def get_bits(self):
        return [np.ceil(-np.log2(np.abs(np.sqrt(3.0) * self.sol[i] / self.r[i]))) for i in range(self.n_vars)]


class ScipySolverMemMode(_SlsqpBase):
    """Memory-budget form (scipy_solver.py:81-134), the one the 3D fluid
    scaling driver calls (run_mpm_fluid_3d_scaling.py:331-336): minimise
    0.5 sum_i g_i x_i^2 subject to sum_i -log2(sqrt(3) |x_i| / R_i) in
    [0, 32 eps n_vars], x_i in [1e-32, 1], with analytic gradients."""

    def __init__(self, n_vars, a=None, eps=None, grad=None):
        super().__init__(n_vars, a, eps, grad)
        self.lb = 1e-32
        self.bounds = [(self.lb, 1) for _ in range(self.n_vars)]

    def run(self):
        from scipy.optimize import NonlinearConstraint, minimize

        con = NonlinearConstraint(fun=self.con, lb=(0,), ub=(self.eps * self.n_vars * 32,), jac=self.con_jac)
        x0 = np.ones(self.n_vars) * (self.eps ** 2 / self.n_vars) / self.grad
        res = minimize(self.obj, x0, jac=self.jac, method="SLSQP", constraints=con, bounds=self.bounds,
                       options={"maxiter": 10000})
        self.sol = np.array(res.x)
        return res

    def con(self, x):
        return np.sum(-np.log2(np.sqrt(3.0) * np.abs(x + 1e-23) / self.r))

    def con_jac(self, x):
        return ((x + self.lb) ** -1) * (-1.0 / np.log(2.0))

    def obj(self, x):
        return 0.5 * np.dot(self.grad, x ** 2)

    def jac(self, x):
        return self.grad * x

    def hess(self, x):
        return np.diag(self.grad)

    def get_bits(self):
        return [np.ceil(-np.log2(self.lb + np.abs(np.sqrt(3.0) * self.sol[i]) / self.r[i]))
                for i in range(self.n_vars)]
