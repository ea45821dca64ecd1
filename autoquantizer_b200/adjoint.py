"""Adjoint of the substep: quantization sensitivities and a torch autograd
Function over substep rollouts.

The reference gets these from Taichi's reverse-mode autodiff with nlogn
checkpointing (MPMSolver.run_forward_with_ad_nlogn / accu_grad /
get_gradients, mpm_exps/engine/mpm_solver.py:1093-1302).  Here the reverse
substep is hand-written CUDA (libaq: aq_adjoint_*), checkpointed every
`every` substeps with each segment recomputed during the backward pass.

    adj = Adjoint(params)                      # aq_params of an unquantized state
    sT = adj.forward(s0, n_substeps, every)    # (n x n_slots) cuda tensors;
                                               # every = 0: logarithmic stash
    g0, sens = adj.backward(dL_dsT)            # dL/ds0 and per-slot sum of
                                               # (dL/ds_t)^2, t = 1..T-1

    sT = Rollout.apply(s0, adj, n_substeps, every)   # differentiable in s0

The error model of the reference (mpm_solver.py:461-470): storing scalar i
with step Delta_i = R_i / 2^(b_i - 1) adds uniform noise of variance
Delta_i^2 / 12 per substep, so E[dL^2] ~= sum_i sens_i Delta_i^2 / 12 and
dE/dDelta_i = sens_i Delta_i / 6.
"""
import ctypes as C

import numpy as np

from . import _lib


class Adjoint:
    def __init__(self, params):
        self._h = C.c_void_p()
        P = _lib.Params()
        C.pointer(P)[0] = params
        P.has_mat = 0
        self.P = P
        self.dim = P.dim
        self.n = P.n_particles
        d = P.dim
        self.n_slots = 2 * d + d * d + (d * d if P.has_F else 1)
        _lib.check(_lib.lib().aq_adjoint_create(C.byref(P), C.byref(self._h)), "aq_adjoint_create")
        self._dtype = None
        self.sens = None

    def _dt(self):
        import torch

        return torch.float64 if self.P.precision else torch.float32

    def forward(self, s0, n_substeps, every=16):
        import torch

        s0 = s0.to(device="cuda", dtype=self._dt()).contiguous()
        assert s0.shape == (self.n, self.n_slots)
        out = torch.empty_like(s0)
        _lib.check(_lib.lib().aq_adjoint_forward(self._h, C.c_void_p(s0.data_ptr()), int(n_substeps), int(every),
                                                 C.c_void_p(out.data_ptr()), _lib.stream_ptr()), "aq_adjoint_forward")
        return out

    def backward(self, seed):
        import torch

        seed = seed.to(device="cuda", dtype=self._dt()).contiguous()
        g0 = torch.empty_like(seed)
        sens = (C.c_double * self.n_slots)()
        _lib.check(_lib.lib().aq_adjoint_backward(self._h, C.c_void_p(seed.data_ptr()), C.c_void_p(g0.data_ptr()),
                                                  sens, _lib.stream_ptr()), "aq_adjoint_backward")
        self.sens = np.array(sens[:])
        return g0, self.sens

    def set_collider(self, sdf, normal, offset, center, theta=0.0, height=0.0, omega=5.0, height_rate=0.1):
        """The rotating SDF collider in every substep (aq_adjoint_set_collider):
        sdf and normal are float32 CUDA tensors ([a, b, c] and [a, b, c, 3])
        kept alive here; theta and height are the values at substep 0."""
        self._col = (sdf, normal)
        dims = (C.c_int32 * 3)(*sdf.shape)
        off = (C.c_int32 * 3)(*offset)
        _lib.check(_lib.lib().aq_adjoint_set_collider(self._h, C.c_void_p(sdf.data_ptr()), C.c_void_p(normal.data_ptr()),
                                                      dims, off, int(center), float(theta), float(height),
                                                      float(omega), float(height_rate)), "aq_adjoint_set_collider")

    def close(self):
        if self._h:
            _lib.lib().aq_adjoint_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _rollout_cls():
    import torch

    class Rollout(torch.autograd.Function):
        """s_T = substep^T(s_0); backward runs the hand-written adjoint and
        leaves the quantization sensitivities in adj.sens."""

        @staticmethod
        def forward(ctx, s0, adj, n_substeps, every=16):
            ctx.adj = adj
            return adj.forward(s0, n_substeps, every)

        @staticmethod
        def backward(ctx, g):
            g0, _ = ctx.adj.backward(g)
            return g0, None, None, None

    return Rollout


_Rollout = None


def rollout(s0, adj, n_substeps, every=16):
    global _Rollout
    if _Rollout is None:
        _Rollout = _rollout_cls()
    return _Rollout.apply(s0, adj, n_substeps, every)


def ek_seed(sT, dim, p_mass, g):
    """dL/ds_T of compute_ek (mpm_solver.py:1043-1052): 2D sum |v|^2, 3D
    sum 0.5 m |v|^2 + g m x_y."""
    import torch

    seed = torch.zeros_like(sT)
    v = sT[:, dim:2 * dim]
    if dim == 3:
        seed[:, dim:2 * dim] = p_mass * v
        seed[:, 1] = g * p_mass
    else:
        seed[:, dim:2 * dim] = 2 * v
    return seed


def ek_loss(sT, dim, p_mass, g):
    v = sT[:, dim:2 * dim]
    if dim == 3:
        return float((0.5 * p_mass * (v * v).sum() + g * p_mass * sT[:, 1].sum()).item())
    return float((v * v).sum().item())


def step_gradient(sens, bits, ranges):
    """dE[dL^2]/dDelta_i = sens_i Delta_i / 6 with Delta_i = R_i / 2^(b_i-1)."""
    delta = np.asarray(ranges, dtype=np.float64) / 2.0 ** (np.asarray(bits, dtype=np.float64) - 1)
    return np.asarray(sens) * delta / 6.0


def group_fields_3d(v):
    """Per-slot values of a 3D F record grouped into 12 fields: x, v
    components, then the rows of C and of F."""
    v = np.asarray(v)
    return np.concatenate([v[0:3], v[3:6], v[6:15].reshape(3, 3).sum(1), v[15:24].reshape(3, 3).sum(1)])
