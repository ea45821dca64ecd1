"""autoquantizer_b200: the quantized MLS-MPM substep of AutoQuantizer
(mpm_exps/engine/mpm_solver.py) on NVIDIA B200, as hand-written sm_100a CUDA
behind the C ABI of include/aq.h (libaq.so), with the reference's
simulator / config / quantization-scheme API on top.
"""
from . import _lib, quant, solvers  # noqa: F401
from .mpm_config import MPMConfig  # noqa: F401
from .solvers import LagrangianCR, LagrangianEB, ScipySolver, ScipySolverMemMode  # noqa: F401


def MPMSolver(*args, **kwargs):
    from .mpm_solver import MPMSolver as _S

    return _S(*args, **kwargs)


__all__ = ["MPMConfig", "MPMSolver", "LagrangianCR", "LagrangianEB", "ScipySolver", "ScipySolverMemMode",
           "quant", "solvers"]
