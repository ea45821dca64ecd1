"""Mesh voxelizer of the particle emitters (mpm_exps/engine/voxelizer.py).

`Voxelizer(res, dx, super_sample=2, padding=3)` keeps the reference's
geometry: every axis of `res` is rounded up to a power of two and multiplied
by `super_sample`, the voxel spacing is dx / super_sample.  `voxelize`
runs the library's CUDA voxelizer (`aq_voxelize`) and leaves the voxel
counts in `self.voxels`, a CUDA int32 tensor (> 0: inside).
"""
import ctypes as C

import numpy as np

from . import _lib


def _pow2_at_least(n):
    r = 1
    while r < n:
        r *= 2
    return r


class Voxelizer:
    def __init__(self, res, dx, super_sample=2, precision="f64", padding=3):
        """voxelizer.py:17-40.  Arithmetic is double precision; precision
        "f32" only selects the reference's larger vertex jitter (1e-4)."""
        if len(res) != 3:
            raise ValueError("the voxelizer is 3D")
        if precision not in ("f32", "f64"):
            raise ValueError("precision must be 'f32' or 'f64'")
        self.res = tuple(_pow2_at_least(int(r)) * super_sample for r in res)
        self.dx = dx / super_sample
        self.inv_dx = 1 / self.dx
        self.precision = precision
        self.padding = int(padding)
        self.jitter_scale = 1e-4 if precision == "f32" else 1e-8
        self.voxels = None

    def voxelize(self, triangles):
        """voxelize (voxelizer.py:107-119): triangles is an n x 9 array of
        corners a, b, c.  Returns the CUDA int32 voxel tensor."""
        import torch

        tris = np.asarray(triangles)
        if tris.ndim != 2 or tris.shape[1] != 9:
            raise ValueError("triangles must be n x 9")
        tris = tris.astype(np.float64)
        if self.precision == "f32":
            tris = tris.astype(np.float32).astype(np.float64)
        d_tris = torch.from_numpy(np.ascontiguousarray(tris)).cuda()
        if self.voxels is None:
            self.voxels = torch.empty(self.res, dtype=torch.int32, device="cuda")
        res = (C.c_int32 * 3)(*self.res)
        _lib.check(_lib.lib().aq_voxelize(C.c_void_p(d_tris.data_ptr()), len(tris), res, self.dx, self.padding,
                                          self.jitter_scale, C.c_void_p(self.voxels.data_ptr()), _lib.stream_ptr()),
                   "aq_voxelize")
        torch.cuda.current_stream().synchronize()
        return self.voxels
