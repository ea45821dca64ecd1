"""ORACLE - test infrastructure only.

ctypes front end of oracle/_build/libaqoracle.so, the CPU restatement of the
reference's bit_pack codec and MLS-MPM substep (see aq_oracle.h for the
reference file:line list).  Only tests/, __graft_entry__.smoke() and the CPU
baseline legs of bench.py import this module; the product never does.

Scalar specs are plain tuples (kind, bits, signed, exp_bits, group, range,
offset) with kind codes FIXED=0, INT=1, FLOAT_EXP=2, SHARED_EXP=3,
RAW_F32=4, RAW_F64=5, so this module does not depend on the product package.
"""
import ctypes as C
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import build as _build  # noqa: E402

MAXS = 32
MAXG = 4


class OrLayout(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("n_words", C.c_int), ("total_bits", C.c_int),
        ("compute_f64", C.c_int), ("dither", C.c_int), ("n_groups", C.c_int),
        ("kind", C.c_int * MAXS), ("bits", C.c_int * MAXS), ("sgn", C.c_int * MAXS),
        ("ebits", C.c_int * MAXS), ("off", C.c_int * MAXS), ("eoff", C.c_int * MAXS),
        ("group", C.c_int * MAXS), ("efirst", C.c_int * MAXS),
        ("scale", C.c_double * MAXS), ("offset", C.c_double * MAXS),
    ]


class OrParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("precision", C.c_int), ("res", C.c_int * 3), ("has_F", C.c_int),
        ("has_mat", C.c_int), ("n_mat", C.c_int), ("friction", C.c_int), ("bound_clip", C.c_int),
        ("dx", C.c_double), ("dt", C.c_double), ("p_vol", C.c_double), ("p_mass", C.c_double),
        ("g", C.c_double), ("lb", C.c_double * 3), ("ub", C.c_double * 3),
        ("mat_kind", C.c_int * 4), ("mat_mu", C.c_double * 4), ("mat_lam", C.c_double * 4),
        ("seed", C.c_uint64), ("threads", C.c_int),
        ("col_on", C.c_int), ("col_n", C.c_int), ("col_dims", C.c_int * 3), ("col_off", C.c_int * 3),
        ("col_yshift", C.c_int), ("col_c", C.c_double), ("col_s", C.c_double), ("col_omega", C.c_double),
        ("col_sdf", C.c_void_p), ("col_nrm", C.c_void_p), ("col_node_cv", C.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        up = C.POINTER(C.c_uint64)
        L.or_layout_build.argtypes = [C.c_int, ip, ip, ip, ip, ip, dp, dp, C.c_int, C.c_int,
                                      C.POINTER(OrLayout)]
        L.or_encode.argtypes = [C.POINTER(OrLayout), dp, up, C.c_int64, C.c_void_p, C.c_uint64,
                                C.c_int64, C.c_void_p]
        L.or_decode.argtypes = [C.POINTER(OrLayout), up, dp, C.c_int64]
        L.or_step_key.argtypes = [C.c_uint64, C.c_int64]
        L.or_step_key.restype = C.c_uint64
        L.or_particle_key.argtypes = [C.c_uint64, C.c_int32]
        L.or_particle_key.restype = C.c_uint64
        L.or_uniform_f32.argtypes = [C.c_uint64, C.c_int]
        L.or_uniform_f32.restype = C.c_float
        L.or_uniform_f64.argtypes = [C.c_uint64, C.c_int]
        L.or_uniform_f64.restype = C.c_double
        for suf in ("f32", "f64"):
            f = getattr(L, "or_substep_" + suf)
            f.argtypes = [C.POINTER(OrParams), C.POINTER(OrLayout), up, C.c_void_p, C.c_int64,
                          C.c_int64, C.c_void_p, dp, C.c_void_p, C.c_void_p]
            f.restype = C.c_int
            g = getattr(L, "or_loss_ek_" + suf)
            g.argtypes = [C.POINTER(OrParams), C.POINTER(OrLayout), up, C.c_int64]
            g.restype = C.c_double
        L.or_voxelize.argtypes = [dp, C.c_int64, C.POINTER(C.c_int32), C.c_double, C.c_int32, C.c_double,
                                  C.POINTER(C.c_int32)]
        L.or_voxelize.restype = None
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def build_layout(specs, compute_f64=False, dither=False):
    """specs: list of (kind, bits, signed, exp_bits, group, range, offset)."""
    n = len(specs)
    cols = list(zip(*specs))
    kind, bits, sgn, eb, grp = (np.ascontiguousarray(c, dtype=np.int32) for c in cols[:5])
    rng, off = (np.ascontiguousarray(c, dtype=np.float64) for c in cols[5:7])
    L = OrLayout()
    rc = lib().or_layout_build(n, _ptr(kind, C.c_int), _ptr(bits, C.c_int), _ptr(sgn, C.c_int),
                               _ptr(eb, C.c_int), _ptr(grp, C.c_int), _ptr(rng, C.c_double),
                               _ptr(off, C.c_double), int(compute_f64), int(dither), C.byref(L))
    if rc != 0:
        raise ValueError("oracle: invalid layout")
    return L


def encode(L, values, pid=None, seed=0, step=0, uniforms=None):
    v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1, L.n)
    n = v.shape[0]
    w = np.zeros((n, L.n_words), dtype=np.uint64)
    p = None if pid is None else np.ascontiguousarray(pid, dtype=np.int32)
    u = None if uniforms is None else np.ascontiguousarray(uniforms, dtype=np.float64).reshape(n, L.n)
    lib().or_encode(C.byref(L), _ptr(v, C.c_double), _ptr(w, C.c_uint64), n,
                    None if p is None else p.ctypes.data, C.c_uint64(seed), step,
                    None if u is None else u.ctypes.data)
    return w


def decode(L, words):
    w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1, L.n_words)
    out = np.zeros((w.shape[0], L.n), dtype=np.float64)
    lib().or_decode(C.byref(L), _ptr(w, C.c_uint64), _ptr(out, C.c_double), w.shape[0])
    return out


def uniform(seed, step, pid, slot, f64=False):
    pk = lib().or_particle_key(lib().or_step_key(C.c_uint64(seed), step), pid)
    return lib().or_uniform_f64(pk, slot) if f64 else lib().or_uniform_f32(pk, slot)


def voxelize(triangles, res, dx, padding=3, jitter_scale=1e-8):
    """Voxel counts of n x 9 triangles on a res voxel grid of spacing dx
    (aq_oracle_emit.c, restating voxelizer.py:53-105)."""
    t = np.ascontiguousarray(triangles, dtype=np.float64).reshape(-1, 9)
    out = np.zeros(tuple(res), dtype=np.int32)
    r = (C.c_int32 * 3)(*res)
    lib().or_voxelize(_ptr(t, C.c_double), len(t), r, float(dx), int(padding), float(jitter_scale),
                      _ptr(out, C.c_int32))
    return out


class Sim:
    """CPU oracle simulator over packed records (particle order = index)."""

    def __init__(self, params: dict, layout: OrLayout, threads=1):
        P = OrParams()
        P.dim = params["dim"]
        P.precision = params.get("precision", 0)
        for k in range(3):
            P.res[k] = params["res"][k] if k < len(params["res"]) else 1
            P.lb[k] = params["lb"][k] if k < len(params["lb"]) else 0
            P.ub[k] = params["ub"][k] if k < len(params["ub"]) else 0
        P.has_F = int(params["has_F"])
        P.has_mat = int(params.get("has_mat", 0))
        mats = params["materials"]
        P.n_mat = len(mats)
        for i, (k, mu, lam) in enumerate(mats):
            P.mat_kind[i], P.mat_mu[i], P.mat_lam[i] = k, mu, lam
        P.friction = int(params.get("use_friction", 0))
        P.bound_clip = int(params.get("use_bound_clip", 0))
        P.dx, P.dt, P.p_vol, P.p_mass, P.g = (params[k] for k in ("dx", "dt", "p_vol", "p_mass", "gravity"))
        P.seed = params.get("seed", 0)
        P.threads = threads
        self.P, self.L = P, layout
        ncell = int(np.prod(params["res"][: P.dim]))
        self.grid = np.zeros(ncell * 4, dtype=np.float64 if P.precision else np.float32)
        self.words = None
        self.pid = None
        self.step = 0
        self.flags = 0
        self.rmax = np.full(layout.n, -np.inf)
        self.rmin = np.full(layout.n, np.inf)

    def set_state(self, values, step=-1):
        v = np.asarray(values, dtype=np.float64)
        self.pid = np.arange(v.shape[0], dtype=np.int32)
        self.words = encode(self.L, v, self.pid, self.P.seed, step)

    def set_words(self, words):
        self.words = np.ascontiguousarray(words, dtype=np.uint64).copy()
        self.pid = np.arange(self.words.shape[0], dtype=np.int32)

    def get_state(self):
        return decode(self.L, self.words)

    def set_collider(self, sdf, normal, offset, center, theta=0.0, height=0.0, omega=5.0, height_rate=0.1,
                     node_velocity=False):
        """The rotating SDF collider (float32 volumes sdf [a,b,c], normal
        [a,b,c,3] placed at grid index offset); angle and height advance by
        omega dt and height_rate dt after every substep.  node_velocity:
        collider velocity from the node itself (sdf_collision_no_arg)."""
        self._col = (np.ascontiguousarray(sdf, dtype=np.float32), np.ascontiguousarray(normal, dtype=np.float32))
        self.P.col_on = 1
        self.P.col_n = int(center)
        for k in range(3):
            self.P.col_dims[k] = self._col[0].shape[k]
            self.P.col_off[k] = int(offset[k])
        self.P.col_sdf = self._col[0].ctypes.data
        self.P.col_nrm = self._col[1].ctypes.data
        self.P.col_omega = float(omega)
        self.P.col_node_cv = int(bool(node_velocity))
        self.col_theta, self.col_height, self.col_rate = float(theta), float(height), float(height_rate)

    def _collider_step_values(self):
        if not getattr(self.P, "col_on", 0):
            return
        self.P.col_c = math.cos(self.col_theta)
        self.P.col_s = math.sin(self.col_theta)
        if not self.P.precision:  # the f32 simulator carries them as float
            self.P.col_c = float(np.float32(self.P.col_c))
            self.P.col_s = float(np.float32(self.P.col_s))
        self.P.col_yshift = int(self.col_height / self.P.dx + 0.5)

    def substeps(self, k, ranges=False):
        f = lib().or_substep_f64 if self.P.precision else lib().or_substep_f32
        n = self.words.shape[0]
        scratch = np.zeros(n * self.L.n, dtype=np.float64)
        for _ in range(k):
            self._collider_step_values()
            self.flags |= f(C.byref(self.P), C.byref(self.L), _ptr(self.words, C.c_uint64),
                            self.pid.ctypes.data, n, self.step, self.grid.ctypes.data,
                            _ptr(scratch, C.c_double),
                            self.rmax.ctypes.data if ranges else None,
                            self.rmin.ctypes.data if ranges else None)
            self.step += 1
            if self.P.col_on:
                self.col_theta += self.P.col_omega * self.P.dt
                self.col_height += self.col_rate * self.P.dt

    def loss(self):
        f = lib().or_loss_ek_f64 if self.P.precision else lib().or_loss_ek_f32
        return f(C.byref(self.P), C.byref(self.L), _ptr(self.words, C.c_uint64), self.words.shape[0])
