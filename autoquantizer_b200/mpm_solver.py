"""MPMSolver: drop-in for the reference simulator's hot path.

Keeps the method names and semantics of mpm_exps/engine/mpm_solver.py
(MPMSolver, :17-1912) that the experiment drivers call: initialize,
add_cube, substep, run_forward_only, compute_loss / loss, set_bits_and_ranges,
reshape_params, detect_bound / get_limits, fetch_data_np / push_data_np.
The substep itself runs in libaq.so (sm_100a kernels behind include/aq.h);
this module only builds the record layout and moves buffers.  PyTorch is used
for device buffers and the current stream.
"""
import ctypes as C
import os

import numpy as np

from . import _lib
from . import quant as Q

FIELD_NAMES = ("x", "v", "C", "F", "J")


class _Loss:
    """Stand-in for the reference's `loss` field: loss[None]."""

    def __init__(self):
        self.value = 0.0

    def __getitem__(self, k):
        return self.value

    def __setitem__(self, k, v):
        self.value = float(v)


def lame(E, nu, softer=False):
    mu = E / (2 * (1 + nu))
    la = E * nu / ((1 + nu) * (1 - 2 * nu))
    if softer:
        mu, la = mu * 0.3, la * 0.3
    return mu, la


class MPMSolver:
    def __init__(self, mpm_param):
        self.param = p = mpm_param
        self.dim = p.dim
        self.n_timestep = int(p.n_timesteps)
        self.n_particles, self.n_grid = int(p.n_particles), p.n_grid
        self.dx = 1 / self.n_grid
        self.inv_dx = 1.0 / self.dx
        self.p_rho, self.p_vol = p.p_rho, p.p_vol
        self.p_mass = self.p_vol * self.p_rho
        self.la = p.la
        self.E, self.nu = p.E, p.nu
        self.mu_0, self.la_0 = lame(self.E, self.nu, p.softer)
        self.dt, self.steps, self.g = p.dt, p.steps, p.g
        self.use_fluid = p.use_fluid
        self.use_quantaichi = p.use_quantaichi
        self.use_difftaichi = p.use_difftaichi
        self.use_bitpack = p.use_bitpack
        self.use_dithering = p.use_dithering
        self.use_bound_clip = p.use_bound_clip
        self.use_friction = p.use_friction
        self.size = p.size
        self.bound = list(p.bound) if p.bound is not None else [3] * self.dim
        self.offset = [0] * self.dim
        # mpm_solver.py:97-105
        self.lb = [b + o for b, o in zip(self.bound, self.offset)]
        self.ub = [self.n_grid * self.size - b for b in self.bound]
        if p.ub is not None:
            self.ub = list(p.ub)
        if p.lb is not None:
            self.lb = list(p.lb)
        if p.quant_bits is not None:
            self.bits = self.reshape_params(p.quant_bits)
            self.ranges = self.reshape_params(p.quant_ranges)
        self.loss = _Loss()
        self.current_idx = 0
        self._host = None  # staged particle values (n x n_slots, float64)
        self._sim = None
        self._dirty = True
        self._layout = None
        self.materials = p.materials
        self._col = None  # SDF collider: (sdf, normal) CUDA tensors, offset, motion state
        self._vox = None  # mesh voxelizer of add_mesh, made on first use
        self.initialize()

    # ------------------------------------------------------------ layout

    @property
    def has_F(self):
        return not self.use_fluid

    @property
    def has_mat(self):
        return bool(self.materials)

    def n_slots(self):
        d = self.dim
        return 2 * d + d * d + (d * d if self.has_F else 1) + (1 if self.has_mat else 0)

    def slot_range(self, name):
        d = self.dim
        return {"x": (0, d), "v": (d, 2 * d), "C": (2 * d, 2 * d + d * d),
                "F": (2 * d + d * d, 2 * d + 2 * d * d), "J": (2 * d + d * d, 2 * d + d * d + 1),
                "mat": (self.n_slots() - 1, self.n_slots())}[name]

    def record(self):
        """The particle record as a BitPack, in the reference's place order
        x, v, C, F|J (init_quantaichi, mpm_solver.py:364-455)."""
        p, d = self.param, self.dim
        rec = Q.BitPack()
        qp = p.quantized_properties or {}
        if not self.use_quantaichi:
            raw = Q.Raw(f64=(p.precision == "f64"))
            rec.place(*[raw] * (self.n_slots() - (1 if self.has_mat else 0)))
        else:
            comp = "f32" if p.compute_fp == "f32" else "f64"
            bits = [int(b) for b in np.asarray(p.quant_bits).ravel()]
            rngs = [float(r) for r in np.asarray(p.quant_ranges).ravel()]
            nfj = d * d if self.has_F else 1
            if len(bits) != 2 * d + d * d + nfj:
                raise ValueError("quant_bits must list x, v, C and F|J scalars (%d)" % (2 * d + d * d + nfj))

            def fx(i, offset=0.0):
                return Q.fixed(bits[i], True, rngs[i], offset, comp, p.use_dithering)

            rec.place(*[fx(i) for i in range(d)])
            if p.v_exp_bits:
                rec.place(*[Q.qfloat(bits[d + i], p.v_exp_bits, True) for i in range(d)], shared_exponent=True)
            else:
                rec.place(*[fx(d + i) for i in range(d)])
            if "C" in qp or not qp:
                rec.place(*[fx(2 * d + i) for i in range(d * d)])
            else:
                rec.place(*[Q.Raw(f64=(p.precision == "f64"))] * (d * d))
            if self.has_F:
                rec.place(*[fx(2 * d + d * d + i) for i in range(d * d)])
            else:
                rec.place(fx(2 * d + d * d, offset=1.0))
        if self.has_mat:
            rec.place(Q.qint(max(1, int(np.ceil(np.log2(max(2, len(self.materials)))))), False))
        return rec

    def layout(self):
        if self._layout is None:
            self._layout = self.record().build()
        return self._layout

    def bytes_per_particle(self):
        return 8 * self.layout().n_words

    def _params(self):
        p, d = self.param, self.dim
        P = _lib.Params()
        P.dim = d
        P.precision = 1 if p.precision == "f64" else 0
        res = p.grid_res if p.grid_res is not None else [int(round(self.n_grid * self.size))] * d
        for k in range(3):
            P.res[k] = int(res[k]) if k < d else 1
            P.lb[k] = float(self.lb[k]) if k < d else 0.0
            P.ub[k] = float(self.ub[k]) if k < d else 0.0
        P.has_F = int(self.has_F)
        P.has_mat = int(self.has_mat)
        if self.has_mat:
            P.n_materials = len(self.materials)
            for i, (kind, E, nu, la) in enumerate(self.materials):
                mu, lam = lame(E, nu, p.softer)
                P.mat[i].kind = kind
                P.mat[i].mu, P.mat[i].lam = (0.0, la) if kind == _lib.AQ_MAT_FLUID else (mu, lam)
        else:
            P.n_materials = 1
            if self.use_fluid:
                P.mat[0].kind, P.mat[0].mu, P.mat[0].lam = _lib.AQ_MAT_FLUID, 0.0, self.la
            else:
                P.mat[0].kind, P.mat[0].mu, P.mat[0].lam = _lib.AQ_MAT_ELASTIC, self.mu_0, self.la_0
        P.use_friction = int(self.use_friction)
        P.use_bound_clip = int(self.use_bound_clip)
        P.sort_interval = int(p.sort_interval)
        P.jit = int(getattr(p, "jit", True))
        P.sparse = int(bool(getattr(p, "sparse_grid", False)))
        P.dx, P.dt, P.p_vol, P.p_mass, P.gravity = self.dx, self.dt, self.p_vol, self.p_mass, self.g
        P.n_particles = self.current_idx
        P.seed = int(p.seed)
        return P

    # ----------------------------------------------------- scene set-up

    def initialize(self):
        """mpm_solver.py:564-576: F = I (or J = 1), C = 0, no particles."""
        self._host = None  # built on first use (_staging)
        self._dev = None
        self.current_idx = 0
        self.loss[None] = 0.0
        self._drop_sim()

    def _staging(self):
        """Host staging array (n_particles x n_slots, float64), created on
        first use with F = I (or J = 1); holds device-provided initial values
        once something needs them on the host."""
        if self._host is None:
            n, d = self.n_particles, self.dim
            h = np.zeros((n, self.n_slots()), dtype=np.float64)
            a, b = self.slot_range("F" if self.has_F else "J")
            if self.has_F:
                h[:, a:b] = np.eye(d).ravel()
            else:
                h[:, a] = 1.0
            if self._dev is not None:
                h[: self._dev.shape[0]] = self._dev.double().cpu().numpy()
            self._host = h
        return self._host

    def _drop_sim(self):
        # the running ranges outlive the simulator (the reference keeps its
        # limit fields for the solver's lifetime, across emissions): fold the
        # device's into the host-side maxima first
        if self._sim is not None and getattr(self, "_ranges_on_device", False):
            ns = self.n_slots()
            mx = (C.c_double * ns)()
            mn = (C.c_double * ns)()
            if _lib.lib().aq_sim_ranges_get(self._sim, mx, mn, _lib.stream_ptr()) == 0:
                cur = np.maximum(np.abs(np.array(mx[:])), np.abs(np.array(mn[:])))
                cur[~np.isfinite(cur)] = 0.0
                h = getattr(self, "_rabs_host", None)
                self._rabs_host = cur if h is None else np.maximum(h, cur)
        self._ranges_on_device = False
        if self._sim is not None:
            if self._col is not None:  # carry the collider's angle and height over
                th, hh = C.c_double(), C.c_double()
                _lib.lib().aq_sim_collider_get(self._sim, C.byref(th), C.byref(hh))
                self._col["theta"], self._col["height"] = th.value, hh.value
            _lib.lib().aq_sim_destroy(self._sim)
            self._sim = None
        self._dirty = True

    def _pull(self):
        """Copy the simulator's state back into the host staging array."""
        if self._sim is not None and not self._dirty:
            self._staging()[: self.current_idx] = self.state_values()
            self._dev = None

    def _rng(self, tag):
        return np.random.default_rng((int(self.param.seed), self.current_idx, tag))

    def _append(self, x, v=None, material=0, what="add"):
        """New particles at current_idx: positions x (cnt x dim), velocity v
        (a dim vector or cnt x dim, default 0), F = I or J = 1, C = 0.  With
        a simulator running, they are encoded on the device behind the
        stored records (aq_sim_append), which stay as they are, as the
        reference's emitters write only the new particles; otherwise they
        go into the host staging array the next simulator starts from."""
        x = np.asarray(x, dtype=np.float64).reshape(-1, self.dim)
        st, cnt = self.current_idx, len(x)
        if st + cnt > self.n_particles:
            raise ValueError("%s: %d particles exceed n_particles=%d" % (what, st + cnt, self.n_particles))
        rows = np.zeros((cnt, self.n_slots()), dtype=np.float64)
        a, b = self.slot_range("x")
        rows[:, a:b] = x
        va, vb = self.slot_range("v")
        if v is not None:
            rows[:, va:vb] = np.broadcast_to(np.asarray(v, dtype=np.float64), (cnt, self.dim))
        fa, fb = self.slot_range("F" if self.has_F else "J")
        rows[:, fa:fb] = np.eye(self.dim).ravel() if self.has_F else 1.0
        if self.has_mat:
            rows[:, self.slot_range("mat")[0]] = material
        if cnt == 0:
            return 0
        if self._sim is not None and not self._dirty:
            import torch

            t = torch.from_numpy(rows).cuda()
            _lib.check(_lib.lib().aq_sim_append(self._sim, C.c_void_p(t.data_ptr()), 1, cnt, _lib.stream_ptr()),
                       "aq_sim_append")
            torch.cuda.current_stream().synchronize()
            self.current_idx = st + cnt
            return cnt
        self._pull()
        h = self._staging()
        self._dev = None
        h[st:st + cnt] = rows
        self.current_idx = st + cnt
        self._drop_sim()
        return cnt

    def add_cube(self, low_corner, box_size, num, material=0):
        """3D: uniform random positions (fill_in_box, :1573-1590), pushed out
        of the SDF collider when one is set; 2D: the deterministic lattice of
        fill_in_box_2duniform (:1561-1571)."""
        d = self.dim
        if d == 3 or len(low_corner) == 3:
            rng = self._rng(0)
            x = np.asarray(low_corner)[None, :] + rng.random((num, d)) * np.asarray(box_size)[None, :]
            if self._col is not None:
                x = self._push_out_of_collider(x, rng)
        else:
            n = int(np.sqrt(num))
            i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
            x = np.stack([low_corner[0] + 1.0 / n * j.ravel() * box_size[0],
                          low_corner[1] + 1.0 / n * i.ravel() * box_size[1]], axis=1)
        self._append(x, None, material, "add_cube")

    def _push_out_of_collider(self, x, rng):
        """fill_in_box with the collider (mpm_solver.py:1582-1588): a particle
        whose cell int(x / dx + 0.5), rotated into the collider's frame
        (rot_scene, :1518-1540), lies inside (sdf < -1e-5) moves along the
        stored normal by (2 + 3 u) dx."""
        c = self._col
        theta, height = self.collider_state()
        sdf, nrm = c["sdf"].cpu().numpy(), c["normal"].cpu().numpy()
        n = int(self.n_grid)
        base = (x / self.dx + 0.5).astype(np.int64)
        i0 = np.where(base[:, 0] >= 2 * n, base[:, 0] - 2 * n, base[:, 0])
        i2 = np.where(base[:, 2] >= 2 * n, base[:, 2] - 2 * n, base[:, 2])
        cs, sn = np.cos(-theta), np.sin(-theta)
        o0, o2 = (i0 - n).astype(np.float64), (i2 - n).astype(np.float64)
        r = np.stack([(cs * o0 + sn * o2 + n + 0.5).astype(np.int64), base[:, 1] - int(height / self.dx + 0.5),
                      (-sn * o0 + cs * o2 + n + 0.5).astype(np.int64)], axis=1)
        r = np.clip(r, np.asarray(self.lb, dtype=np.int64), np.asarray(self.ub, dtype=np.int64))
        q = r - np.asarray(c["offset"])
        ok = np.all((q >= 0) & (q < np.asarray(sdf.shape)), axis=1)
        inside = np.zeros(len(x), dtype=bool)
        inside[ok] = sdf[q[ok, 0], q[ok, 1], q[ok, 2]] < -1e-5
        u = rng.random(len(x))
        x = x.copy()
        g = nrm[q[inside, 0], q[inside, 1], q[inside, 2]]
        x[inside] += g * ((u[inside] * 3 + 2) * self.dx)[:, None]
        return x

    def add_ball(self, center, radius, num, material=0):
        """fill_in_ball (mpm_solver.py:1592-1598, 1620-1627): uniform points
        in the ball by rejection, at rest.  As in the reference, nothing is
        added unless current_idx + num < n_particles."""
        if self.current_idx + num >= self.n_particles:
            return 0
        rng = self._rng(1)
        pts = np.empty((0, self.dim))
        while len(pts) < num:
            p = rng.random((2 * num + 16, self.dim)) * 2 - 1
            pts = np.concatenate([pts, p[(p * p).sum(1) <= 1]])
        return self._append(np.asarray(center)[None, :] + pts[:num] * radius, None, material, "add_ball")

    def emit_water(self, center, radius, velocity, num, material=0):
        """fill_in_ball_with_vel (mpm_solver.py:1600-1618, 1629-1632): points
        at angle 2 pi u1 and distance radius u2 from the centre in the xy
        plane, all moving with velocity; nothing is added unless
        current_idx + num < n_particles."""
        if self.current_idx + num >= self.n_particles:
            return 0
        rng = self._rng(2)
        th, r = rng.random(num) * np.pi * 2.0, rng.random(num)
        off = np.zeros((num, self.dim))
        off[:, 0], off[:, 1] = np.cos(th) * r, np.sin(th) * r
        x = np.asarray(center[:self.dim], dtype=np.float64)[None, :] + off * radius
        return self._append(x, velocity[:self.dim], material, "emit_water")

    # mesh emitters (3D)

    def _voxelizer(self):
        if self.dim != 3:
            raise ValueError("mesh emitters are 3D")
        if self._vox is None:
            from .voxelizer import Voxelizer

            self.voxelizer_super_sample = 2
            self._vox = Voxelizer(res=(self.n_grid,) * 3, dx=self.dx, super_sample=self.voxelizer_super_sample)
        return self._vox

    @property
    def voxelizer(self):
        return self._voxelizer()

    def add_mesh(self, triangles, material=None, color=0xFFFFFF, sample_density=None, velocity=None,
                 translation=None, s=0):
        """add_mesh (mpm_solver.py:1356-1376): voxelize the triangles, then
        seed sample_density + 1 particles per inside voxel."""
        if sample_density is None:
            sample_density = 2 ** self.dim
        self._voxelizer().voxelize(triangles)
        return self.add_particles_from_voxels(sample_density, translation, velocity, s,
                                              material if isinstance(material, int) else 0)

    def cnt_mesh_particles_num(self, triangles, material=None, color=0xFFFFFF, sample_density=None, velocity=None,
                               translation=None):
        """Particles add_mesh would emit (mpm_solver.py:1382-1400)."""
        if sample_density is None:
            sample_density = 2 ** self.dim
        vox = self._voxelizer().voxelize(triangles)
        return int((vox > 0).sum()) * (sample_density + 1)

    def add_particles_from_voxels(self, sample_density, translation=None, velocity=None, s=0, material=0):
        """seed_from_voxels (mpm_solver.py:1415-1440): for every voxel (i, j,
        k) with a positive count, sample_density + 1 particles at
        (u + (i, j, k)) dx + translation with the given velocity.  dx is the
        simulation grid's spacing, not the voxel's, as in the reference.
        Particles are appended in voxel order (row-major), then sample."""
        import torch

        vox = self._voxelizer().voxels
        # inside voxels in row-major order, found on the device (the voxel
        # grid is up to 2 x 2^k per axis; only the indices come back)
        idx = torch.nonzero(vox > 0).cpu().numpy().astype(np.float64)
        k = int(sample_density) + 1
        rng = self._rng(3)
        x = (rng.random((len(idx), k, 3)) + idx[:, None, :]) * self.dx
        x = x.reshape(-1, 3) + np.asarray([0.0, 0.0, 0.0] if translation is None else list(translation))
        v = np.zeros(3) if velocity is None else np.asarray(list(velocity), dtype=np.float64)
        return self._append(x, v, material, "add_mesh")

    def set_emit_data(self, data):
        """Positions the letters emitter places (mpm_solver.py:124-128)."""
        self._emit_data = np.asarray(data, dtype=np.float64).reshape(-1, self.dim)

    def emit_letters_one_frame(self, velocity=(0.0, -2.0, 0.0)):
        """emit_letters_one_frame (mpm_solver.py:130-135): the set_emit_data
        positions, moving with velocity (0, -2, 0)."""
        if getattr(self, "_emit_data", None) is None:
            raise ValueError("set_emit_data first")
        return self._append(self._emit_data, np.asarray(velocity[:self.dim]), 0, "emit_letters_one_frame")

    def set_particles(self, values):
        """Set all active particles from an (n x n_slots) array: numpy (host),
        or a CUDA float32/float64 tensor, which the simulator then encodes
        straight from device memory."""
        if getattr(values, "is_cuda", False):
            if values.dim() != 2 or values.shape[1] != self.n_slots() or values.shape[0] > self.n_particles:
                raise ValueError("set_particles: expected (<= %d) x %d values" % (self.n_particles, self.n_slots()))
            self._dev = values.contiguous()
            self._host = None
            self.current_idx = values.shape[0]
            self._drop_sim()
            return
        v = np.asarray(values, dtype=np.float64)
        self._staging()[: v.shape[0]] = v
        self._dev = None
        self.current_idx = v.shape[0]
        self._drop_sim()

    # ------------------------------------------------------------ running

    def _ensure_sim(self):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("MPMSolver needs a CUDA device (sm_100a); there is no CPU fallback")
        if self._sim is not None and not self._dirty:
            return
        if self._sim is None:
            # room for n_particles records (the emitters append on the
            # device), current_idx of them active
            P = self._params()
            P.n_particles = max(int(self.n_particles), int(self.current_idx))
            sim = C.c_void_p()
            _lib.check(_lib.lib().aq_sim_create(C.byref(P), C.byref(self.layout()), C.byref(sim)), "aq_sim_create")
            self._sim = sim
            if self.current_idx < P.n_particles:
                _lib.check(_lib.lib().aq_sim_set_count(self._sim, int(self.current_idx)), "aq_sim_set_count")
            if self._col is not None:
                self._apply_collider()
        if self._dev is not None and self._host is None:
            vals = self._dev
            if vals.dtype not in (torch.float32, torch.float64):
                vals = vals.double()
        else:
            vals = torch.from_numpy(np.ascontiguousarray(self._staging()[: self.current_idx])).cuda()
        _lib.check(_lib.lib().aq_sim_set_state(self._sim, C.c_void_p(vals.data_ptr()),
                                               int(vals.dtype == torch.float64), _lib.stream_ptr()),
                   "aq_sim_set_state")
        torch.cuda.current_stream().synchronize()
        self._dirty = False

    def substeps(self, n):
        """n forward substeps (substep, mpm_solver.py:624-631), the collider
        (when set) as sdf_collision and advanced after every substep."""
        self._ensure_sim()
        self._collider_velocity_from_node(False)
        _lib.check(_lib.lib().aq_sim_substeps(self._sim, int(n), _lib.stream_ptr()), "aq_sim_substeps")

    def substep(self, s=0, t=None):
        """One substep (mpm_solver.py:624-631)."""
        self.substeps(1)

    def _substep_difftaichi_form(self):
        """One substep with the autodiff path's collider (sdf_collision_no_arg:
        collider velocity from the node itself)."""
        self._ensure_sim()
        self._collider_velocity_from_node(True)
        _lib.check(_lib.lib().aq_sim_substeps(self._sim, 1, _lib.stream_ptr()), "aq_sim_substeps")

    def run_forward_only(self, save_pics=False, save_states=False):
        """run_forward_only of the drivers (run_mpm_elastic_2d.py:124-162):
        n_timestep-1 substeps, then the loss; with save_states the positions
        are dumped after every frame of `steps` substeps (dump_states)."""
        total = self.n_timestep - 1
        if not save_states:
            self.substeps(total)
        else:
            s, frame = 0, 0
            while s < total:
                k = min(int(self.param.steps), total - s)
                self.substeps(k)
                s += k
                self.dump_states(frame)
                frame += 1
        self.compute_loss()
        return self.loss[None]

    def compute_loss(self):
        self._ensure_sim()
        out = C.c_double()
        _lib.check(_lib.lib().aq_sim_loss(self._sim, 0, C.byref(out), _lib.stream_ptr()), "aq_sim_loss")
        self.loss[None] = out.value
        return out.value

    def field_stats(self, reference=None):
        """Per-slot statistics of the current state on the device
        (aq_sim_field_stats): an (n_slots x 5) array of sum |v|, sum v,
        sum v^2, max |v| and sum |v - reference| (reference: a CUDA tensor of
        initial values in particle order, or None)."""
        import torch

        self._ensure_sim()
        ns = self.n_slots()
        out = (C.c_double * (5 * ns))()
        if reference is not None:
            if not reference.is_cuda or reference.dtype not in (torch.float32, torch.float64) or \
                    tuple(reference.shape) != (self.current_idx, ns) or not reference.is_contiguous():
                raise ValueError("field_stats: reference must be a contiguous CUDA float tensor of %d x %d"
                                 % (self.current_idx, ns))
            ref, f64 = C.c_void_p(reference.data_ptr()), int(reference.dtype == torch.float64)
        else:
            ref, f64 = None, 0
        _lib.check(_lib.lib().aq_sim_field_stats(self._sim, ref, f64, out, _lib.stream_ptr()), "aq_sim_field_stats")
        return np.array(out[:]).reshape(ns, 5)

    # ------------------------------------------------------------- state

    def state_values(self, f64=True):
        """Decoded state, particle order, (n x n_slots) numpy array."""
        t = self.state_tensor(f64)
        return t.cpu().numpy()

    def state_tensor(self, f64=True):
        import torch

        self._ensure_sim()
        out = torch.empty((self.current_idx, self.n_slots()), dtype=torch.float64 if f64 else torch.float32,
                          device="cuda")
        _lib.check(_lib.lib().aq_sim_get_state(self._sim, C.c_void_p(out.data_ptr()), int(f64), _lib.stream_ptr()),
                   "aq_sim_get_state")
        return out

    def words(self):
        import torch

        self._ensure_sim()
        out = torch.empty((self.current_idx, self.layout().n_words), dtype=torch.int64, device="cuda")
        _lib.check(_lib.lib().aq_sim_get_words(self._sim, C.c_void_p(out.data_ptr()), _lib.stream_ptr()),
                   "aq_sim_get_words")
        return out.cpu().numpy().view(np.uint64)

    def set_words(self, words):
        import torch

        self._ensure_sim()
        w = torch.from_numpy(np.ascontiguousarray(words).view(np.int64)).cuda()
        _lib.check(_lib.lib().aq_sim_set_words(self._sim, C.c_void_p(w.data_ptr()), _lib.stream_ptr()),
                   "aq_sim_set_words")
        torch.cuda.current_stream().synchronize()

    def fetch_data_np(self, name, parts=10):
        """mpm_solver.py:1782-1830 (x, v: n x dim; C, F: n x dim x dim; J: n)."""
        a, b = self.slot_range(name)
        v = self.state_values()[:, a:b]
        if name in ("C", "F"):
            return v.reshape(-1, self.dim, self.dim).astype(np.float32)
        if name == "J":
            return v[:, 0].astype(np.float32)
        return v.astype(np.float32)

    def push_data_np(self, name, data):
        """mpm_solver.py:1832-1867."""
        self._pull()
        a, b = self.slot_range(name)
        self._staging()[: len(data), a:b] = np.asarray(data, dtype=np.float64).reshape(len(data), b - a)
        self._dev = None
        self._dirty = True
        if self._sim is not None:
            self._ensure_sim()
        return data

    def step_count(self):
        """Substeps run by the simulator (the dithering step index)."""
        if self._sim is None:
            return 0
        v = C.c_int64()
        _lib.check(_lib.lib().aq_sim_step_count(self._sim, C.byref(v)), "aq_sim_step_count")
        return v.value

    def save_checkpoint(self, fn):
        """The packed state as .npz: the records' words in particle order, the
        layout they follow (slot specs), the substep count and the
        collider's angle and height; load_checkpoint resumes from it with
        the same dithering draws as an uninterrupted run."""
        words = self.words()
        col = self.collider_state()
        np.savez_compressed(fn, words=words, n_particles=np.int64(self.current_idx),
                            specs=np.array(self.record().spec_tuples(), dtype=np.float64),
                            step=np.int64(self.step_count()), seed=np.int64(int(self.param.seed)),
                            collider=np.array(col if col is not None else [np.nan, np.nan]))
        return fn

    def load_checkpoint(self, fn):
        """Resume from save_checkpoint's file: the layout must be this
        solver's; the particle count becomes the file's."""
        d = np.load(fn)
        specs = np.array(self.record().spec_tuples(), dtype=np.float64)
        if d["specs"].shape != specs.shape or not np.array_equal(d["specs"], specs):
            raise ValueError("load_checkpoint: the file's record layout differs from this solver's")
        n = int(d["n_particles"])
        if n > self.n_particles:
            raise ValueError("load_checkpoint: %d particles exceed n_particles=%d" % (n, self.n_particles))
        if int(d["seed"]) != int(self.param.seed):
            raise ValueError("load_checkpoint: the file was written with seed %d" % int(d["seed"]))
        self._pull()
        self._staging()
        self._dev = None
        self.current_idx = n
        self._drop_sim()
        col = d["collider"]
        if self._col is not None and np.all(np.isfinite(col)):
            self._col["theta"], self._col["height"] = float(col[0]), float(col[1])
        self.set_words(d["words"])
        self.set_step_count(int(d["step"]))
        if self._col is not None:
            self._apply_collider()

    def set_step_count(self, step):
        """Set the dithering step index (aq_sim_set_step_count)."""
        self._ensure_sim()
        _lib.check(_lib.lib().aq_sim_set_step_count(self._sim, int(step)), "aq_sim_set_step_count")

    fetch_mat_data_np = fetch_data_np
    fetch_scalar_data_np = fetch_data_np
    push_mat_data_np = push_data_np
    push_scalar_data_np = push_data_np

    # ------------------------------------------------------ on-disk formats

    def _out_folder(self):
        folder = self.param.pos_output_folder
        if not folder:
            raise ValueError("pos_output_folder is not set")
        os.makedirs(folder, exist_ok=True)
        return folder

    def dump_states(self, frame):
        """Positions as data_{frame:06d}.ply in pos_output_folder
        (mpm_solver.py:1776-1780); 2D positions get z = 0."""
        from .mesh_io import write_point_cloud_packed

        x = self.fetch_data_np("x")
        if self.dim == 2:
            x = np.concatenate([x, np.zeros((len(x), 1), np.float32)], axis=1)
        fn = os.path.join(self._out_folder(), "data_%06d.ply" % frame)
        write_point_cloud_packed(fn, x, len(x))
        return fn

    def checkpoint_states(self, frame):
        """v.npy, C.npy and J.npy (fluid) or F.npy in pos_output_folder, the
        rest of the state load_states needs (mpm_solver.py:1761-1774)."""
        folder = self._out_folder()
        for name in ("v", "C", "F" if self.has_F else "J"):
            np.save(os.path.join(folder, "%s.npy" % name), self.fetch_data_np(name))
        return folder

    def load_states(self, folder, frame):
        """Particles from data_{frame:06d}.ply plus v.npy, C.npy and F.npy
        or J.npy (mpm_solver.py:1869-1895); the particle count is the file's."""
        from .mesh_io import load_particles_only

        x = load_particles_only(os.path.join(folder, "data_%06d.ply" % frame))[:, :self.dim]
        n = len(x)
        if n > self.n_particles:
            raise ValueError("load_states: %d particles exceed n_particles=%d" % (n, self.n_particles))
        self._pull()  # a running simulator holds the current values (particles appended on the device too)
        vals = np.array(self._staging()[:n], copy=True)
        vals[:, slice(*self.slot_range("x"))] = x
        for name in ("v", "C", "F" if self.has_F else "J"):
            a, b = self.slot_range(name)
            vals[:, a:b] = np.load(os.path.join(folder, "%s.npy" % name)).reshape(n, b - a)
        self.set_particles(vals)

    def grid_mass(self):
        """Node masses of the latest substep's P2G (a res-shaped float32
        CUDA tensor): the grid_m of dump_grid."""
        import torch

        self._ensure_sim()
        out = torch.empty(tuple(self._params().res[:self.dim]), dtype=torch.float32, device="cuda")
        _lib.check(_lib.lib().aq_sim_grid_mass(self._sim, C.c_void_p(out.data_ptr()), _lib.stream_ptr()),
                   "aq_sim_grid_mass")
        return out

    def dump_grid(self, frame, grid_m=None):
        """density_{frame:06d}.npz (m as float16) in pos_output_folder
        (mpm_solver.py:1755-1759); grid_m defaults to grid_mass()."""
        m = self.grid_mass() if grid_m is None else grid_m
        m = m.cpu().numpy() if hasattr(m, "cpu") else np.asarray(m)
        fn = os.path.join(self._out_folder(), "density_%06d.npz" % frame)
        np.savez_compressed(fn, m=m.astype(np.float16))
        return fn

    def status(self, clear=False):
        self._ensure_sim()
        f = C.c_uint32()
        fb = C.c_int64()
        _lib.check(_lib.lib().aq_sim_status(self._sim, C.byref(f), C.byref(fb), int(clear), _lib.stream_ptr()),
                   "aq_sim_status")
        return f.value, fb.value

    def sparse_blocks(self):
        """Sparse grid: (pool slots handed out, grid blocks holding particles
        at the last re-binning)."""
        self._ensure_sim()
        a, b = C.c_int64(), C.c_int64()
        _lib.check(_lib.lib().aq_sim_sparse_blocks(self._sim, C.byref(a), C.byref(b), _lib.stream_ptr()),
                   "aq_sim_sparse_blocks")
        return a.value, b.value

    def kernel_is_jit(self):
        self._ensure_sim()
        v = C.c_int32()
        _lib.check(_lib.lib().aq_sim_kernel_is_jit(self._sim, C.byref(v)), "aq_sim_kernel_is_jit")
        return bool(v.value)

    def launches(self):
        n = C.c_int64()
        if self._sim is None:
            return 0
        _lib.check(_lib.lib().aq_sim_launches(self._sim, C.byref(n)), "aq_sim_launches")
        return n.value

    # ------------------------------------------------------ SDF collider

    def init_sdf_value(self, sdf, normal, offset=None, theta=0.0, height=0.0, omega=5.0, height_rate=0.1):
        """The rotating SDF collider (init_sdf_collider / init_sdf_value,
        mpm_solver.py:284-318): sdf [a, b, c] signed distances and normal
        [a, b, c, 3] (e.g. the reference's inputs/propeller_*.npz, array
        'sdf'), placed at grid index offset (default the solver's
        sdf_offset, zero).  After every substep the angle advances by
        omega dt and the height by height_rate dt (step_collider,
        :1542-1547).  3D only."""
        import torch

        if self.dim != 3:
            raise ValueError("the SDF collider is 3D")
        sdf = np.asarray(sdf)
        normal = np.asarray(normal)
        if sdf.ndim != 3 or normal.shape != sdf.shape + (3,):
            raise ValueError("sdf must be [a, b, c] and normal [a, b, c, 3]")
        self._col = {
            "sdf": torch.from_numpy(np.ascontiguousarray(sdf, dtype=np.float32)).cuda(),
            "normal": torch.from_numpy(np.ascontiguousarray(normal, dtype=np.float32)).cuda(),
            "offset": [int(o) for o in (offset if offset is not None else [0, 0, 0])],
            "theta": float(theta), "height": float(height), "omega": float(omega), "rate": float(height_rate),
        }
        if self._sim is not None:
            self._apply_collider()

    def _apply_collider(self):
        c = self._col
        dims = (C.c_int32 * 3)(*c["sdf"].shape)
        off = (C.c_int32 * 3)(*c["offset"])
        _lib.check(_lib.lib().aq_sim_set_collider(self._sim, C.c_void_p(c["sdf"].data_ptr()),
                                                  C.c_void_p(c["normal"].data_ptr()), dims, off, int(self.n_grid),
                                                  c["theta"], c["height"], c["omega"], c["rate"]),
                   "aq_sim_set_collider")
        _lib.check(_lib.lib().aq_sim_collider_velocity_mode(self._sim, int(c.get("node_cv", False))),
                   "aq_sim_collider_velocity_mode")

    def _collider_velocity_from_node(self, on):
        """sdf_collision (off: omega x r from the rotated index, the forward
        substep) or sdf_collision_no_arg (on: from the node itself, the
        autodiff path's substep_difftaichi)."""
        c = self._col
        if c is None or bool(c.get("node_cv", False)) == bool(on):
            return
        c["node_cv"] = bool(on)
        if self._sim is not None:
            _lib.check(_lib.lib().aq_sim_collider_velocity_mode(self._sim, int(bool(on))),
                       "aq_sim_collider_velocity_mode")

    def collider_state(self):
        """(angle, height) of the collider now."""
        if self._col is None:
            return None
        if self._sim is None:
            return self._col["theta"], self._col["height"]
        th, hh = C.c_double(), C.c_double()
        _lib.check(_lib.lib().aq_sim_collider_get(self._sim, C.byref(th), C.byref(hh)), "aq_sim_collider_get")
        return th.value, hh.value

    # ------------------------------------------------- scheme parameters

    def reshape_params(self, ranges):
        """mpm_solver.py:522-535: flat x, v, C, J|F list -> per-field arrays."""
        d, qp = self.dim, self.param.quantized_properties or {"x": 1, "v": 1, "C": 1, ("J" if self.use_fluid else "F"): 1}
        ranges = np.asarray(ranges)
        r = []
        if "x" in qp:
            r.append(np.array(ranges[:d]))
        if "v" in qp:
            r.append(np.array(ranges[d:2 * d]))
        if "C" in qp:
            r.append(np.array(ranges[2 * d:2 * d + d * d]))
        if "J" in qp:
            r.append(np.array(ranges[-1:]))
        if "F" in qp:
            r.append(np.array(ranges[-d * d:]))
        return r

    def set_bits_and_ranges(self, bits, ranges):
        """mpm_solver.py:494-520: clamp bits to [1, 32] and rebuild the layout."""
        bits = [max(min(int(b), 32), 1) for b in bits]
        self.param.quant_bits = np.array(bits)
        self.param.quant_ranges = np.asarray(ranges, dtype=np.float64)
        self.bits = self.reshape_params(bits)
        self.ranges = self.reshape_params(ranges)
        self._pull()
        self._layout = None
        self._drop_sim()

    # ------------------------------------------------------------ adjoint

    def run_forward_with_ad_nlogn(self, save_pics=False, ggui=None, every=64):
        """The autodiff pass (mpm_solver.py:1093-1302, drivers' ad()): forward
        n_timestep-1 substeps on unquantized state with checkpoints, loss
        compute_ek, then the hand-written reverse pass; the per-scalar
        sensitivities are kept for get_gradients().  Returns the loss.
        every > 0: a checkpoint every `every` substeps, each segment
        recomputed once in the reverse pass (memory T/every + every states,
        T extra substeps); every = 0: the reference's logarithmic stash
        (memory log2 T states, about T log2(T) / 2 extra substeps), for
        horizons whose segment states would not fit."""
        import torch

        from .adjoint import Adjoint, ek_loss, ek_seed

        if self.has_mat:
            raise ValueError("the adjoint runs single-material scenes")
        self._pull()
        P = self._params()
        n, ns = self.current_idx, self.n_slots()
        adj = Adjoint(P)
        if self._col is not None:  # from the collider's current angle and height
            c = self._col
            th, hh = self.collider_state()
            adj.set_collider(c["sdf"], c["normal"], c["offset"], int(self.n_grid), th, hh, c["omega"], c["rate"])
        dt = torch.float64 if self.param.precision == "f64" else torch.float32
        if self._dev is not None and self._host is None:
            s0 = self._dev[:n, :ns].to(dt).contiguous()
        else:
            s0 = torch.from_numpy(np.ascontiguousarray(self._staging()[:n, :ns])).to("cuda", dt)
        sT = adj.forward(s0, self.n_timestep - 1, every)
        loss = ek_loss(sT, self.dim, self.p_mass, self.g)
        adj.backward(ek_seed(sT, self.dim, self.p_mass, self.g))
        self._grads = adj.sens
        self._ad_final = sT
        adj.close()
        self.loss[None] = loss
        return loss

    def get_gradients(self):
        """Per-scalar sum over substeps and particles of (dL/dq)^2, in the
        x, v, C, F|J order of get_gradients (mpm_solver.py:1273-1302)."""
        return np.asarray(self._grads)

    # ------------------------------------------------- range detection

    def run_forward_detect_ranges(self, n=None):
        """Range detection (run_forward_detect_ranges, mpm_solver.py:933-945):
        running max/min of every scalar after each substep, folded on the
        device.  The reference steps with nlogn_loop_forward, i.e. the
        autodiff path's substep and collider schedule; without a collider
        that is the plain substep, run fused here."""
        self._ensure_sim()
        self._rabs_host = None
        _lib.check(_lib.lib().aq_sim_ranges_enable(self._sim, 1, _lib.stream_ptr()), "aq_sim_ranges_enable")
        self._ranges_on_device = True
        total = self.n_timestep - 1 if n is None else n
        if self._col is None:
            self.substeps(total)
        else:
            for s in range(total):
                self.nlogn_step_forward(s)
        _lib.check(_lib.lib().aq_sim_ranges_enable(self._sim, 0, _lib.stream_ptr()), "aq_sim_ranges_enable")
        self.detect_bound()
        return self.get_limits()

    def detect_bound(self, s=0):
        """Running ranges so far: the device's (run_forward_detect_ranges)
        and the states detect_bound_kernel folded in."""
        ns = self.n_slots()
        self._rmax, self._rmin = np.full(ns, -np.inf), np.full(ns, np.inf)
        if getattr(self, "_ranges_on_device", False) and self._sim is not None:
            mx = (C.c_double * ns)()
            mn = (C.c_double * ns)()
            _lib.check(_lib.lib().aq_sim_ranges_get(self._sim, mx, mn, _lib.stream_ptr()), "aq_sim_ranges_get")
            self._rmax, self._rmin = np.array(mx[:]), np.array(mn[:])
        h = getattr(self, "_rabs_host", None)
        if h is not None:
            self._rmax, self._rmin = np.maximum(self._rmax, h), np.minimum(self._rmin, -h)

    # ------------------------------------- the drivers' own substep loops

    def nlogn_step_forward(self, s, emit_func=None):
        """Substep s of the drivers' own loops (nlogn_step_forward,
        mpm_solver.py:1161-1167): emit_func(s, self) first when given, then
        substep_difftaichi, then, with a collider, step_collider_difftaichi(s)
        (angle omega dt s, height 0.15 dt s for the next substep)."""
        if emit_func is not None:
            emit_func(s, self)
        self._substep_difftaichi_form()
        if self._col is not None:
            self.step_collider_difftaichi(s)

    def substep_difftaichi(self, s, t=None):
        """One substep of the autodiff path (mpm_solver.py:791-797): p2g,
        grid_op, the collider as sdf_collision_no_arg, g2p; the collider is
        not moved."""
        pose = self.collider_state() if self._col is not None else None
        self._substep_difftaichi_form()
        if pose is not None:  # the simulator advanced it: put it back
            self._set_collider_pose(*pose)

    def detect_bound_kernel(self, s=0):
        """Fold the current state into the running ranges (update_limits_*,
        mpm_solver.py:943-979): per scalar the max |q| of the state now, and
        only of this state (the drivers call it after every substep or once
        per frame)."""
        self._ensure_sim()
        cur = self.field_stats()[:, 3].copy()
        h = getattr(self, "_rabs_host", None)
        self._rabs_host = cur if h is None else np.maximum(h, cur)

    def step_collider(self):
        """The drivers call this after every substep (mpm_solver.py:1542-1547);
        the simulator already advances the collider by omega dt and
        height_rate dt inside each substep, so there is nothing left to do."""

    def step_collider_difftaichi(self, step):
        """Put the collider at substep `step` of the autodiff schedule:
        angle omega dt step, height 0.15 dt step (mpm_solver.py:1554-1559)."""
        if self._col is None:
            return
        self._set_collider_pose(self._col["omega"] * self.dt * step, 0.15 * self.dt * step)

    def _set_collider_pose(self, theta, height):
        self._col["theta"], self._col["height"] = float(theta), float(height)
        if self._sim is not None:
            _lib.check(_lib.lib().aq_sim_collider_pose(self._sim, float(theta), float(height)),
                       "aq_sim_collider_pose")

    @staticmethod
    def cnt_ending_zero(s):
        """Trailing zero bits of s + 1 (mpm_solver.py:1200-1207)."""
        cnt, s = 0, s + 1
        while s % 2 == 0:
            cnt += 1
            s >>= 1
        return cnt

    def dump_grad(self, s=0, fn=None):
        """Print the per-scalar sensitivities (mpm_solver.py:1328-1331)."""
        grads = np.hstack(self.get_gradients())
        print(grads)
        return grads

    def get_limits(self):
        """mpm_solver.py:981-992: [2]*dim for x, then max(|max|, |min|) of
        v, C and J|F."""
        d = self.dim
        lim = np.maximum(np.abs(self._rmax), np.abs(self._rmin))
        end = self.n_slots() - (1 if self.has_mat else 0)
        return np.hstack([[2.0] * d, lim[d:end]])

    def __del__(self):
        try:
            self._drop_sim()
        except Exception:
            pass
