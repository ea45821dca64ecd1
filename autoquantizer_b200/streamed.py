"""Out-of-core (streamed) simulation of an MPMSolver scene.

The packed records of every particle live in pinned host memory owned by
libaq; each pass over the particles (a substep, the loss) moves them through
the device in chunks of at most `chunk` records: upload, binning of the
chunk, the fused substep kernel, download.  The grids stay on the device and
collect all chunks, so the result is the in-core simulator's up to the order
in which grid sums are added.  This is for scenes whose records do not fit in
device memory; the host link then bounds the speed, in proportion to the
record's bytes, which is where a quantized record pays in full.

    s = MPMSolver(cfg); s.set_particles(values)
    st = StreamedSolver(s, chunk=1 << 24)   # the scene's records move to the host
    st.substeps(100)
    values = st.state_values()

The reference keeps its particle fields in device memory
(mpm_exps/engine/mpm_solver.py:190-207) and has no such mode.
"""
import ctypes as C

import numpy as np

from . import _lib


def encode_values(solver, batch):
    """The packed records (n x n_words, particle order) of a solver's
    particle values as it holds them before a simulator runs (host staging
    array or device tensor), encoded on the device `batch` particles at a
    time with the codes a simulator's aq_sim_set_state gives them
    (dithering keyed on the particle ids at the initial-state step)."""
    import torch

    L = solver.layout()
    n, W = int(solver.current_idx), L.n_words
    out = np.empty((n, W), dtype=np.uint64)
    dev = solver._dev if (solver._dev is not None and solver._host is None) else None
    for a in range(0, n, batch):
        b = min(n, a + batch)
        if dev is not None:
            v = dev[a:b].to(torch.float64).contiguous()
        else:
            v = torch.from_numpy(np.ascontiguousarray(solver._staging()[a:b])).cuda()
        ids = torch.arange(a, b, dtype=torch.int32, device="cuda")
        w = torch.empty((b - a, W), dtype=torch.int64, device="cuda")
        _lib.check(_lib.lib().aq_encode(C.byref(L), C.c_void_p(v.data_ptr()), 1, C.c_void_p(w.data_ptr()), b - a,
                                        C.c_void_p(ids.data_ptr()), int(solver.param.seed), -1, None,
                                        _lib.stream_ptr()), "aq_encode")
        out[a:b] = w.cpu().numpy().view(np.uint64)
    return out


class StreamedSolver:
    """A streamed copy of `solver`'s scene: its parameters, record layout,
    current records and substep count (the dithering generator's step
    index).  The SDF collider and sparse grids are not streamed."""

    def __init__(self, solver, chunk):
        if solver._col is not None:
            raise ValueError("StreamedSolver: the SDF collider is not streamed")
        if getattr(solver.param, "sparse_grid", False):
            raise ValueError("StreamedSolver: streamed chunks bin on a dense grid")
        if solver._sim is not None and not solver._dirty:
            words = solver.words()  # a running simulator: its current records
        else:  # no simulator (a scene set up but not run): encode chunk by chunk, none in device memory whole
            words = encode_values(solver, chunk)
        step = solver.step_count()
        self.dim = solver.dim
        self.n_particles = int(solver.current_idx)
        self._layout = solver.layout()
        self.n_words = self._layout.n_words
        P = solver._params()
        sim = C.c_void_p()
        _lib.check(_lib.lib().aq_sim_create_streamed(C.byref(P), C.byref(self._layout), int(chunk), C.byref(sim)),
                   "aq_sim_create_streamed")
        self._sim = sim
        self.set_words(words)
        _lib.check(_lib.lib().aq_sim_set_step_count(self._sim, int(step)), "aq_sim_set_step_count")

    def chunks(self):
        """(records per chunk, particles)."""
        a, b = C.c_int64(), C.c_int64()
        _lib.check(_lib.lib().aq_sim_stream_chunks(self._sim, C.byref(a), C.byref(b)), "aq_sim_stream_chunks")
        return a.value, b.value

    def set_words(self, words):
        """Packed records (n x n_words uint64, particle order) from host memory."""
        w = np.ascontiguousarray(words, dtype=np.uint64)
        if w.shape != (self.n_particles, self.n_words):
            raise ValueError("set_words: expected %s records" % ((self.n_particles, self.n_words),))
        _lib.check(_lib.lib().aq_sim_stream_set_words(self._sim, C.c_void_p(w.ctypes.data), _lib.stream_ptr()),
                   "aq_sim_stream_set_words")

    def words(self):
        out = np.empty((self.n_particles, self.n_words), dtype=np.uint64)
        _lib.check(_lib.lib().aq_sim_stream_get_words(self._sim, C.c_void_p(out.ctypes.data), _lib.stream_ptr()),
                   "aq_sim_stream_get_words")
        return out

    def state_values(self, f64=True, batch=1 << 22):
        """Decoded state, particle order (n x n_slots), decoded on the device
        `batch` records at a time."""
        import torch

        w = self.words()
        ns = self._layout.n_slots
        out = np.empty((self.n_particles, ns), dtype=np.float64 if f64 else np.float32)
        for a in range(0, self.n_particles, batch):
            b = min(self.n_particles, a + batch)
            dw = torch.from_numpy(w[a:b].view(np.int64)).cuda()
            dv = torch.empty((b - a, ns), dtype=torch.float64 if f64 else torch.float32, device="cuda")
            _lib.check(_lib.lib().aq_decode(C.byref(self._layout), C.c_void_p(dw.data_ptr()), C.c_void_p(dv.data_ptr()),
                                            int(f64), b - a, _lib.stream_ptr()), "aq_decode")
            out[a:b] = dv.cpu().numpy()
        return out

    def substeps(self, n):
        _lib.check(_lib.lib().aq_sim_substeps(self._sim, int(n), _lib.stream_ptr()), "aq_sim_substeps")

    def compute_loss(self):
        out = C.c_double()
        _lib.check(_lib.lib().aq_sim_loss(self._sim, 0, C.byref(out), _lib.stream_ptr()), "aq_sim_loss")
        return out.value

    def step_count(self):
        v = C.c_int64()
        _lib.check(_lib.lib().aq_sim_step_count(self._sim, C.byref(v)), "aq_sim_step_count")
        return v.value

    def status(self, clear=False):
        f, fb = C.c_uint32(), C.c_int64()
        _lib.check(_lib.lib().aq_sim_status(self._sim, C.byref(f), C.byref(fb), int(clear), _lib.stream_ptr()),
                   "aq_sim_status")
        return f.value, fb.value

    def close(self):
        if getattr(self, "_sim", None) is not None:
            _lib.lib().aq_sim_destroy(self._sim)
            self._sim = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
