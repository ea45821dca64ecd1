"""The streamed (out-of-core) simulator against the in-core one.

Both start from the same records and substep count (so the dithering draws
are the same); the streamed one keeps its records in host memory and passes
them through the device in chunks (sizes that are not multiples of the
32-record groups included), binning each chunk on its own.  Grid sums are
then added in another order, so the comparison allows what two in-core runs
differ by: 2e-5 relative plus two quantization steps per slot over a few
substeps (f32), 1e-9 relative in f64 compute.
"""
import ctypes as C

import numpy as np
import pytest

from autoquantizer_b200 import _lib, scenes
from autoquantizer_b200.mpm_solver import MPMSolver
from autoquantizer_b200.streamed import StreamedSolver
from helpers import quant_steps

pytestmark = pytest.mark.gpu


def _close(a, b, s, rel=2e-5, steps=2.0):
    q = quant_steps(s)
    for k in range(a.shape[1]):
        scale = max(1.0, float(np.max(np.abs(b[:, k]))))
        tol = rel * scale + (steps * q[k] if q[k] > 0 else 2.0 ** -10 * scale if np.isnan(q[k]) else 0.0)
        err = float(np.max(np.abs(a[:, k] - b[:, k])))
        assert err <= tol, (k, err, tol)


def _pair(cfg, vals, chunk, warm=0):
    s = MPMSolver(cfg)
    s.set_particles(vals)
    if warm:
        s.substeps(warm)
    return s, StreamedSolver(s, chunk)


def test_words_round_trip_through_host_chunks():
    """A scene set up but not run is encoded chunk by chunk, with no
    in-core simulator, to the codes the in-core simulator gives it
    (dithered layout: the draws are keyed on the same particle ids), and
    records go through the host chunks and back unchanged."""
    cfg, vals = scenes.dam_break_2d(n=5000, n_grid=64)
    s, st = _pair(cfg, vals, chunk=1234)
    assert s._sim is None
    assert st.chunks() == (1234, 5000)
    w = s.words()
    assert np.array_equal(st.words(), w)
    st.set_words(w[::-1].copy())
    assert np.array_equal(st.words(), w[::-1])
    st.close()


@pytest.mark.parametrize("chunk", [3000, 4096, 8192])
def test_streamed_quantized_2d_matches_in_core(chunk):
    """The quantized, dithered 2D dam break (8,192 particles, 128^2) in
    three, two or one chunks, 4 substeps after 8 in-core ones (the passes
    of a chain overlap whatever the chunk count)."""
    cfg, vals = scenes.dam_break_2d(n=8192, n_grid=128)
    s, st = _pair(cfg, vals, chunk=chunk, warm=8)
    assert st.step_count() == s.step_count() == 8
    s.substeps(4)
    st.substeps(4)
    assert st.step_count() == 12
    _close(st.state_values(), s.state_values(), s)
    assert st.compute_loss() == pytest.approx(s.compute_loss(), rel=1e-5)
    assert st.status()[0] == 0
    st.close()


def test_streamed_3d_f64_matches_in_core():
    """The 3D mixed scene (40,000 particles, 32^3, FP32-state record layout,
    f64 compute) in chunks of 7,000 records over 6 substeps: the grid sums
    differ only in their order of addition."""
    cfg, vals = scenes.mixed_boxes_3d(n=40000, n_grid=32, quantized=False, precision="f64")
    s, st = _pair(cfg, vals, chunk=7000)
    s.substeps(6)
    st.substeps(6)
    a, b = st.state_values(), s.state_values()
    for k in range(a.shape[1]):
        scale = max(1.0, float(np.max(np.abs(b[:, k]))))
        assert float(np.max(np.abs(a[:, k] - b[:, k]))) <= 1e-9 * scale, k
    assert st.compute_loss() == pytest.approx(s.compute_loss(), rel=1e-10)
    st.close()


def test_streamed_simulator_refuses_device_state_calls():
    """The state of a streamed simulator is in host memory: the entry points
    that take device buffers of the whole state return AQ_E_STATE."""
    import torch

    cfg, vals = scenes.dam_break_2d(n=2048, n_grid=64)
    s, st = _pair(cfg, vals, chunk=1000)
    out = torch.empty((2048, s.n_slots()), dtype=torch.float64, device="cuda")
    rc = _lib.lib().aq_sim_get_state(st._sim, C.c_void_p(out.data_ptr()), 1, _lib.stream_ptr())
    assert rc == -5
    w = torch.empty((2048, s.layout().n_words), dtype=torch.int64, device="cuda")
    assert _lib.lib().aq_sim_get_words(st._sim, C.c_void_p(w.data_ptr()), _lib.stream_ptr()) == -5
    s.substeps(0)  # an in-core simulator: the streamed entry points refuse it
    assert _lib.lib().aq_sim_stream_get_words(s._sim, C.c_void_p(w.data_ptr()), _lib.stream_ptr()) == -5
    st.close()
