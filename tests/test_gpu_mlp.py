"""The surrogate MLP kernels (aq_mlp_*) against the numpy oracle, and the
trained surrogate against the method without it.

The kernels' contractions run on bf16 tensor cores with fp32 accumulation,
the oracle restates them in float64 from the same bf16-rounded operands.  An
activation the kernel computes in fp32 (erff GELU) and the oracle in float64
can round to neighbouring bf16 values, which moves a downstream sum by one
bf16 step (2^-7 relative) of one of its terms: hence 2e-3 (relative to the
largest value) rather than fp32 rounding."""
import ctypes as C

import numpy as np
import pytest

import mlp_oracle as MO
from autoquantizer_b200 import _lib
from autoquantizer_b200 import surrogate as SG

pytestmark = pytest.mark.gpu
DIMS = (SG.N_IN, SG.N_H, SG.N_OUT)


def _mlp(seed=0):
    m = SG.MLP(seed=seed)
    rng = np.random.default_rng(seed + 1)
    # non-zero biases exercise the bias paths
    p = m.p.cpu().numpy()
    p += rng.normal(0, 0.05, p.shape).astype(np.float32)
    import torch

    m.p.copy_(torch.from_numpy(p))
    _lib.check(_lib.lib().aq_mlp_to_bf16(C.c_void_p(m.p.data_ptr()), C.c_void_p(m.pb.data_ptr()), m.n,
                                         _lib.stream_ptr()))
    return m, p


def test_forward_matches_oracle():
    m, p = _mlp()
    x = np.random.default_rng(5).normal(size=(257, SG.N_IN)).astype(np.float32)
    y = m.forward_raw(x).cpu().numpy()
    yo, _ = MO.forward(p, x, DIMS)
    assert np.max(np.abs(y - yo)) < 2e-3 * max(1.0, np.abs(yo).max())


def test_backward_matches_oracle():
    m, p = _mlp(3)
    rng = np.random.default_rng(7)
    x = rng.normal(size=(130, SG.N_IN)).astype(np.float32)
    dy = rng.normal(size=(130, SG.N_OUT)).astype(np.float32)
    g = m.grad_raw(x, dy).cpu().numpy()
    go = MO.backward(p, x, dy, DIMS)
    scale = np.abs(go).max()
    assert np.max(np.abs(g - go)) < 2e-3 * scale


def test_adam_step_matches_oracle():
    import torch

    m, p = _mlp(4)
    rng = np.random.default_rng(8)
    g = rng.normal(size=m.n).astype(np.float32)
    m.g.copy_(torch.from_numpy(g))
    mm, vv = np.zeros(m.n), np.zeros(m.n)
    pp = p.astype(np.float64)
    for t in (1, 2, 3):
        m.t = t
        _lib.check(_lib.lib().aq_mlp_adam(C.c_void_p(m.p.data_ptr()), C.c_void_p(m.pb.data_ptr()),
                                          C.c_void_p(m.m.data_ptr()), C.c_void_p(m.v.data_ptr()),
                                          C.c_void_p(m.g.data_ptr()), m.n, 1e-3, 0.9, 0.999, 1e-8, t,
                                          _lib.stream_ptr()))
        pp, mm, vv = MO.adam(pp, mm, vv, g.astype(np.float64), t)
    assert m.p.cpu().numpy() == pytest.approx(pp, rel=1e-5, abs=1e-7)
    assert (m.pb.cpu().numpy().astype(np.uint16).astype(np.uint32) << 16).view(np.float32) == pytest.approx(
        MO.bf16(m.p.cpu().numpy()), rel=0, abs=0)


def test_fit_learns_a_smooth_map():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(512, SG.N_IN))
    A = rng.normal(size=(SG.N_IN, SG.N_OUT)) / 8
    Y = np.tanh(X @ A) + 0.1 * X[:, :SG.N_OUT] ** 2
    M = np.ones_like(Y)
    mlp = SG.MLP(seed=1)
    hist = mlp.fit(X, Y, M, steps=1500, lr=1e-3, batch=128)
    assert hist[-1][1] < 0.2 * hist[0][1]
    err = np.mean((mlp.predict(X) - Y) ** 2) / np.var(Y)
    assert err < 0.1


def test_surrogate_beats_the_method_without_it():
    """Small-scale version of the C5 experiment: scenes of 10k-30k particles,
    32-substep horizons.  The method without the network predicts every
    scene's log-sensitivities by the training mean; the network must predict
    them better and derive schemes closer to the adjoint's."""
    Xtr, Ytr, Mtr, _ = SG.make_dataset(48, 11, n_min=10_000, n_max=30_000, horizon=32)
    Xte, Yte, Mte, mte = SG.make_dataset(16, 12, n_min=10_000, n_max=30_000, horizon=32)
    mlp = SG.MLP(seed=0)
    mlp.fit(Xtr, Ytr, Mtr, steps=1500, lr=1e-3, batch=32)
    base = (Ytr * Mtr).sum(0) / np.maximum(Mtr.sum(0), 1)
    sur, bl = SG.evaluate(mlp, Xte, Yte, Mte, mte, baseline=base)
    assert sur["log_err"] < 0.7 * bl["log_err"], (sur, bl)
    assert sur["within_1_bit"] >= bl["within_1_bit"], (sur, bl)


def test_ensemble_predicts_the_members_mean():
    """The ensemble's on-device mean equals the mean of its members' own
    predictions; the members start from different weights and batch orders."""
    rng = np.random.default_rng(2)
    X = rng.normal(size=(64, SG.N_IN))
    Y = rng.normal(size=(64, SG.N_OUT))
    e = SG.Ensemble(3, seed=5)
    e.fit(X, Y, np.ones_like(Y), steps=20, batch=32)
    each = [m.predict(X) for m in e.members]
    assert not np.allclose(each[0], each[1])
    assert e.predict(X) == pytest.approx(np.mean(each, axis=0), rel=1e-5, abs=1e-6)
    mean, spread = e.predict_spread(X)
    assert mean == pytest.approx(np.mean(each, axis=0), rel=1e-5, abs=1e-6)
    assert spread == pytest.approx(np.std(each, axis=0), rel=1e-4, abs=1e-6)


def test_derive_scheme_falls_back_to_the_adjoint():
    """derive_scheme takes the ensemble's prediction when the widths its
    members derive agree within max_span bits and the adjoint's sensitivities
    otherwise; the
    fallback's widths are the adjoint-derived scheme's (to a bit: two
    adjoint runs add their atomic sums in different orders)."""
    import torch

    Xtr, Ytr, Mtr, _ = SG.make_dataset(24, 11, n_min=10_000, n_max=20_000, horizon=32)
    e = SG.Ensemble(2, seed=1)
    e.fit(Xtr, Ytr, Mtr, steps=200, batch=16)
    rng = np.random.default_rng(7)
    cfg, vals = SG.random_scene(rng, 10_000, 20_000, horizon=32)
    s0 = torch.from_numpy(vals).to("cuda", torch.float32)
    b_fb, mask, how = SG.derive_scheme(cfg, s0, e, max_span=-1)
    assert how == "adjoint"
    sens, loss = SG.adjoint_sensitivities(cfg, s0)
    ys, m2 = SG.group_sensitivities(cfg, sens)
    st = SG.window_stats(cfg, s0)
    assert np.abs(b_fb - SG.scheme_bits(ys, m2, SG.group_ranges(cfg, st), loss)).max() <= 1
    b_sur, _, how = SG.derive_scheme(cfg, s0, e, max_span=99)
    assert how == "surrogate"
    assert b_sur.shape == b_fb.shape and np.all(b_sur[mask > 0] >= SG.MIN_WIDTH)
