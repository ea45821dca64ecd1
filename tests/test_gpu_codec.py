"""GPU codec parity: aq_encode / aq_decode (sm_100a) against the oracle,
bit-exact on the packed words and on the decoded values."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from autoquantizer_b200 import _lib
from autoquantizer_b200 import quant as Q
from test_capi import _random_pack

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def gpu_encode(L, vals, pid=None, seed=0, step=0, uniforms=None, f64=True):
    torch = _torch()
    n = vals.shape[0]
    v = torch.from_numpy(np.ascontiguousarray(vals, dtype=np.float64 if f64 else np.float32)).cuda()
    w = torch.zeros((n, L.n_words), dtype=torch.int64, device="cuda")
    p = None if pid is None else torch.from_numpy(np.ascontiguousarray(pid, dtype=np.int32)).cuda()
    u = None
    if uniforms is not None:
        u = torch.from_numpy(np.ascontiguousarray(uniforms, dtype=np.float64 if L.compute_f64 else np.float32)).cuda()
    _lib.check(_lib.lib().aq_encode(C.byref(L), C.c_void_p(v.data_ptr()), int(f64), C.c_void_p(w.data_ptr()), n,
                                    None if p is None else C.c_void_p(p.data_ptr()), seed, step,
                                    None if u is None else C.c_void_p(u.data_ptr()), _lib.stream_ptr()), "aq_encode")
    return w.cpu().numpy().view(np.uint64)


def gpu_decode(L, words, f64=True):
    torch = _torch()
    w = torch.from_numpy(np.ascontiguousarray(words).view(np.int64)).cuda()
    out = torch.zeros((words.shape[0], L.n_slots), dtype=torch.float64 if f64 else torch.float32, device="cuda")
    _lib.check(_lib.lib().aq_decode(C.byref(L), C.c_void_p(w.data_ptr()), C.c_void_p(out.data_ptr()), int(f64),
                                    words.shape[0], _lib.stream_ptr()), "aq_decode")
    return out.cpu().numpy()


def _values_for(rec, n, rng):
    cols = []
    for t, _ in rec.items:
        if isinstance(t, Q.Fixed):
            r = t.range * 1.2
            c = rng.uniform(-r if t.signed else -0.1 * r, r, n) + t.offset
        elif isinstance(t, Q.Int):
            hi = 2 ** (t.bits - 1) if t.signed else 2 ** t.bits
            c = rng.integers(-hi if t.signed else 0, hi, n).astype(np.float64)
        elif isinstance(t, Q.Float):
            c = rng.choice([-1, 1], n) * 10 ** rng.uniform(-12, 12, n)
            if not t.signed:
                c = np.abs(c)
            c[rng.random(n) < 0.05] = 0.0
        else:
            c = rng.normal(0, 10, n)
        cols.append(c)
    return np.stack(cols, 1)


def _same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


@pytest.mark.parametrize("seed", range(20))
def test_random_layout_codec_bit_exact(seed):
    rng = np.random.default_rng(100 + seed)
    rec = _random_pack(rng)
    if len(rec.items) > 32 or len({g for _, g in rec.items if g is not None}) > 4:
        pytest.skip("over the slot/group limits")
    L = rec.build()
    f64, dith = rec.compute_and_dithering()
    Lo = O.build_layout(rec.spec_tuples(), f64, dith)
    n = 4096
    vals = _values_for(rec, n, rng)
    pid = rng.permutation(n).astype(np.int32)
    wg = gpu_encode(L, vals, pid=pid, seed=seed + 7, step=seed * 3 - 1)
    wo = O.encode(Lo, vals, pid=pid, seed=seed + 7, step=seed * 3 - 1)
    assert np.array_equal(wg, wo)
    assert _same_bits(gpu_decode(L, wo), O.decode(Lo, wo))


def test_explicit_uniforms_bit_exact():
    rng = np.random.default_rng(5)
    for f64 in (False, True):
        rec = Q.BitPack()
        rec.place(*[Q.fixed(b, True, 2.0, 0.0, "f64" if f64 else "f32", True) for b in (5, 11, 17, 23, 32)])
        L = rec.build()
        Lo = O.build_layout(rec.spec_tuples(), f64, True)
        vals = rng.uniform(-2.2, 2.2, (8192, 5))
        u = rng.random((8192, 5))
        if not f64:
            u = u.astype(np.float32).astype(np.float64)
        assert np.array_equal(gpu_encode(L, vals, uniforms=u), O.encode(Lo, vals, uniforms=u))


def test_f32_values_input():
    rng = np.random.default_rng(9)
    rec = Q.BitPack()
    rec.place(Q.fixed(21, True, 1.0, 0.0, "f32", True))
    rec.place(Q.qfloat(12, 6), Q.qfloat(12, 6), shared_exponent=True)
    L = rec.build()
    Lo = O.build_layout(rec.spec_tuples(), False, True)
    vals = rng.uniform(-1, 1, (5000, 3)).astype(np.float32)
    wg = gpu_encode(L, vals, seed=3, step=11, f64=False)
    wo = O.encode(Lo, vals.astype(np.float64), seed=3, step=11)
    assert np.array_equal(wg, wo)
    dg = gpu_decode(L, wo, f64=False)
    assert np.array_equal(dg, O.decode(Lo, wo).astype(np.float32))


def test_dithering_ratio_on_gpu():
    rec = Q.BitPack()
    rec.place(Q.fixed(5, True, 2.0, 0.0, "f64", True))
    L = rec.build()
    out = gpu_decode(L, gpu_encode(L, np.full((400000, 1), 1.1), seed=1234, step=7))[:, 0]
    up, down = (out == 1.125).sum(), (out == 1.0).sum()
    assert up + down == 400000 and abs(up / down - 4) < 0.05  # three binomial standard deviations


def test_c2_record_words_match_oracle_at_full_size():
    # the 2D dam-break record (152 bits) over all 65,536 particles
    rec = Q.BitPack()
    rec.place(Q.fixed(20, range=1.0, use_dithering=True), Q.fixed(20, range=1.0, use_dithering=True))
    rec.place(Q.qfloat(13, 6), Q.qfloat(13, 6), shared_exponent=True)
    rec.place(*[Q.fixed(16, range=64.0, use_dithering=True)] * 4)
    rec.place(Q.fixed(16, range=0.5, offset=1.0, use_dithering=True))
    L = rec.build()
    Lo = O.build_layout(rec.spec_tuples(), False, True)
    rng = np.random.default_rng(1)
    n = 65536
    vals = np.concatenate([rng.random((n, 2)), rng.normal(0, 2, (n, 2)), rng.normal(0, 20, (n, 4)),
                           rng.uniform(0.6, 1.4, (n, 1))], 1)
    wg = gpu_encode(L, vals, seed=42, step=3999)
    assert np.array_equal(wg, O.encode(Lo, vals, seed=42, step=3999))


@pytest.mark.parametrize("kind", ["fixed", "exponent", "shared"])
def test_time_integration_through_the_gpu_codec(kind):
    """test_custom_float_time_integration.py:10-66 with every store going
    through aq_encode / aq_decode: the circle closes to 2e-2 (3e-2 for the
    final y), and every stored position equals the oracle codec's."""
    import math

    rec = Q.BitPack()
    if kind == "fixed":
        rec.place(Q.fixed(16, True, 2.0), Q.fixed(16, True, 2.0))
    elif kind == "exponent":
        rec.place(Q.qfloat(13, 6, True), Q.qfloat(13, 6, True))
    else:
        rec.place(Q.qfloat(13, 6, True), Q.qfloat(13, 6, True), shared_exponent=True)
    L = rec.build()
    OL = O.build_layout(rec.spec_tuples(), *rec.compute_and_dithering())

    def store(p):
        p = np.asarray(p, dtype=np.float32).astype(np.float64)[None]
        w = gpu_encode(L, p)
        assert np.array_equal(w, O.encode(OL, p))
        return gpu_decode(L, w)[0]

    def v_at(p):
        return np.array([-p[1], p[0]], dtype=np.float32)

    x = store([1.0, 0.0])
    n = 1000
    dt = np.float32(math.pi * 2 / n)
    px, py = [], []
    for _ in range(n):
        xf = x.astype(np.float32)
        x = store(xf + v_at(xf + np.float32(0.5) * dt * v_at(xf)) * dt)
        px.append(x[0])
        py.append(x[1])
    assert abs(px[n // 2 - 1] + 1) <= 2e-2 and abs(py[n // 2 - 1]) <= 2e-2
    assert abs(px[-1] - 1) <= 2e-2 and abs(py[-1]) <= 3e-2
