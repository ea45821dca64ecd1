"""Pins the CPU oracle to the reference's own known-answer tests.

Each test restates the semantics of one of the reference's quant tests
(paths inside the AutoQuantizer repository) on the oracle codec.  Where the
reference test stores one field of a bit_struct/bit_pack, the helper
`store` re-encodes the whole record with the other fields at their decoded
values, which is what the reference's masked read-modify-write store
(codegen_llvm_quant.cpp:347-457) computes for a shared-exponent group.
"""
import math

import numpy as np
import pytest
from pytest import approx

import oracle as O

FIXED, INT, FLOAT_EXP, SHARED_EXP, RAW_F32, RAW_F64 = range(6)


def fixed(bits, rng=1.0, signed=True, offset=0.0):
    return (FIXED, bits, int(signed), 0, -1, rng, offset)


def qint(bits, signed=False):
    return (INT, bits, int(signed), 0, -1, 0.0, 0.0)


def fexp(bits, ebits, signed=True):
    return (FLOAT_EXP, bits, int(signed), ebits, -1, 0.0, 0.0)


def shexp(bits, ebits, signed=False, group=0):
    return (SHARED_EXP, bits, int(signed), ebits, group, 0.0, 0.0)


class Rec:
    """One record of a layout, with per-field store as the reference does."""

    def __init__(self, specs, compute_f64=False, dither=False, seed=0):
        self.L = O.build_layout(specs, compute_f64, dither)
        self.w = np.zeros((1, self.L.n_words), dtype=np.uint64)
        self.seed, self.step = seed, 0

    def vals(self):
        return O.decode(self.L, self.w)[0]

    def __getitem__(self, i):
        return self.vals()[i]

    def store(self, i, value):
        v = self.vals()
        v[i] = value
        self.assign(v)

    def assign(self, values):
        self.w = O.encode(self.L, np.asarray(values, dtype=np.float64)[None], seed=self.seed, step=self.step)
        self.step += 1


# ---------------------------------------------------------------- layout


def test_layout_offsets_follow_place_order():
    # struct_llvm.cpp:77-116: consecutive bit positions; a shared exponent
    # precedes the first member of its group (snode_expr_utils.cpp:44-66)
    L = O.build_layout([fixed(20), fixed(20), shexp(13, 6, True), shexp(13, 6, True),
                        fixed(16, 64), fixed(16, 64), fixed(16, 64), fixed(16, 64), fixed(16, 0.5, offset=1.0)])
    offs = [L.off[i] for i in range(L.n)]
    assert offs == [0, 20, 46, 59, 72, 88, 104, 120, 136]
    assert L.eoff[2] == 40 and L.eoff[3] == 40
    assert L.total_bits == 152 and L.n_words == 3


def test_layout_3d_throughput_record_is_seven_words():
    specs = [fixed(21)] * 3 + [shexp(12, 6, True)] * 3 + [fixed(16, 64)] * 9 + [fixed(16, 2)] * 9
    L = O.build_layout(specs)
    assert L.total_bits == 393 and L.n_words == 7


# ------------------------------------------------- test_bit_pack_assign.py


def test_bit_pack_assign_values():
    # test_bit_pack_assign.py:10-38: 3 x fixed(21, range 2) + int15, f32
    r = Rec([fixed(21, 2.0)] * 3 + [qint(15)])
    r.assign([1.5, 1.2, 1.3, 15])
    v = r.vals()
    assert v[0] == approx(1.5, rel=1e-4) and v[1] == approx(1.2, rel=1e-4) and v[2] == approx(1.3, rel=1e-4)
    assert v[3] == 15
    r.assign([-1.1, 1.3, -1.2, 16])
    v = r.vals()
    assert v[0] == approx(-1.1, rel=1e-4) and v[1] == approx(1.3, rel=1e-4) and v[2] == approx(-1.2, rel=1e-4)
    assert v[3] == 16


def test_bit_pack_assign_split_exactly_on_64():
    # test_bit_pack_assign.py:40-69: 4 x fixed(16) ends exactly on bit 64
    r = Rec([fixed(16, 2.0)] * 4 + [qint(15)])
    assert r.L.n_words == 2 and r.L.off[4] == 64
    r.assign([1.5, 1.2, 1.3, 1.6, 15])
    v = r.vals()
    assert list(np.round(v[:4], 3)) == approx([1.5, 1.2, 1.3, 1.6], rel=1e-4)
    assert v[4] == 15
    r.assign([-1.1, 1.3, -1.2, -1.6, 16])
    v = r.vals()
    assert list(v[:4]) == approx([-1.1, 1.3, -1.2, -1.6], rel=1e-4)
    assert v[4] == 16


def test_bit_pack_assign_exact_codes():
    # 1.5 with scale 2/2^20: code 786432, stored little-endian from bit 0
    L = O.build_layout([fixed(21, 2.0)] * 3 + [qint(15)])
    w = O.encode(L, np.array([[1.5, 1.2, 1.3, 15]]))
    codes = [(int(w[0, 0]) >> 0) & (2**21 - 1), (int(w[0, 0]) >> 21) & (2**21 - 1)]
    assert codes[0] == 786432
    assert codes[1] == int(np.float32(np.float32(1.2) * np.float32(2**20 / 2.0)) + 0.5)


# -------------------------------------------------------- test_bit_pack.py


def test_simple_array_int_roundtrip():
    # test_bit_pack.py:7-37: int13 signed and uint19 in one pack
    L = O.build_layout([qint(13, True), qint(19, False)])
    vals = np.array([[-(2**i), 2**i - 1] for i in range(12)], dtype=np.float64)
    assert (O.decode(L, O.encode(L, vals)) == vals).all()


def test_custom_int_load_and_store():
    # test_bit_pack.py:40-78: 31/29/8-bit boundary values; 31+29 > 64 splits
    L = O.build_layout([qint(31, True), qint(29, False), qint(8, True)])
    cases = np.array([[2**30 - 1, 2**29 - 1, -(2**7)], [2**30 - 1, 2**29 - 1, -(2**7 - 1)],
                      [0, 0, 0], [123, 4567, 8], [10, 31, 11]], dtype=np.float64)
    assert (O.decode(L, O.encode(L, cases)) == cases).all()


def test_fixed32_struct_for_values():
    # test_bit_pack.py:80-105: fixed(32, range 1024) holds small integers
    L = O.build_layout([fixed(32, 1024.0)])
    vals = np.arange(64, dtype=np.float64)[:, None]
    assert O.decode(L, O.encode(L, vals)) == approx(vals, abs=1e-3)


# --------------------------------------------------------- test_dithering.py


def _dither_ratio(trials):
    # test_dithering.py:4-31: fixed(5 bits, range 2, f64, dithering).  The
    # stored value is 1.1 (Taichi forwards the 0.7 store into the add), whose
    # exact code is 8.8: 9 (1.125) with probability 0.8, 8 (1.0) with 0.2.
    L = O.build_layout([fixed(5, 2.0)], compute_f64=True, dither=True)
    vals = np.full((trials, 1), 1.1)
    out = O.decode(L, O.encode(L, vals, seed=1234, step=7))[:, 0]
    up, down = int((out == 1.125).sum()), int((out == 1.0).sum())
    assert up + down == trials
    return up / down


# The up/down ratio of n dithered stores has a binomial spread of about
# 0.1 at n = 10,000 (the size of the reference's test, which asserts 0.1,
# i.e. one standard deviation); the bounds here are three.
def test_dithering_ratio_reference_size():
    assert abs(_dither_ratio(10000) - 4) < 0.3


def test_dithering_ratio_large_sample():
    assert abs(_dither_ratio(400000) - 4) < 0.05


def test_dithering_uniforms_are_uniform_and_uncorrelated():
    n = 4000
    u = np.array([[O.uniform(99, 3, p, s) for s in range(4)] for p in range(n)])
    for s in range(4):
        h, _ = np.histogram(u[:, s], bins=10, range=(0, 1))
        assert ((h - n / 10) ** 2 / (n / 10)).sum() < 30  # chi2, 9 dof: p < 0.001
        assert abs(np.corrcoef(u[:, s], u[:, (s + 1) % 4])[0, 1]) < 0.06


def test_dithering_given_uniform_is_deterministic():
    # encode takes u explicitly: code = trunc(c + u - 0.5 + 0.5) for c >= 0
    L = O.build_layout([fixed(5, 2.0)], compute_f64=True, dither=True)
    for u, expect in [(0.0, 1.0), (0.19, 1.0), (0.2000001, 1.125), (0.999, 1.125)]:
        out = O.decode(L, O.encode(L, np.array([[1.1]]), uniforms=np.array([[u]])))
        assert out[0, 0] == expect


def test_rounding_half_away_from_zero():
    # rounding_prepare (runtime.cpp:1732-1753): f + copysign(0.5, f), trunc
    L = O.build_layout([fixed(8, 128.0)])  # scale 1
    vals = np.array([[2.5], [-2.5], [2.4999], [-2.4999], [0.5], [-0.5]])
    assert list(O.decode(L, O.encode(L, vals))[:, 0]) == [3, -3, 2, -2, 1, -1]


def test_fixed_wraps_out_of_range():
    # custom_type_to_bits masks the code without clamping (:174-180)
    L = O.build_layout([fixed(4, 8.0)])  # scale 1, codes -8..7
    assert O.decode(L, O.encode(L, np.array([[9.0]])))[0, 0] == -7


# ------------------------------------------------------ test_fxp_offset.py


def test_fxp_offset():
    # test_fxp_offset.py:10-23: fixed(29, range 2, offset 1)
    r = Rec([fixed(29, 2.0, offset=1.0)])
    for v in [1.1, 0.64, 0.66, 2.8]:
        r.store(0, v)
        assert r[0] == approx(v, rel=1e-4)


# ------------------------------------------------------ test_custom_float.py


def test_custom_float_fixed32_in_pack():
    # test_custom_float.py:9-28
    r = Rec([fixed(32, 2.0)])
    for v in [1.1, 0.64, 0.66]:
        r.store(0, v)
        assert r[0] == approx(v)


def test_custom_matrix_rotation():
    # test_custom_float.py:31-62: a fixed(28, range 1.2) 2x2 matrix rotated by
    # 18 degrees five times in f32, re-quantized after every rotation
    r = Rec([fixed(28, 1.2)] * 4)
    r.assign([1.0, 0.0, 0.0, 1.0])
    a = np.float32(math.pi / 10)
    rot = np.array([[np.cos(a), np.sin(a)], [-np.sin(a), np.cos(a)]], dtype=np.float32)
    for _ in range(5):
        m = r.vals().astype(np.float32).reshape(2, 2)
        r.assign((m @ rot).astype(np.float64).ravel())
    m = r.vals().reshape(2, 2)
    assert m == approx(np.array([[0, 1], [-1, 0]]), abs=1e-4)


def test_custom_float_implicit_cast():
    # test_custom_float.py:65-77 (13-bit int digits, scale 0.1 ~ fixed range)
    r = Rec([(FIXED, 13, 1, 0, -1, 0.1 * 2**12, 0.0)])
    r.store(0, 10)
    assert r[0] == approx(10.0)


# ---------------------------------------------- test_custom_float_exponents.py


def test_custom_float_unsigned_exact():
    # test_custom_float_exponents.py:9-30
    r = Rec([fexp(13, 6, signed=False)])
    assert r[0] == 0
    for v in [0, 1 / 1024, 1.75 / 1024, 0.25, 0.5, 0.75, 1, 2, 3, 4, 5, 6, 7, 128, 256, 512, 1024]:
        r.store(0, v)
        assert r[0] == v


def test_custom_float_signed_exact_and_ftz():
    # test_custom_float_exponents.py:33-62
    r = Rec([fexp(13, 6, signed=True)])
    for v in [0, 0.125, 0.5, 2, 4, 6, 7, 8, 9]:
        r.store(0, v)
        assert r[0] == v
        r.store(0, -v)
        assert r[0] == -v
    for v in [1e-30, 1e-20, 1e-10, 1e-2]:
        r.store(0, v)
        assert r[0] == approx(v, abs=1e-5)
        r.store(0, -v)
        assert r[0] == approx(-v, abs=1e-5)


@pytest.mark.parametrize("digits_bits", [23, 24])
def test_custom_float_precision(digits_bits):
    # test_custom_float_exponents.py:65-86
    r = Rec([fexp(digits_bits, 8, signed=True)])
    for v in [np.float32(np.pi), np.float32(np.pi * (1 << 100))]:
        r.store(0, float(v))
        if digits_bits == 24:
            assert np.float32(r[0]) == v
        else:
            assert np.float32(r[0]) != v
            assert r[0] == approx(float(v), rel=3e-7)


@pytest.mark.parametrize("signed", [True, False])
def test_custom_float_truncation(signed):
    # test_custom_float_exponents.py:89-116
    r = Rec([fexp(2, 5, signed=signed)])
    for v in [1, 1.5]:
        r.store(0, v)
        assert r[0] == v
    r.store(0, 1.75)
    assert r[0] == (2 if signed else 1.75)
    r.store(0, 1.625)
    assert r[0] == (1.5 if signed else 1.75)


# ---------------------------------------------- test_custom_float_shared_exp.py


def _shared(ebits, b_signed=False):
    return Rec([shexp(10, ebits, False), shexp(14, ebits, b_signed)])


@pytest.mark.parametrize("ebits", [5, 6, 7, 8])
def test_shared_exponents(ebits):
    # test_custom_float_shared_exp.py:7-72
    r = _shared(ebits)
    assert r[0] == 0.0 and r[1] == 0.0
    r.store(0, 10)
    assert r[0] == 10.0 and r[1] == 0.0
    r.store(0, 0)
    assert r[0] == 0.0 and r[1] == 0.0
    r.assign([3.2, 0.25])
    assert r[0] == approx(3.2, rel=1e-3) and r[1] == approx(0.25, rel=2e-2)
    r.store(0, 0.27)
    assert r[0] == approx(0.27, rel=1e-2) and r[1] == approx(0.25, rel=2e-2)
    r.store(0, 100)
    assert r[0] == approx(100, rel=1e-3) and r[1] == approx(0.25, rel=1e-2)
    r.store(1, 0)
    assert r[0] == approx(100, rel=1e-3) and r[1] == 0
    r.assign([0, 0])
    assert r[0] == 0.0 and r[1] == 0.0
    r.assign([1000, 1e-6])  # flush to zero
    assert r[0] == 1000.0 and r[1] == 0.0
    r.assign([1000, 1000])
    assert r[0] == 1000.0 and r[1] == 1000.0
    r.assign([1e-30, 1e-30])
    if ebits == 8:
        assert r[0] == approx(1e-30, rel=1e-3) and r[1] == approx(1e-30, rel=1e-4)
    else:
        assert r[0] == 0 and r[1] == 0


@pytest.mark.parametrize("ebits", [5, 6, 7, 8])
def test_shared_exponent_add(ebits):
    # test_custom_float_shared_exp.py:75-112
    r = _shared(ebits)
    r.store(0, 4)
    assert r[0] == 4 and r[1] == 0
    r.store(1, 3)
    assert r[0] == 4 and r[1] == 3
    r.store(1, r[1] + 1)
    assert r[0] == 4 and r[1] == 4
    for i in range(100):
        r.store(0, r[0] + 4)
        r.store(1, r[1] + 1)
        assert r[0] == 4 + (i + 1) * 4
        assert r[1] == 4 + (i + 1)


@pytest.mark.parametrize("ebits", [5, 6, 7, 8])
def test_shared_exponent_borrow(ebits):
    # test_custom_float_shared_exp.py:115-144
    r = _shared(ebits)
    r.assign([0, 100])
    for i in range(100):
        assert r[0] == i and r[1] == 100 - i
        r.store(0, r[0] + 1)
        r.store(1, r[1] - 1)


@pytest.mark.parametrize("ebits", [5, 6, 7, 8])
def test_shared_exponent_negative(ebits):
    # test_custom_float_shared_exp.py:147-165
    r = _shared(ebits, b_signed=True)
    r.store(0, 37)
    assert r[0] == 37
    r.store(1, -123)
    assert r[1] == -123


def test_raw_fields_roundtrip():
    L = O.build_layout([(RAW_F32, 32, 1, 0, -1, 0, 0), (RAW_F64, 64, 1, 0, -1, 0, 0), fixed(7)])
    assert L.off[1] == 32 and L.off[2] == 96
    vals = np.array([[np.float32(1.1), 1.1, 0.25]])
    out = O.decode(L, O.encode(L, vals))
    assert out[0, 0] == np.float32(1.1) and out[0, 1] == 1.1 and out[0, 2] == 0.25


# ------------------------------------------------------ SDF collider (oracle)

def test_oracle_collider_holds_a_block_on_a_static_slab():
    """sdf_collision with omega 0: grid velocities into a slab (normal up)
    are removed, so a block resting on it stops falling, while the same
    block without the collider keeps falling."""
    import oracle as Orc

    n = 2000
    rng = np.random.default_rng(0)
    x = np.column_stack([0.45 + 0.1 * rng.random(n), 0.40 + 0.1 * rng.random(n), 0.45 + 0.1 * rng.random(n)])
    vals = np.zeros((n, 24))
    vals[:, :3] = x
    vals[:, 15] = vals[:, 19] = vals[:, 23] = 1.0
    P = {"dim": 3, "precision": 0, "res": [32, 32, 32], "lb": [3, 3, 3], "ub": [29, 29, 29], "has_F": 1,
         "has_mat": 0, "materials": [(1, 50.0, 50.0)], "use_friction": 0, "use_bound_clip": 0,
         "dx": 1 / 32, "dt": 1e-4, "p_vol": (0.5 / 32) ** 3, "p_mass": (0.5 / 32) ** 3, "gravity": 9.8, "seed": 0}
    L = Orc.build_layout([(4, 32, 1, 0, 0, 0.0, 0.0)] * 24, False, False)  # raw f32 slots
    sdf = np.full((32, 32, 32), 0.02, dtype=np.float32)
    sdf[:, 10:13, :] = -0.01  # slab under the block (block bottom at y = 0.40 -> node 12.8)
    nrm = np.zeros((32, 32, 32, 3), dtype=np.float32)
    nrm[..., 1] = 1.0
    ys = []
    for col in (False, True):
        o = Orc.Sim(P, L)
        o.set_state(vals)
        if col:
            o.set_collider(sdf, nrm, offset=(0, 0, 0), center=16, omega=0.0, height_rate=0.0)
        o.substeps(1000)
        ys.append(o.get_state()[:, 1].min())
    assert ys[0] < 0.40 - 0.04  # free fall over 0.1 s: 0.5 g t^2 = 0.049
    assert ys[1] > 0.375 - 0.01  # held at the slab's top (node 13 = 0.406, stencil reach one cell)


# taichi_submission/tests/python/test_custom_float_time_integration.py:10-66:
# midpoint integration of a point around the unit circle, 1000 steps of
# 2 pi / 1000, the position stored after every step as f32, as a 16-bit
# fixed point with scale 2^-14 (range 2), as floats with 13-bit signed
# significands and their own 6-bit exponents, or with one shared 6-bit
# exponent; the position after half a turn must be (-1, 0) and after a
# full turn (1, 0) to 2e-2 (3e-2 for the final y).
@pytest.mark.parametrize("kind", ["f32", "fixed", "exponent", "shared"])
def test_custom_float_time_integration(kind):
    specs = {"f32": None,
             "fixed": [fixed(16, 2.0)] * 2,
             "exponent": [fexp(13, 6)] * 2,
             "shared": [shexp(13, 6, True)] * 2}[kind]
    L = O.build_layout(specs) if specs else None

    def store(p):
        p = np.asarray(p, dtype=np.float32).astype(np.float64)
        return p if L is None else O.decode(L, O.encode(L, p[None]))[0]

    def v_at(p):
        return np.array([-p[1], p[0]], dtype=np.float32)

    x = store([1.0, 0.0])
    n = 1000
    dt = np.float32(math.pi * 2 / n)
    px, py = [], []
    for _ in range(n):
        xf = x.astype(np.float32)
        v_mid = v_at(xf + np.float32(0.5) * dt * v_at(xf))
        x = store(xf + v_mid * dt)
        px.append(x[0])
        py.append(x[1])
    assert px[n // 2 - 1] == approx(-1, abs=2e-2)
    assert py[n // 2 - 1] == approx(0, abs=2e-2)
    assert px[-1] == approx(1, abs=2e-2)
    assert py[-1] == approx(0, abs=3e-2)


def test_custom_int_implicit_cast():
    # test_custom_int.py:4-16: a float stored into int(13, signed) truncates
    L = O.build_layout([qint(13, True)])
    assert O.decode(L, O.encode(L, np.array([[10.3]])))[0, 0] == 10
    assert O.decode(L, O.encode(L, np.array([[-10.7]])))[0, 0] == -10


def test_bit_struct_load_and_store():
    # test_bit_struct.py:38-78 (13/14/5-bit fields) and :92-133 (three
    # fields of the given widths at their extreme and ordinary values)
    L = O.build_layout([qint(13, True), qint(14, False), qint(5, True)])
    cases = np.array([[2**12 - 1, 2**14 - 1, -(2**3)], [2**11 - 1, 2**13 - 1, -(2**2)],
                      [0, 0, 0], [123, 4567, 8], [10, 31, 11]], dtype=np.float64)
    assert (O.decode(L, O.encode(L, cases)) == cases).all()
    for bits, vals in [([3, 3, 2], [2**2 - 1, 2**3 - 1, -2**1]), ([4, 7, 5], [2**3 - 1, 2**7 - 1, -2**4]),
                       ([17, 11, 4], [2**16 - 1, 2**10 - 1, -2**3]), ([32, 23, 9], [2**31 - 1, 2**23 - 1, -2**8]),
                       ([7, 12, 13], [2**6 - 1, 2**12 - 1, -2**12]), ([18, 22, 24], [2**17 - 1, 2**22 - 1, -2**23]),
                       ([5, 5, 6], [15, 5, 20]), ([10, 10, 12], [11, 19, 2020])]:
        L = O.build_layout([qint(bits[0], True), qint(bits[1], False), qint(bits[2], True)])
        v = np.array([vals], dtype=np.float64)
        assert (O.decode(L, O.encode(L, v)) == v).all(), bits


def test_custom_int_full_struct():
    # test_bit_struct.py:81-90: a 32-bit signed int filling its word
    L = O.build_layout([qint(32, True)])
    for v in (15, 12, -2**31, 2**31 - 1):
        assert O.decode(L, O.encode(L, np.array([[v]], dtype=np.float64)))[0, 0] == v
