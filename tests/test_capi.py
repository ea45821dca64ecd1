"""CPU checks of the C ABI: libaq.so loads, exports every declared symbol,
its structs match the ctypes mirror, and its layout builder agrees with the
oracle's restatement of the reference layout pass."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
from autoquantizer_b200 import _lib
from autoquantizer_b200 import quant as Q

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "aq.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\*?\s+\*?(aq_[a-z_0-9]+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_lib.EXPORTS) == names


def test_abi_version_and_errors():
    L = _lib.lib()
    assert L.aq_abi_version() == 1
    for code, msg in _lib.ERRORS.items():
        if code != -3:
            assert L.aq_error_string(code).decode() == msg


def test_struct_sizes():
    assert C.sizeof(_lib.ScalarSpec) == 40
    assert C.sizeof(_lib.Slot) == 80
    assert C.sizeof(_lib.Layout) == 32 + 80 * _lib.AQ_MAX_SLOTS


def _random_pack(rng):
    rec = Q.BitPack()
    n = 0
    f64 = bool(rng.integers(2))
    dith = bool(rng.integers(2))
    while n < rng.integers(3, 24):
        k = rng.integers(5)
        if k == 0:
            rec.place(Q.fixed(int(rng.integers(1, 33)), bool(rng.integers(2)), float(rng.uniform(0.1, 100)),
                              float(rng.choice([0.0, 1.0])), "f64" if f64 else "f32", dith))
            n += 1
        elif k == 1:
            rec.place(Q.qint(int(rng.integers(1, 33)), bool(rng.integers(2))))
            n += 1
        elif k == 2:
            rec.place(Q.qfloat(int(rng.integers(3, 24)), int(rng.integers(2, 9)), True))
            n += 1
        elif k == 3:
            eb = int(rng.integers(4, 9))
            m = int(rng.integers(1, 4))
            rec.place(*[Q.qfloat(int(rng.integers(3, 15)), eb, bool(rng.integers(2))) for _ in range(m)],
                      shared_exponent=True)
            n += m
        else:
            rec.place(Q.Raw(bool(rng.integers(2))))
            n += 1
    return rec


@pytest.mark.parametrize("seed", range(20))
def test_layout_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    rec = _random_pack(rng)
    if len(rec.items) > 32 or len({g for _, g in rec.items if g is not None}) > 4:
        pytest.skip("over the slot/group limits")
    L = rec.build()
    f64, dith = rec.compute_and_dithering()
    Lo = O.build_layout(rec.spec_tuples(), f64, dith)
    assert L.n_slots == Lo.n and L.n_words == Lo.n_words and L.total_bits == Lo.total_bits
    for i in range(L.n_slots):
        S = L.slot[i]
        assert S.bit_offset == Lo.off[i] and S.bits == Lo.bits[i]
        if S.kind in (_lib.AQ_FLOAT_EXP, _lib.AQ_SHARED_EXP):
            assert S.exp_offset == Lo.eoff[i]
        if S.kind == _lib.AQ_FIXED:
            assert S.scale_f64 == Lo.scale[i]


def test_layout_rejects_bad_widths():
    for bad in ([Q.fixed(0)], [Q.fixed(33)], [Q.qfloat(25, 6)], [Q.qfloat(10, 9)]):
        rec = Q.BitPack()
        rec.place(*bad)
        with pytest.raises(_lib.AqError):
            rec.build()


def test_dam_break_record_is_152_bits():
    from autoquantizer_b200 import scenes
    from autoquantizer_b200.mpm_config import MPMConfig  # noqa: F401

    cfg, _ = scenes.dam_break_2d(n=16)
    # built without a GPU: only the layout
    rec = Q.BitPack()
    rec.place(Q.fixed(20, range=1.0, use_dithering=True), Q.fixed(20, range=1.0, use_dithering=True))
    rec.place(Q.qfloat(13, 6), Q.qfloat(13, 6), shared_exponent=True)
    rec.place(*[Q.fixed(16, range=64.0, use_dithering=True)] * 4)
    rec.place(Q.fixed(16, range=0.5, offset=1.0, use_dithering=True))
    L = rec.build()
    assert L.total_bits == 152 and L.n_words == 3
    assert cfg.v_exp_bits == 6


def test_every_entry_point_is_mapped_to_a_reference_interface():
    """include/aq_reference_map.json names, for every function include/aq.h
    declares, the reference interface it replaces (families may be named
    with a `*`), and names no function the header does not declare."""
    import json

    with open(os.path.join(ROOT, "include", "aq_reference_map.json")) as f:
        rows = json.load(f)["rows"]
    names = [n for r in rows for n in r["entry_points"]]
    assert all(r["replaces"].strip() for r in rows)
    families = [n[:-1] for n in names if n.endswith("*")]
    exact = set(n for n in names if not n.endswith("*"))
    declared = declared_functions()
    missing = [f for f in declared if f not in exact and not any(f.startswith(p) for p in families)]
    assert not missing, missing
    assert not exact - set(declared), exact - set(declared)


def test_new_entry_points_reject_bad_arguments_before_any_cuda_call():
    """The streamed-mode and append entry points validate their arguments
    first: null handles and pointers, a chunk below one record, a sparse
    grid for a streamed simulator and an empty scene give AQ_E_ARG."""
    L = _lib.lib()
    P = _lib.Params()
    P.dim, P.res[0], P.res[1], P.res[2], P.n_particles = 3, 32, 32, 32, 1000
    P.dx, P.dt = 1.0 / 32, 1e-4
    lay = _lib.Layout()
    sim = C.c_void_p()
    assert L.aq_sim_create_streamed(None, C.byref(lay), 100, C.byref(sim)) == -1
    assert L.aq_sim_create_streamed(C.byref(P), C.byref(lay), 0, C.byref(sim)) == -1
    P.sparse = 1
    assert L.aq_sim_create_streamed(C.byref(P), C.byref(lay), 100, C.byref(sim)) == -1
    P.sparse, P.n_particles = 0, 0
    assert L.aq_sim_create_streamed(C.byref(P), C.byref(lay), 100, C.byref(sim)) == -1
    n, cap = C.c_int64(), C.c_int64()
    assert L.aq_sim_append(None, None, 0, 10, None) == -1
    assert L.aq_sim_set_count(None, 5) == -1
    assert L.aq_sim_count(None, C.byref(n), C.byref(cap)) == -1
    assert L.aq_sim_stream_set_words(None, None, None) == -1
    assert L.aq_sim_stream_get_words(None, None, None) == -1
    assert L.aq_sim_stream_chunks(None, C.byref(n), C.byref(cap)) == -1
