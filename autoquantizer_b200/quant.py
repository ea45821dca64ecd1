"""Quantized scalar types and the bit_pack record layout.

Mirrors the reference's type constructors (taichi_submission/python/taichi/
lang/quant_impl.py:12-73) and `SNode.bit_pack().place(...)` (snode.py:108-180)
for one particle record:

    rec = BitPack()
    rec.place(fixed(20, range=1.0), fixed(20, range=1.0))           # x
    rec.place(fixed_float(13, 6), fixed_float(13, 6), shared_exponent=True)  # v
    layout = rec.build()

`build()` resolves bit offsets through libaq's aq_layout_build (the single
layout implementation of the product).
"""
import ctypes as C
from dataclasses import dataclass

from . import _lib


@dataclass(frozen=True)
class Fixed:
    """ti.quant.fixed(frac, signed, range, offset, compute, use_dithering):
    `bits` total bits including the sign bit; scale = range / 2^(bits-1)
    (signed) or range / 2^bits (unsigned)."""
    bits: int
    signed: bool = True
    range: float = 1.0
    offset: float = 0.0
    compute: str = "f32"
    use_dithering: bool = False

    @property
    def scale(self):
        return self.range / 2 ** (self.bits - 1) if self.signed else self.range / 2 ** self.bits


@dataclass(frozen=True)
class Int:
    """ti.quant.int(bits, signed)."""
    bits: int
    signed: bool = False


@dataclass(frozen=True)
class Float:
    """ti.quant.float(exp, frac, signed): `bits` digits incl. sign, its own
    (or, placed with shared_exponent=True, a shared) exponent of exp_bits."""
    bits: int
    exp_bits: int
    signed: bool = True


@dataclass(frozen=True)
class Raw:
    """An unquantized IEEE value (f32 or f64) stored in the record."""
    f64: bool = False


def fixed(frac, signed=True, range=1.0, offset=0.0, compute="f32", use_dithering=False):
    return Fixed(int(frac), bool(signed), float(range), float(offset), compute, bool(use_dithering))


def qint(bits, signed=False):
    return Int(int(bits), bool(signed))


def qfloat(frac, exp, signed=True):
    return Float(int(frac), int(exp), bool(signed))


class BitPack:
    """Ordered list of scalars of one particle record (place order)."""

    def __init__(self):
        self.items = []  # (type, shared group id or None)
        self._next_group = 0

    def place(self, *types, shared_exponent=False):
        group = None
        if shared_exponent:
            group = self._next_group
            self._next_group += 1
            if not all(isinstance(t, Float) for t in types):
                raise TypeError("shared_exponent needs quant floats")
            if len({t.exp_bits for t in types}) != 1:
                raise TypeError("types with a shared exponent must share the exponent type")
        for t in types:
            self.items.append((t, group))
        return self

    def specs(self):
        out = []
        for t, g in self.items:
            s = _lib.ScalarSpec()
            if isinstance(t, Fixed):
                s.kind, s.bits, s.is_signed, s.range, s.offset = _lib.AQ_FIXED, t.bits, int(t.signed), t.range, t.offset
            elif isinstance(t, Int):
                s.kind, s.bits, s.is_signed = _lib.AQ_INT, t.bits, int(t.signed)
            elif isinstance(t, Float):
                s.kind = _lib.AQ_SHARED_EXP if g is not None else _lib.AQ_FLOAT_EXP
                s.bits, s.is_signed, s.exp_bits, s.group = t.bits, int(t.signed), t.exp_bits, g if g is not None else -1
            elif isinstance(t, Raw):
                s.kind, s.bits = (_lib.AQ_RAW_F64, 64) if t.f64 else (_lib.AQ_RAW_F32, 32)
            else:
                raise TypeError(t)
            out.append(s)
        return out

    def spec_tuples(self):
        """(kind, bits, signed, exp_bits, group, range, offset) per scalar."""
        return [(s.kind, s.bits, s.is_signed, s.exp_bits, s.group, s.range, s.offset) for s in self.specs()]

    def compute_and_dithering(self):
        fx = [t for t, _ in self.items if isinstance(t, Fixed)]
        if not fx:
            return False, False
        comp = {t.compute for t in fx}
        dith = {t.use_dithering for t in fx}
        if len(comp) != 1 or len(dith) != 1:
            raise ValueError("all fixed-point types of one record share compute type and dithering")
        return comp.pop() == "f64", dith.pop()

    def build(self):
        specs = self.specs()
        arr = (_lib.ScalarSpec * len(specs))(*specs)
        f64, dith = self.compute_and_dithering()
        L = _lib.Layout()
        _lib.check(_lib.lib().aq_layout_build(len(specs), arr, int(f64), int(dith), C.byref(L)), "aq_layout_build")
        return L


def layout_summary(L):
    return {"n_slots": L.n_slots, "n_words": L.n_words, "total_bits": L.total_bits,
            "bytes_per_record": 8 * L.n_words,
            "offsets": [L.slot[i].bit_offset for i in range(L.n_slots)]}
