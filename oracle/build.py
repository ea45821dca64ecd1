"""ORACLE - test infrastructure only.  Builds oracle/_build/libaqoracle.so
from the C restatement in this folder with plain gcc (no build system):

    python oracle/build.py

The codec unit is compiled once; the substep unit twice (REAL=float and
REAL=double).  -ffp-contract=off keeps every multiply and add separately
rounded, as the reference's LLVM IR states them.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libaqoracle.so")
SRCS = ["aq_oracle.h", "aq_oracle_codec.c", "aq_oracle_mpm.c", "aq_oracle_emit.c"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(os.path.join(HERE, s)) > t for s in SRCS)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    os.makedirs(OUT, exist_ok=True)
    cflags = ["-O2", "-fPIC", "-std=c99", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-Wall"]
    objs = []
    units = [
        ("aq_oracle_codec.c", "codec.o", []),
        ("aq_oracle_mpm.c", "mpm_f32.o", ["-DREAL=float", "-DSUF(x)=x##_f32"]),
        ("aq_oracle_mpm.c", "mpm_f64.o", ["-DREAL=double", "-DSUF(x)=x##_f64"]),
        ("aq_oracle_emit.c", "emit.o", []),
    ]
    for src, obj, defs in units:
        o = os.path.join(OUT, obj)
        cmd = ["gcc", *cflags, *defs, "-c", os.path.join(HERE, src), "-o", o]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        objs.append(o)
    tmp = LIB + ".tmp"
    subprocess.check_call(["gcc", "-shared", "-fopenmp", "-o", tmp, *objs, "-lm"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
