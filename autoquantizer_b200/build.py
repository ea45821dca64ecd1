"""Build libaq.so (the sm_100a kernels and the C ABI of include/aq.h) in-tree.

    python -m autoquantizer_b200.build [--force] [--verbose]

Each .cu under csrc/ is compiled by nvcc for sm_100a (in parallel), then
linked into autoquantizer_b200/libaq.so.  The shared object travels with the
source tree; nothing is installed.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libaq.so")
GENCODE = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hdrs + [os.path.join(ROOT, "include", "aq.h")]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    files = [os.path.join(CSRC, s) for s in sources()] + _deps()
    return any(os.path.getmtime(f) > t for f in files)


# headers compiled again at run time by NVRTC (layout-specialized k_step);
# the names are the include strings the sources use
JIT_HEADERS = [("aq_kernels.cuh", os.path.join(CSRC, "aq_kernels.cuh")),
               ("aq_codec.cuh", os.path.join(CSRC, "aq_codec.cuh")),
               ("aq_step_config.h", os.path.join(CSRC, "aq_step_config.h")),
               ("../../include/aq.h", os.path.join(ROOT, "include", "aq.h"))]


def write_jit_sources():
    """Embed the kernel headers into the library as C string literals."""
    out = ["// generated by autoquantizer_b200/build.py: headers for NVRTC", ""]
    names, srcs = [], []
    for i, (name, path) in enumerate(JIT_HEADERS):
        text = open(path).read()
        assert ")AQSRC" not in text
        out.append('static const char kAqJitSrc%d[] = R"AQSRC(%s)AQSRC";' % (i, text))
        names.append('"%s"' % name)
        srcs.append("kAqJitSrc%d" % i)
    out.append("static const int kAqJitHeaderCount = %d;" % len(JIT_HEADERS))
    out.append("static const char* const kAqJitHeaderName[] = {%s};" % ", ".join(names))
    out.append("static const char* const kAqJitHeaderSrc[] = {%s};" % ", ".join(srcs))
    path = os.path.join(OUT, "aq_jit_sources.inc")
    text = "\n".join(out) + "\n"
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)


def build(force=False, verbose=False, extra=()):
    if not force and not stale():
        return LIB
    os.makedirs(OUT, exist_ok=True)
    write_jit_sources()
    flags = [GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
             "-I" + os.path.join(ROOT, "include"), "-I" + OUT, *extra]
    if verbose:
        flags += ["-Xptxas", "-v"]

    def compile_one(src):
        obj = os.path.join(OUT, src[:-3] + ".o")
        cmd = [nvcc(), *flags, "-c", os.path.join(CSRC, src), "-o", obj]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), p.stderr))
        return obj, p.stderr

    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, sources()))
    if verbose:
        for _, err in results:
            if err:
                print(err)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), GENCODE, "-shared", "-o", tmp, *[r[0] for r in results], "-lcudart", "-ldl"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
