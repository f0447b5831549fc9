"""Build libttgpu.so (all CUDA sources, sm_100a) in-tree.

``python -m ttgpu.build`` (from ``tt-toolbox_b200/``) or ``build()`` from
Python.  Objects go to ``tt-toolbox_b200/_build/``; the shared library is
written next to this file so it travels with the source tree.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
CSRC = os.path.join(PKG_ROOT, "csrc")
BUILD = os.path.join(PKG_ROOT, "_build")
LIB = os.path.join(HERE, "libttgpu.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no contraction of separate multiplies and adds into FMAs, so
# a kernel body computes bit-identical results in every instantiation (its
# plain launch and the grouped launch of a grouped batch); FMAs the code
# wants are written as fma().
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
          "--expt-relaxed-constexpr",
          "-Xcompiler", "-Wall", "-Xcompiler", "-Wno-unused-function"]
LIBS = ["-lcusolver", "-lcublas", "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(os.path.dirname(PKG_ROOT), "include", "ttgpu.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def _compile(src, extra, verbose):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()):
        return obj
    cmd = [NVCC, "-c", src, "-o", obj] + ARCH + CFLAGS + extra
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    if verbose and (r.stdout.strip() or r.stderr.strip()):
        print(r.stdout, r.stderr, flush=True)
    return obj


def _flags_changed(extra):
    """True (and the stamp rewritten) when the compile flags differ from the
    ones the objects in _build/ were made with."""
    stamp = os.path.join(BUILD, "flags.txt")
    now = " ".join(ARCH + CFLAGS + list(extra))
    old = open(stamp).read() if os.path.exists(stamp) else None
    if old != now:
        with open(stamp, "w") as f:
            f.write(now)
        return True
    return False


def build(verbose=False, extra=()):
    """Compile every ``csrc/*.cu`` for sm_100a and link ``libttgpu.so``."""
    os.makedirs(BUILD, exist_ok=True)
    if _flags_changed(extra):
        for f in os.listdir(BUILD):
            if f.endswith(".o"):
                os.remove(os.path.join(BUILD, f))
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, list(extra), verbose), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC, "-shared", "-o", LIB] + objs + ARCH + LIBS
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(verbose=True, extra=extra))
