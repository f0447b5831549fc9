"""Build ``oracle/_ref/libsolve3d_ref.so`` from the reference's own C source.

TEST INFRASTRUCTURE ONLY.  Compiles TT-Toolbox's ``fmex/solve3d.c`` where it
lies in the reference tree (nothing is copied into this repository) against
the MEX/BLAS/LAPACK stand-ins in ``oracle/ref_shim/`` and links numpy's
ILP64 OpenBLAS, so that the reference's own ``dgmresr_hh`` (Householder
GMRES, ``fmex/solve3d.c:339-518``), ``bfun3`` (``:141-195``) and the centre
block-Jacobi routines ``dcjacgen``/``dcjacapply`` (``:47-139``) can be called
through ctypes to pin the oracle's restatements (``tests/test_oracle_ref.py``).

Usage: ``python oracle/build_ref.py <TT-Toolbox source tree>``; the output
goes to ``oracle/_ref/`` only.  Returns the library path, or None when the
reference tree or numpy's OpenBLAS is missing.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libsolve3d_ref.so")


def openblas64():
    import numpy
    libs = glob.glob(os.path.join(os.path.dirname(os.path.dirname(numpy.__file__)),
                                  "numpy.libs", "libscipy_openblas64_*.so"))
    return libs[0] if libs else None


def build(ref_root):
    src = os.path.join(ref_root, "fmex", "solve3d.c")
    blas = openblas64()
    if not os.path.exists(src) or blas is None:
        return None
    shim = os.path.join(HERE, "ref_shim")
    stubs = os.path.join(shim, "mex_stubs.c")
    deps = [src, stubs] + glob.glob(os.path.join(shim, "*.h"))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-w", "-I", shim, src, stubs, "-o", LIB, blas,
           "-Wl,-rpath," + os.path.dirname(blas), "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("building the reference checker failed:\n" + r.stderr)
    return LIB


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python oracle/build_ref.py <TT-Toolbox source tree>")
    print(build(sys.argv[1]))
