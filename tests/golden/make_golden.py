"""Convert the reference's fixtures into .npz.

(1) Known-answer linear systems.

The reference ships ``tests/tt-solve/*.mat`` (``tests/tt-solve/README:1-16``):
each holds a TT matrix ``A``, a right-hand side ``rhs`` and the published
approximate solution ``x`` (Dolgov & Oseledets 2011).  The GPU box has no copy
of the reference tree, so this script (run once, here) stores the flat cores
and shapes of the small ones as compressed ``.npz`` next to itself, plus the
relative residual ``||A x - rhs|| / ||rhs||`` recomputed by the oracle.

(2) The SDV TT files ``fmex/A.sdv`` and ``fmex/b.sdv`` (a QTT operator of 80
2x2 cores and a right-hand side): parsed header fields, shapes, cores and
the SHA-256 of the original bytes, so the tests can rebuild the exact files.

Usage: ``python tests/golden/make_golden.py <path-to-TT-Toolbox>`` (required).
"""
import os
import sys

import numpy as np
import scipy.io as sio

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import sdv  # noqa: E402
from oracle.tt import TT, TTMatrix, true_residual  # noqa: E402

FILES = {
    "ex2": "tt-solve_ex2_6-10.mat",
    "ex2_1": "tt-solve_ex2.1_6-8.mat",
    "ex6": "tt-solve_ex6.mat",
}


def _iv(v):
    return np.asarray(v, dtype=np.float64).ravel().astype(np.int64)


def load_mat(path):
    m = sio.loadmat(path, struct_as_record=False, squeeze_me=False)

    def tt_of(o):
        o = o[0, 0] if hasattr(o, "shape") else o
        return TT.from_flat(_iv(o.n), _iv(o.r), np.asarray(o.core, dtype=np.float64).ravel())

    Am = m["A"][0, 0]
    tt = Am.tt[0, 0] if hasattr(Am.tt, "shape") else Am.tt
    A = TTMatrix.from_flat(_iv(Am.n), _iv(Am.m), _iv(tt.r), np.asarray(tt.core, dtype=np.float64).ravel())
    return A, tt_of(m["rhs"]), tt_of(m["x"])


def main(ref_root):
    for key, fname in FILES.items():
        A, rhs, x = load_mat(os.path.join(ref_root, "tests", "tt-solve", fname))
        res = true_residual(A, x, rhs)
        np.savez_compressed(
            os.path.join(HERE, "ttsolve_%s.npz" % key),
            A_n=A.n, A_m=A.m, A_r=A.r, A_core=A.flat(),
            rhs_n=rhs.n, rhs_r=rhs.r, rhs_core=rhs.flat(),
            x_n=x.n, x_r=x.r, x_core=x.flat(),
            residual=np.float64(res), source=np.array(fname))
        print(key, fname, "d=%d" % A.d, "max rank x=%d" % x.r.max(), "residual=%.3e" % res)
    for name in ("A", "b"):
        data = open(os.path.join(ref_root, "fmex", name + ".sdv"), "rb").read()
        f = sdv.parse(data)
        assert sdv.write(f, f["n"], f["r"], f["core"]) == data
        np.savez_compressed(
            os.path.join(HERE, "sdv_%s.npz" % name), txt=np.frombuffer(f["txt"], np.uint8),
            ver=np.array(f["ver"]), inf=np.array(f["inf"]),
            comment=np.frombuffer(f["comment"], np.uint8), i=np.array(f["i"]),
            lm=np.array(f["lm"]), n=f["n"], r=f["r"], core=f["core"],
            sha256=np.array(sdv.sha256(data)), source=np.array("fmex/%s.sdv" % name))
        print(name + ".sdv", "d=%d" % f["d"], "max rank %d" % f["r"].max(), sdv.sha256(data))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <TT-Toolbox source tree>")
    main(sys.argv[1])
