"""Loader of the committed golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

from oracle.tt import TT, TTMatrix

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture(key):
    """(A, rhs, x_stored, residual) of the reference system ``key``."""
    g = np.load(os.path.join(GOLDEN, "ttsolve_%s.npz" % key))
    A = TTMatrix.from_flat(g["A_n"], g["A_m"], g["A_r"], g["A_core"])
    rhs = TT.from_flat(g["rhs_n"], g["rhs_r"], g["rhs_core"])
    x = TT.from_flat(g["x_n"], g["x_r"], g["x_core"])
    return A, rhs, x, float(g["residual"])


def load_sdv(name):
    """(header fields, bytes) of the reference's SDV file ``name`` ('A' or 'b'),
    rebuilt from the fixture; the bytes hash to the recorded SHA-256."""
    from oracle import sdv
    g = np.load(os.path.join(GOLDEN, "sdv_%s.npz" % name))
    hd = dict(txt=g["txt"].tobytes(), ver=tuple(int(v) for v in g["ver"]),
              inf=tuple(int(v) for v in g["inf"]), comment=g["comment"].tobytes(),
              i=tuple(int(v) for v in g["i"]), lm=tuple(int(v) for v in g["lm"]))
    data = sdv.write(hd, g["n"], g["r"], g["core"])
    assert sdv.sha256(data) == str(g["sha256"]), "fixture does not rebuild the reference file"
    return hd, g, data
