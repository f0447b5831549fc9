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
