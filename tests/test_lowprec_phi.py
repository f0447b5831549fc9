"""Precision the interface (Phi) contractions need (CPU, oracle only).

The mixed form wants BF16/TF32 Phi/core contractions with FP64
refinement of the local residual.  This measures it on the oracle: the
operands of every ``compute_next_Phi`` product (``solve/amen_solve2.m:834-920``)
are rounded to BF16, TF32 or FP32 (FP64 accumulation, everything else FP64)
on a small anisotropic system (d = 4, n = 16, tol 1e-8, rank cap 256).
The FP64 interfaces reach the tolerance; rounded ones stall at roughly the
operand precision times the operator's conditioning, because the local
systems that the FP64 refinement solves are no longer projections of the
global operator.  So the library keeps the interfaces in FP64 and puts the
low precision in the Krylov matvecs only.
"""
from oracle import amen as oamen
from oracle.builders import aniso_config
from oracle.lowprec_phi import round_to, rounded_phi
from oracle.tt import true_residual

import numpy as np


def _solve(fmt):
    A, y, x0, z0 = aniso_config(d=4, n=16, seed=3)
    if fmt == "fp64":
        x, info = oamen.amen_solve2(A, y, 1e-8, x0, z0, rmax=256, nswp=20)
    else:
        with rounded_phi(fmt):
            x, info = oamen.amen_solve2(A, y, 1e-8, x0, z0, rmax=256, nswp=20)
    return true_residual(A, x, y), len(info["max_res"])


def test_round_to_formats():
    v = np.array([1.0 + 2.0 ** -9, 1.0 + 2.0 ** -8 + 2.0 ** -9, 3.0, -1.0 / 3.0])
    assert round_to(v, "bf16")[0] == 1.0                       # tie to even
    assert round_to(v, "bf16")[1] == 1.0 + 2.0 ** -7            # tie to even (up)
    assert round_to(v, "bf16")[2] == 3.0
    assert abs(round_to(v, "bf16")[3] + 1.0 / 3.0) <= 2.0 ** -9 / 3 * 2
    assert abs(round_to(v, "tf32")[3] + 1.0 / 3.0) <= 2.0 ** -12
    assert round_to(v, "fp32")[3] == np.float32(-1.0 / 3.0)


def test_fp64_interfaces_reach_tolerance_low_precision_ones_stall():
    res64, sw64 = _solve("fp64")
    assert res64 < 1e-8 and sw64 < 20
    res32, _ = _solve("fp32")
    assert res32 > 1e-8                 # even FP32 operands miss 1e-8
    for fmt in ("tf32", "bf16"):
        res, sweeps = _solve(fmt)
        assert res > 1e-5 and sweeps == 20, (fmt, res, sweeps)
