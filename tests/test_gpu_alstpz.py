"""``ttg_alstpz_solve`` (``solve/alstpz_solve.m``, ALS(t+z), kicktype 'svd')
against the FP64 oracle ``oracle/alstpz.py`` on the same seeded inputs,
through the C ABI.

With every local system solved densely (``max_full_size`` above every local
size, LU on both sides) the two implementations differ by rounding only:
identical ranks after every sweep and 1e-10 TT-relative difference.  With
the default branch rule the local GMRES stops at its tolerance
(``(tol/sqrt(d))/resid_damp``), so two implementations whose rounding
differs may stop one Krylov step apart: the ranks must still agree, the
solutions within the solve tolerance, and the true residual must reach it.
"""
import numpy as np
import pytest

import ttgpu
from oracle.alstpz import alstpz_solve
from oracle.builders import aniso_config, laplace_config
from oracle.tt import TT, true_residual, tt_norm

pytestmark = pytest.mark.gpu


def _gpu(A, y, x0, tol, **kw):
    st = {}
    got = ttgpu.alstpz_solve(ttgpu.TTMatrix(A.n, A.m, A.r, A.flat()),
                             ttgpu.TensorTrain(y.n, y.r, y.flat()), tol,
                             x0=ttgpu.TensorTrain(x0.n, x0.r, x0.flat()), stats=st, **kw)
    return TT.from_flat(got.n, got.r, got.core), st


@pytest.mark.parametrize("d,n", [(4, 8), (5, 8)])
def test_alstpz_dense_local_solves_match_oracle(ctx, d, n):
    A, y, x0, _ = laplace_config(d=d, n=n)
    big = 10 ** 9
    ref, info = alstpz_solve(A, y, 1e-8, x0, max_full_size=big)
    got, st = _gpu(A, y, x0, 1e-8, max_full_size=big)
    assert st["sweeps"] == 10 and st["local_solves"] == 0
    assert list(got.r) == list(ref.r)
    assert tt_norm(got - ref) <= 1e-10 * tt_norm(ref)
    # The local residuals after each sweep's rounding differ by the rounding
    # (both truncate to tol at the same ranks, along different rounding
    # errors): 2e-8 absolute measured at res_prev = 3e-4.
    np.testing.assert_allclose(st["max_res"], info["max_res"], rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("cfg", ["lap6", "lap8", "aniso5"])
def test_alstpz_gmres_matches_oracle(ctx, cfg):
    if cfg == "lap6":
        A, y, x0, _ = laplace_config(d=6, n=16)
    elif cfg == "lap8":
        A, y, x0, _ = laplace_config(d=8, n=32)
    else:
        A, y, x0, _ = aniso_config(d=5, n=16, seed=2)
    tol = 1e-8
    ref, info = alstpz_solve(A, y, tol, x0)
    got, st = _gpu(A, y, x0, tol)
    assert st["sweeps"] == 10 and st["local_solves"] > 0
    assert list(got.r) == list(ref.r)
    assert tt_norm(got - ref) <= tol * tt_norm(ref)
    res_ref, res_got = true_residual(A, ref, y), true_residual(A, got, y)
    assert res_got <= max(1e-8, 2 * res_ref), (res_got, res_ref)
    np.testing.assert_allclose(st["max_res"][0], info["max_res"][0], rtol=1e-6)


def test_alstpz_mixed_reaches_the_tolerance(ctx):
    """BF16 tcgen05 local matvecs with FP64 refinement inside the same
    sweeps: the local solves meet the same FP64 tolerance."""
    A, y, x0, _ = laplace_config(d=6, n=16)
    ref, _ = alstpz_solve(A, y, 1e-8, x0)
    got, st = _gpu(A, y, x0, 1e-8, precision="mixed")
    assert st["sweeps"] == 10
    assert true_residual(A, got, y) <= max(1e-8, 2 * true_residual(A, ref, y))


def test_alstpz_options_and_errors(ctx):
    A, y, x0, _ = laplace_config(d=4, n=8)
    with pytest.raises(ValueError, match="Unrecognized option"):
        _gpu(A, y, x0, 1e-8, bogus=1)
    with pytest.raises(ttgpu.TTGError):
        _gpu(A, y, x0, 1e-8, kicktype="als")
    got, st = _gpu(A, y, x0, 1e-8, nswp=3, kickrank=0)
    assert st["sweeps"] == 3
    # without an initial guess a device-drawn rank-2 TT starts the sweeps
    st2 = {}
    x = ttgpu.alstpz_solve(ttgpu.TTMatrix(A.n, A.m, A.r, A.flat()),
                           ttgpu.TensorTrain(y.n, y.r, y.flat()), 1e-8, stats=st2)
    assert true_residual(A, TT.from_flat(x.n, x.r, x.core), y) < 1e-8
