"""AMEn approximate matvec (ttg_amen_mv, core/amen_mv.m) against the FP64
oracle restatement from the same initial y0 / z0, and against the exact
product."""
import numpy as np
import pytest

import ttgpu
from oracle.amen_mv import amen_mv as o_amen_mv
from oracle.builders import aniso_config, laplace_config
from oracle.tt import TT, tt_matvec, tt_norm, tt_rand, tt_randn

pytestmark = pytest.mark.gpu


def host_tt(t):
    return ttgpu.TensorTrain(t.n, t.r, t.flat())


def host_mat(A):
    return ttgpu.TTMatrix(A.n, A.m, A.r, A.flat())


def back(t):
    return TT.from_flat(t.n, t.r, t.core)


@pytest.mark.parametrize("cfg", [dict(d=6, n=8, rx=5, kick=4), dict(d=5, n=16, rx=9, kick=4),
                                 dict(d=4, n=6, rx=3, kick=0)])
def test_amen_mv_tight_tolerance_parity(ctx, cfg):
    """Tight tolerance: both implementations agree to 1e-10; with enrichment
    (kickrank > 0) y reaches the exact (rank ra*rx) product, without it the
    ranks stay those of y0 (plain ALS, as in the reference) and y is the
    converged rank-2 approximation."""
    A, _, _, _ = aniso_config(d=cfg["d"], n=cfg["n"])
    rng = np.random.default_rng(cfg["d"] * 10 + cfg["n"])
    x = tt_randn(cfg["n"], cfg["d"], cfg["rx"], rng)
    y0 = tt_rand(cfg["n"], cfg["d"], 2, np.random.default_rng(1))
    z0 = tt_rand(cfg["n"], cfg["d"], max(cfg["kick"], 1), np.random.default_rng(2))
    ex = tt_matvec(A, x)
    ref, _, info = o_amen_mv(A, x, 1e-12, y0, z0, kickrank=cfg["kick"])
    got, z, sweeps = ttgpu.amen_mv(host_mat(A), host_tt(x), 1e-12, y0=host_tt(y0),
                                   z0=host_tt(z0), kickrank=cfg["kick"], ctx=ctx)
    got = back(got)
    assert sweeps == info["sweeps"]
    assert list(got.r) == list(ref.r)
    assert tt_norm(got - ref) <= 1e-10 * tt_norm(ref)
    if cfg["kick"]:
        assert tt_norm(got - ex) <= 1e-10 * tt_norm(ex)
        assert z is not None and z.d == cfg["d"]
    else:
        assert max(got.r) == 2 and z is None


def test_amen_mv_loose_tolerance(ctx):
    """Loose tolerance: the approximation error tracks tol, like the oracle's."""
    A, _, _, _ = laplace_config(d=8, n=16)
    rng = np.random.default_rng(5)
    x = tt_randn(16, 8, 6, rng)
    ex = tt_matvec(A, x)
    y0 = tt_rand(16, 8, 2, np.random.default_rng(1))
    z0 = tt_rand(16, 8, 4, np.random.default_rng(2))
    ref, _, info = o_amen_mv(A, x, 1e-4, y0, z0)
    got, _, sweeps = ttgpu.amen_mv(host_mat(A), host_tt(x), 1e-4, y0=host_tt(y0),
                                   z0=host_tt(z0), ctx=ctx)
    got = back(got)
    eg, er = tt_norm(got - ex) / tt_norm(ex), tt_norm(ref - ex) / tt_norm(ex)
    assert eg < 1e-3 and er < 1e-3
    assert abs(sweeps - info["sweeps"]) <= 1
    # random initial guesses drawn on the device also work
    got2, _, _ = ttgpu.amen_mv(host_mat(A), host_tt(x), 1e-8, ctx=ctx)
    assert tt_norm(back(got2) - ex) <= 1e-6 * tt_norm(ex)


def test_amen_mv_errors(ctx):
    A, _, _, _ = laplace_config(d=4, n=4)
    x = tt_randn(5, 4, 2, np.random.default_rng(0))
    with pytest.raises(ttgpu.TTGError, match="square A cores"):
        ttgpu.amen_mv(host_mat(A), host_tt(x), 1e-6, ctx=ctx)
    with pytest.raises(ttgpu.TTGError, match="tol"):
        ttgpu.amen_mv(host_mat(A), host_tt(tt_randn(4, 4, 2, np.random.default_rng(0))), -1.0,
                      ctx=ctx)
