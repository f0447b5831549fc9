"""Failure detection without a GPU fault.

* Every bounded device wait (grid barriers of the Householder GMRES, of the
  cooperative Jacobi SVD and of the Arnoldi kernels; the mbarrier waits of
  the tcgen05 pipeline) is run on a condition that nothing satisfies, with a
  small poll limit: it gives up, the host reads TTG_ERR_TIMEOUT, and the
  context keeps working.
* Non-finite inputs are refused with TTG_ERR_INVALID before any sweep.
* A Jacobi SVD that reaches its sweep limit: ttg_dense_svd and AMEn fail
  with TTG_ERR_NOCONV (MATLAB's svd errors, amen_solve2.m:533); rounding
  takes the fallback SVD as round.m:64-74 falls back to svds, and still
  matches the oracle.
* An AMEn solve that cannot reach its tolerance returns its iterate without
  an error, as the reference does, and its decisions still follow the
  oracle's.
* Degenerate input: rounding the zero tensor gives the rank-1 zero tensor
  (my_chop2.m:18-21, round.m:94-107).
"""
import numpy as np
import pytest

import ttgpu
from oracle import amen as oamen
from oracle.builders import aniso_config, laplace_config, round_config
from oracle.round import tt_round
from oracle.tt import TT, tt_norm, true_residual
from test_gpu_parity import back, host_mat, host_tt, tt_rel

pytestmark = pytest.mark.gpu

TIMEOUT, INVALID, NOCONV = 6, 1, 4


@pytest.mark.parametrize("which", [0, 1, 2, 3])
def test_bounded_wait_gives_up(ctx, which):
    with pytest.raises(ttgpu.TTGError) as e:
        ctx.selftest_wait(which)
    assert e.value.code == TIMEOUT
    # the context is still usable: a local matvec against the oracle
    rng = np.random.default_rng(which)
    Phi1, A, Phi2 = (rng.standard_normal((5, 5, 2)), rng.standard_normal((2, 7, 7, 3)),
                     rng.standard_normal((4, 3, 4)))
    x = rng.standard_normal(5 * 7 * 4)
    y = ttgpu.bfun3(Phi1, A, Phi2, x, ctx=ctx)
    ref = oamen.bfun3(Phi1, A, Phi2, x)
    assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref)


def _poison(t, value):
    core = np.array(t.flat(), dtype=np.float64)
    core[core.size // 2] = value
    return core


@pytest.mark.parametrize("value", [np.nan, np.inf, -np.inf])
def test_nonfinite_inputs_are_refused(ctx, value):
    A, y, x0, z0 = laplace_config(d=4, n=8)
    bad_y = ttgpu.TensorTrain(y.n, y.r, _poison(y, value))
    with pytest.raises(ttgpu.TTGError, match="non-finite") as e:
        ttgpu.amen_solve2(host_mat(A), bad_y, 1e-8, x0=host_tt(x0), z0=host_tt(z0), ctx=ctx)
    assert e.value.code == INVALID
    bad_A = ttgpu.TTMatrix(A.n, A.m, A.r, _poison(A, value))
    with pytest.raises(ttgpu.TTGError, match="non-finite"):
        ttgpu.amen_solve2(bad_A, host_tt(y), 1e-8, x0=host_tt(x0), z0=host_tt(z0), ctx=ctx)
    bad_x0 = ttgpu.TensorTrain(x0.n, x0.r, _poison(x0, value))
    with pytest.raises(ttgpu.TTGError, match="non-finite"):
        ttgpu.amen_solve2(host_mat(A), host_tt(y), 1e-8, x0=bad_x0, z0=host_tt(z0), ctx=ctx)
    x = round_config(d=5, n=4, r=3, terms=2, seed=1)
    with pytest.raises(ttgpu.TTGError, match="non-finite") as e:
        ttgpu.round(ttgpu.TensorTrain(x.n, x.r, _poison(x, value)), 1e-8, ctx=ctx)
    assert e.value.code == INVALID
    with pytest.raises(ttgpu.TTGError, match="non-finite"):
        ttgpu.amen_mv(host_mat(A), ttgpu.TensorTrain(x0.n, x0.r, _poison(x0, value)), 1e-6,
                      ctx=ctx)


@pytest.fixture
def capped_ctx():
    """A context whose Jacobi SVDs stop after one sweep."""
    c = ttgpu.Context(ctx_device())
    c.set_option(ttgpu.Context.OPT_JACOBI_MAX_SWEEPS, 1)
    yield c
    c.close()


def ctx_device():
    import os
    return int(os.environ.get("TTG_DEVICE", "0"))


def test_svd_sweep_limit_is_reported(capped_ctx):
    rng = np.random.default_rng(3)
    M = rng.standard_normal((48, 40))
    with pytest.raises(ttgpu.TTGError) as e:
        ttgpu.dense_svd(M, ctx=capped_ctx)
    assert e.value.code == NOCONV


def test_amen_svd_sweep_limit_is_an_error(capped_ctx):
    A, y, x0, z0 = aniso_config(d=5, n=16)
    with pytest.raises(ttgpu.TTGError) as e:
        ttgpu.amen_solve2(host_mat(A), host_tt(y), 1e-8, x0=host_tt(x0), z0=host_tt(z0),
                          rmax=64, nswp=4, ctx=capped_ctx)
    assert e.value.code == NOCONV


def test_round_falls_back_when_svd_does_not_converge(capped_ctx):
    """round.m:64-74: when svd fails to converge the reference takes svds;
    here the fallback SVD of the core, with the same ranks and result."""
    rng = np.random.default_rng(23)
    from oracle.tt import tt_randn
    x = tt_randn(16, 6, 40, rng, scale=lambda r1, nn, r2: 1.0 / np.sqrt(r1 * nn))
    cores = [c.copy() for c in x.cores]
    for k in range(x.d - 1):
        cores[k] = cores[k] * np.exp(-0.3 * np.arange(cores[k].shape[2]))[None, None, :]
    xt = TT(cores)
    ref, _ = tt_round(xt, 1e-4)
    st = {}
    got = back(ttgpu.round(host_tt(xt), 1e-4, ctx=capped_ctx, stats=st))
    assert st["svd_fallbacks"] >= 1
    assert list(got.r) == list(ref.r)
    assert tt_rel(got, ref) < 1e-10


def test_amen_unreachable_tolerance_returns_iterate(ctx):
    """tol 1e-14 with one short restart per local solve: the solve runs all
    its sweeps without reaching tol and returns its iterate with status OK
    (amen_solve2.m:796-812 just stops), as the oracle does.  (Four Krylov
    steps from an N(0,1) initial guess leave every local solve far from its
    tolerance, so the two residual histories agree only roughly.)"""
    A, y, x0, z0 = laplace_config(d=5, n=16)
    opts = dict(rmax=12, nswp=3, local_restart=4, local_iters=1)
    st = {}
    got = back(ttgpu.amen_solve2(host_mat(A), host_tt(y), 1e-14, x0=host_tt(x0), z0=host_tt(z0),
                                 ctx=ctx, stats=st, **opts))
    ref, info = oamen.amen_solve2(A, y, 1e-14, x0, z0, **opts)
    assert st["sweeps"] == info["sweeps"] == 3
    assert st["max_res"][-1] > 1e-14 and info["max_res"][-1] > 1e-14
    assert np.all(np.isfinite(got.flat()))
    assert max(got.r) <= 12 + 4
    rg, rr = true_residual(A, got, y), true_residual(A, ref, y)
    assert 0.5 * rr <= rg <= 2.0 * rr


def test_round_zero_tensor(ctx):
    z = TT([np.zeros((1, 4, 3)), np.zeros((3, 4, 3)), np.zeros((3, 4, 1))])
    ref, _ = tt_round(z, 1e-8)
    got = back(ttgpu.round(host_tt(z), 1e-8, ctx=ctx))
    assert list(got.r) == list(ref.r) == [1, 1, 1, 1]
    assert np.all(got.full() == 0.0)
