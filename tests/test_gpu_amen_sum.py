"""GPU parity of amen_sum (core/amen_sum.m default path for TT inputs)
against the oracle restatement, through the C ABI, on identical y0 / z0.

Ranks come from my_chop2 on singular values of the projected sums: they
must be identical wherever the decision is not a near tie; the results must
agree to 1e-10 (TT-relative) and match the exact combination at tight
tolerance."""
import numpy as np
import pytest

import ttgpu
from oracle.amen_sum import amen_sum as ref_amen_sum
from oracle.tt import TT, tt_norm, tt_rand, tt_randn

pytestmark = pytest.mark.gpu


def host_tt(t):
    return ttgpu.TensorTrain(t.n, t.r, t.flat())


def back(t):
    return TT.from_flat(t.n, t.r, t.core)


def _full_with_outputs(y):
    M = int(y.r[-1])
    return TT(y.cores + [np.eye(M).reshape(M, M, 1)]).full()


def _pair(ctx, X, c, tol, y0, z0, **kw):
    ref, zref, info = ref_amen_sum(X, c, tol, y0, z0, **kw)
    y, z, sweeps = ttgpu.amen_sum([host_tt(x) for x in X], c, tol, y0=host_tt(y0),
                                  z0=host_tt(z0) if z0 is not None else None, ctx=ctx, **kw)
    return ref, back(y), info, sweeps


def test_amen_sum_exact_two_outputs(ctx):
    rng = np.random.default_rng(0)
    d, n = 5, 5
    X = [tt_randn(n, d, r, rng) for r in (2, 3, 2)]
    c = rng.standard_normal((3, 2))
    ref, got, info, sweeps = _pair(ctx, X, c, 1e-10, tt_randn(n, d, 2, rng), tt_rand(n, d, 4, rng))
    assert list(got.r) == list(ref.r)
    assert sweeps == info["sweeps"]
    G, R = _full_with_outputs(got), _full_with_outputs(ref)
    assert np.linalg.norm(G - R) <= 1e-10 * np.linalg.norm(R)
    F = sum(np.multiply.outer(Xj.full(), c[j]) for j, Xj in enumerate(X))
    assert np.linalg.norm(G - F) <= 1e-10 * np.linalg.norm(F)


@pytest.mark.parametrize("kickrank", [4, 0])
def test_amen_sum_loose_tolerance(ctx, kickrank):
    """Summands of overall scales 1, 1e-2, 1e-4, 1e-6 at tol 1e-3 and 1e-6:
    some of them fall below the truncation threshold."""
    rng = np.random.default_rng(2)
    d, n = 6, 6
    X = [tt_randn(n, d, 3, rng, scale=s ** (1.0 / d)) for s in (1.0, 1e-2, 1e-4, 1e-6)]
    c = np.ones((4, 1))
    for tol in (1e-3, 1e-6):
        y0, z0 = tt_randn(n, d, 2, rng), tt_rand(n, d, 4, rng)
        ref, got, info, sweeps = _pair(ctx, X, c, tol, y0, z0, kickrank=kickrank)
        assert list(got.r) == list(ref.r)
        assert sweeps == info["sweeps"]
        assert tt_norm(got - ref) <= 1e-10 * tt_norm(ref)


def test_amen_sum_larger_ranks_and_rmax(ctx):
    """d=8, n=16: three rank-12 summands (rank 36 in exact arithmetic), first
    without a cap, then capped at rmax 20."""
    rng = np.random.default_rng(5)
    d, n = 8, 16
    X = [tt_randn(n, d, 12, rng, scale=lambda r1, nn, r2: 1.0 / np.sqrt(r1 * nn))
         for _ in range(3)]
    c = np.array([1.0, -2.0, 0.5])
    y0, z0 = tt_randn(n, d, 2, rng), tt_rand(n, d, 4, rng)
    ref, got, info, sweeps = _pair(ctx, X, c, 1e-8, y0, z0)
    assert list(got.r) == list(ref.r)
    assert tt_norm(got - ref) <= 1e-10 * tt_norm(ref)
    ref2, got2, _, _ = _pair(ctx, X, c, 1e-8, y0, z0, rmax=20, nswp=4)
    assert max(got2.r) <= 20 + 4   # the backward kick adds up to kickrank
    assert list(got2.r) == list(ref2.r)
    assert tt_norm(got2 - ref2) <= 1e-10 * tt_norm(ref2)


def test_amen_sum_errors(ctx):
    rng = np.random.default_rng(3)
    X = [tt_randn(4, 4, 2, rng), tt_randn(5, 4, 2, rng)]
    with pytest.raises(ttgpu.TTGError, match="mode size"):
        ttgpu.amen_sum([host_tt(x) for x in X], [1.0, 1.0], 1e-8, ctx=ctx)
    with pytest.raises(ValueError):
        ttgpu.amen_sum([host_tt(X[0])], [1.0, 2.0], 1e-8, ctx=ctx)
