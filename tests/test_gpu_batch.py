"""Batched AMEn (``ttg_amen_solve_batch``): systems of uneven d, n and rmax
solved concurrently on several streams must give what the single-system
entry gives, and what the FP64 oracle gives at tight tolerance (1e-10
relative, identical sweeps and ranks).
"""
import numpy as np
import pytest

import ttgpu
from oracle import amen as oamen
from oracle.builders import kron_sum_operator, lap1d
from oracle.tt import TT, TTMatrix, tt_norm, tt_rand, tt_randn, true_residual

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-10


def system(d, n, seed):
    A = kron_sum_operator([lap1d(n)] * d)
    y = TT([np.ones((1, n, 1)) for _ in range(d)])
    rng = np.random.default_rng(seed)
    x0 = tt_randn(n, d, 2, rng)
    z0 = tt_rand(n, d, 4, rng)
    return A, y, x0, z0


def host_tt(t):
    return ttgpu.TensorTrain(t.n, t.r, t.flat())


def host_mat(A):
    return ttgpu.TTMatrix(A.n, A.m, A.r, A.flat())


def back(t):
    return TT.from_flat(t.n, t.r, t.core)


SHAPES = [(4, 8, 24), (3, 16, 32), (5, 8, 16), (6, 4, 12), (4, 32, 8), (3, 12, 20), (7, 8, 10)]


def test_batch_matches_single_and_oracle(ctx):
    systems = [system(d, n, 10 + i) for i, (d, n, _) in enumerate(SHAPES)]
    tol = 1e-12
    As = [host_mat(s[0]) for s in systems]
    ys = [host_tt(s[1]) for s in systems]
    x0s = [host_tt(s[2]) for s in systems]
    z0s = [host_tt(s[3]) for s in systems]
    per = [dict(rmax=r) for (_, _, r) in SHAPES]
    stats = []
    xs = ttgpu.amen_solve2_batch(As, ys, tol, x0s=x0s, z0s=z0s, workers=4, ctx=ctx,
                                 stats=stats, per_system=per, nswp=8, kickrank=4)
    for i, ((A, y, x0, z0), (d, n, r)) in enumerate(zip(systems, SHAPES)):
        st1 = {}
        x1 = ttgpu.amen_solve2(As[i], ys[i], tol, x0=x0s[i], z0=z0s[i], ctx=ctx, stats=st1,
                               rmax=r, nswp=8, kickrank=4)
        assert stats[i]["status"] == 0
        if st1["max_res"][-1] < 1e-10:
            # converged to the exact low-rank solution: no rank decision is
            # near a tie, so batch, single and oracle agree to 1e-10
            assert stats[i]["sweeps"] == st1["sweeps"]
            assert list(xs[i].r) == list(x1.r)
            assert tt_norm(back(xs[i]) - back(x1)) <= SOLVE_TOL * tt_norm(back(x1))
            ref, info = oamen.amen_solve2(A, y, tol, x0, z0, rmax=r, nswp=8, kickrank=4)
            assert tt_norm(back(xs[i]) - ref) <= SOLVE_TOL * tt_norm(ref)
        else:
            # stopped by the rank cap / sweep limit: the batch streams use other
            # reduction orders, so compare the reached residuals
            rb = true_residual(A, back(xs[i]), y)
            r1 = true_residual(A, back(x1), y)
            assert rb <= 2 * r1 + 1e-12 and r1 <= 2 * rb + 1e-12


def test_batch_reports_failing_system(ctx):
    """A system that cannot be solved (rectangular operator) fails alone; the
    others are solved and the call raises with the failing index."""
    good = [system(4, 8, 1), system(3, 8, 2)]
    As = [host_mat(good[0][0]), None, host_mat(good[1][0])]
    ys = [host_tt(good[0][1]), None, host_tt(good[1][1])]
    rng = np.random.default_rng(0)
    rect = TTMatrix([rng.standard_normal((1, 8, 6, 1)) for _ in range(4)])
    As[1] = host_mat(rect)
    ys[1] = host_tt(TT([np.ones((1, 8, 1)) for _ in range(4)]))
    stats = []
    with pytest.raises(ttgpu.TTGError, match="system 1"):
        ttgpu.amen_solve2_batch(As, ys, 1e-8, workers=3, ctx=ctx, stats=stats, nswp=4)
    assert [s["status"] for s in stats][0] == 0 and stats[1]["status"] != 0
    assert stats[2]["status"] == 0


def test_batch_uneven_systems_sample(ctx):
    """A seeded sample of the batched workload (uneven d, n, rmax; tol 1e-8):
    every system either meets the stopping criterion or ran all sweeps at its
    rank cap, and the converged solutions have small true residuals."""
    from ttgpu import workloads
    As, ys, rmaxs, info = workloads.batch_systems(count=24, seed=5)
    stats = []
    xs = ttgpu.amen_solve2_batch(As, ys, 1e-8, workers=8, ctx=ctx, stats=stats,
                                 per_system=[dict(rmax=r) for r in rmaxs])
    for i, (A, y, x) in enumerate(zip(As, ys, xs)):
        st = stats[i]
        assert st["status"] == 0
        converged = st["max_res"][st["sweeps"] - 1] < 1e-8
        assert converged or st["sweeps"] == 20 or st["max_rank"] >= rmaxs[i]
        if converged:
            Ao = TTMatrix.from_flat(A.n, A.m, A.r, A.core)
            yo = TT.from_flat(y.n, y.r, y.core)
            # the FP64 oracle on the same systems: at most 6.4e-9
            assert true_residual(Ao, back(x), yo) <= 1e-8
