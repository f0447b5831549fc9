"""Grouped batch (``ttg_amen_solve_grouped``): the systems of a batch advance
together, their recorded launches merged kernel by kernel into grouped
launches.  Each system must get exactly what it gets when solved alone
(bit for bit, when the solves size their grids as a solve alone does), the
merged run must issue far fewer launches than the solves recorded, and a
failing system must fail alone.
"""
import numpy as np
import pytest

import ttgpu
from ttgpu import workloads
from oracle.builders import kron_sum_operator, lap1d
from oracle.tt import TT, TTMatrix, true_residual

pytestmark = pytest.mark.gpu


def _upload(ctx, As, ys):
    return ([ttgpu.DeviceTT.upload(ctx, a) for a in As],
            [ttgpu.DeviceTT.upload(ctx, y) for y in ys])


def _host(t):
    return t.download() if isinstance(t, ttgpu.DeviceTT) else t


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_grouped_matches_sequential_bitwise(ctx, precision):
    """With every solve sizing its grids from the whole device, the grouped
    batch runs each system's kernels with the launch configurations and the
    order of a solve run alone: cores, ranks and sweep counts are identical."""
    As, ys, rmaxs, _ = workloads.batch_systems(count=12, seed=7)
    dAs, dys = _upload(ctx, As, ys)
    ctx.set_option(ttgpu.Context.OPT_GROUP_SMS, 4096)
    try:
        stats, gs = [], {}
        xs = ttgpu.amen_solve2_batch(dAs, dys, 1e-8, ctx=ctx, stats=stats, grouped=True,
                                     group_stats=gs, precision=precision,
                                     per_system=[dict(rmax=r) for r in rmaxs])
    finally:
        ctx.set_option(ttgpu.Context.OPT_GROUP_SMS, 0)
    assert gs["flushes"] > 0 and gs["grouped_records"] > 0
    for i in range(len(As)):
        st1 = {}
        x1 = ttgpu.amen_solve2(dAs[i], dys[i], 1e-8, ctx=ctx, stats=st1, rmax=rmaxs[i],
                               precision=precision)
        a, b = _host(xs[i]), _host(x1)
        assert stats[i]["status"] == 0
        assert stats[i]["sweeps"] == st1["sweeps"]
        assert list(a.r) == list(b.r)
        assert np.array_equal(a.core, b.core), "system %d differs" % i
        for t in (xs[i], x1):
            if isinstance(t, ttgpu.DeviceTT):
                t.free()
    for h in dAs + dys:
        h.free()


def test_grouped_uneven_systems_sample(ctx):
    """A seeded sample of the batched workload with the default SM shares:
    every system meets the stopping criterion or stops at its rank cap or
    sweep limit, converged solutions have small true residuals, and the
    grouped launches replace most of the recorded ones."""
    As, ys, rmaxs, _ = workloads.batch_systems(count=24, seed=5)
    stats, gs = [], {}
    xs = ttgpu.amen_solve2_batch(As, ys, 1e-8, ctx=ctx, stats=stats, grouped=True,
                                 group_stats=gs, precision="mixed",
                                 per_system=[dict(rmax=r) for r in rmaxs])
    for i, (A, y, x) in enumerate(zip(As, ys, xs)):
        st = stats[i]
        assert st["status"] == 0
        converged = st["max_res"][st["sweeps"] - 1] < 1e-8
        assert converged or st["sweeps"] == 20 or st["max_rank"] >= rmaxs[i]
        if converged:
            Ao = TTMatrix.from_flat(A.n, A.m, A.r, A.core)
            yo = TT.from_flat(y.n, y.r, y.core)
            xo = TT.from_flat(x.n, x.r, x.core)
            assert true_residual(Ao, xo, yo) <= 1e-8  # the FP64 oracle: at most 6.4e-9
    assert gs["launches"] < gs["records"], gs
    assert gs["grouped_records"] > gs["records"] / 3, gs
    # The executor's count of BF16 GEMM work (recorded GEMMs less the skipped
    # Krylov steps) is the solves' own count of BF16 matvec FLOPs.
    lp = sum(q["gflop_lp"] for q in stats)
    assert lp > 0
    assert abs(gs["tc_gflop"] - lp) <= 1e-9 * lp, (gs["tc_gflop"], lp)
    assert gs["tc_records"] == 3 * sum(q["matvecs_lp"] for q in stats), gs
    assert gs["tc_launches"] > 0
    assert gs["tc_ms"] == 0.0  # untimed unless TTG_GROUP_TIME=1


def test_grouped_gemm_timing(ctx, monkeypatch):
    """TTG_GROUP_TIME=1 brackets every BF16 GEMM launch with CUDA events:
    the summed launch time is positive and the results are unchanged."""
    As, ys, rmaxs, _ = workloads.batch_systems(count=8, seed=9)
    per = [dict(rmax=r) for r in rmaxs]
    ref = ttgpu.amen_solve2_batch(As, ys, 1e-8, ctx=ctx, grouped=True, precision="mixed",
                                  per_system=per)
    monkeypatch.setenv("TTG_GROUP_TIME", "1")
    gs = {}
    got = ttgpu.amen_solve2_batch(As, ys, 1e-8, ctx=ctx, grouped=True, group_stats=gs,
                                  precision="mixed", per_system=per)
    assert gs["tc_ms"] > 0 and gs["tc_launches"] > 0 and gs["tc_gflop"] > 0, gs
    for a, b in zip(ref, got):
        assert list(a.r) == list(b.r) and np.array_equal(a.core, b.core)


def test_grouped_reports_failing_systems(ctx):
    """A rectangular operator and a right-hand side holding a NaN fail alone
    with their own status; the other systems are solved as usual."""
    def lap(d, n):
        return (kron_sum_operator([lap1d(n)] * d), TT([np.ones((1, n, 1)) for _ in range(d)]))
    A0, y0 = lap(4, 8)
    A2, y2 = lap(3, 8)
    rng = np.random.default_rng(0)
    rect = TTMatrix([rng.standard_normal((1, 8, 6, 1)) for _ in range(4)])
    ybad = TT([np.ones((1, 8, 1)) for _ in range(4)])
    ybad.cores[2][0, 3, 0] = np.nan
    mat = lambda A: ttgpu.TTMatrix(A.n, A.m, A.r, A.flat())
    ten = lambda t: ttgpu.TensorTrain(t.n, t.r, t.flat())
    As = [mat(A0), mat(rect), mat(A2), mat(A0)]
    ys = [ten(y0), ten(TT([np.ones((1, 8, 1)) for _ in range(4)])), ten(y2), ten(ybad)]
    stats = []
    with pytest.raises(ttgpu.TTGError, match="system 1"):
        ttgpu.amen_solve2_batch(As, ys, 1e-8, ctx=ctx, stats=stats, grouped=True, nswp=6)
    assert stats[0]["status"] == 0 and stats[2]["status"] == 0
    assert stats[1]["status"] != 0 and stats[3]["status"] != 0
    assert stats[0]["max_res"][stats[0]["sweeps"] - 1] < 1e-8
