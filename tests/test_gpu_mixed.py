"""GPU tests of the mixed-precision path (BF16 tcgen05 matvec, FP32 Krylov,
FP64 refinement), through the C ABI.

Tolerances: the BF16 local matvec agrees with the FP64 oracle to 2e-2
relative (BF16 operands and intermediates, FP32 accumulation); the mixed
local solve and the mixed AMEn solve reach the same FP64 residual targets as
the FP64 path (the refinement residual is computed in FP64).
"""
import numpy as np
import pytest

import ttgpu
from oracle import amen as oamen
from oracle.builders import aniso_config, laplace_config
from oracle.tt import TT, true_residual

pytestmark = pytest.mark.gpu

BF16_MV_TOL = 2e-2


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


@pytest.mark.parametrize("rx1,n,rx2,ra1,ra2", [(1, 64, 2, 1, 3), (5, 16, 7, 2, 3), (33, 17, 65, 3, 2),
                                               (61, 64, 59, 3, 3), (128, 64, 128, 3, 3),
                                               (132, 32, 100, 2, 2)])
def test_bf16_matvec_vs_oracle(ctx, rx1, n, rx2, ra1, ra2):
    rng = np.random.default_rng(rx1 + 3 * rx2 + n)
    Phi1 = rng.standard_normal((rx1, rx1, ra1))
    A = rng.standard_normal((ra1, n, n, ra2))
    Phi2 = rng.standard_normal((rx2, ra2, rx2))
    x = rng.standard_normal(rx1 * n * rx2)
    ref = oamen.bfun3(Phi1, A, Phi2, x)
    got = ttgpu.bfun3(Phi1, A, Phi2, x, ctx=ctx, precision="mixed")
    assert rel(got, ref) < BF16_MV_TOL


def test_bf16_matvec_repeatable(ctx):
    rng = np.random.default_rng(5)
    Phi1 = rng.standard_normal((40, 40, 3))
    A = rng.standard_normal((3, 32, 32, 3))
    Phi2 = rng.standard_normal((36, 3, 36))
    x = rng.standard_normal(40 * 32 * 36)
    a = ttgpu.bfun3(Phi1, A, Phi2, x, ctx=ctx, precision="mixed")
    b = ttgpu.bfun3(Phi1, A, Phi2, x, ctx=ctx, precision="mixed")
    assert np.array_equal(a, b)


def _local_system(rng, rx1, n, rx2):
    from oracle.builders import kron_sum_operator, lap1d
    A = kron_sum_operator([lap1d(n) / (n + 1) ** 2] * 3).cores[1]
    Phi1 = rng.standard_normal((rx1, rx1, 2)) * 0.1
    Phi1 = Phi1 + np.transpose(Phi1, (1, 0, 2))
    Phi1[:, :, 1] += 10 * np.eye(rx1)
    Phi2 = rng.standard_normal((rx2, 2, rx2)) * 0.1
    Phi2 = Phi2 + np.transpose(Phi2, (2, 1, 0))
    Phi2[:, 0, :] += 10 * np.eye(rx2)
    return Phi1, A, Phi2


@pytest.mark.parametrize("rx1,n,rx2", [(8, 16, 9), (30, 32, 30)])
def test_mixed_local_solve_reaches_fp64_target(ctx, rx1, n, rx2):
    rng = np.random.default_rng(rx1)
    Phi1, A, Phi2 = _local_system(rng, rx1, n, rx2)
    sz = rx1 * n * rx2
    rhs = rng.standard_normal(sz)
    sol_prev = np.zeros(sz)
    tol = 1e-9
    got = ttgpu.solve3d_2(Phi1, A, Phi2, rhs, tol, 1, sol_prev, 0, 40, 2, 0, ctx=ctx,
                          precision="mixed")
    res = np.linalg.norm(oamen.bfun3(Phi1, A, Phi2, got) - rhs) / np.linalg.norm(rhs)
    ref = oamen.solve3d_2(Phi1, A, Phi2, rhs, tol, sol_prev, 40, 2)
    res_ref = np.linalg.norm(oamen.bfun3(Phi1, A, Phi2, ref) - rhs) / np.linalg.norm(rhs)
    assert res <= max(tol, 2 * res_ref)


def _solve(ctx, A, y, x0, z0, tol, prec, **opts):
    st = {}
    got = ttgpu.amen_solve2(ttgpu.TTMatrix(A.n, A.m, A.r, A.flat()),
                            ttgpu.TensorTrain(y.n, y.r, y.flat()), tol,
                            x0=ttgpu.TensorTrain(x0.n, x0.r, x0.flat()),
                            z0=ttgpu.TensorTrain(z0.n, z0.r, z0.flat()),
                            ctx=ctx, stats=st, precision=prec, **opts)
    return TT.from_flat(got.n, got.r, got.core), st


def test_mixed_amen_laplace(ctx):
    A, y, x0, z0 = laplace_config(d=6, n=32)
    x, st = _solve(ctx, A, y, x0, z0, 1e-8, "mixed", rmax=30)
    assert st["max_res"][-1] < 1e-8
    # the stated residual of the mixed form (the FP64 oracle: 2.8e-9)
    res = true_residual(A, x, y)
    print("mixed laplace d=6 n=32 true residual %.3e" % res)
    assert res <= 1e-8


def test_mixed_amen_aniso_matches_fp64_residual(ctx):
    A, y, x0, z0 = aniso_config(d=6, n=32)
    xm, stm = _solve(ctx, A, y, x0, z0, 1e-8, "mixed", rmax=64)
    xd, std = _solve(ctx, A, y, x0, z0, 1e-8, "fp64", rmax=64)
    rm, rd = true_residual(A, xm, y), true_residual(A, xd, y)
    print("aniso d=6 n=32 true residual mixed %.3e fp64 %.3e" % (rm, rd))
    assert stm["max_res"][-1] < 1e-8
    # the stated residual of the mixed form (the FP64 oracle: 9.0e-9)
    assert rm <= 1e-8
