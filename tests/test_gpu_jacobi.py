"""Block-Jacobi local preconditioners (solve/solve3d_2ml.m:21-70,120-146):
'cjacobi' (MEX prec 1), 'ljacobi' (2) and 'rjacobi' (3).  The preconditioned
device local solves and AMEn with each local_prec against the FP64 oracle
(1e-10)."""
import numpy as np
import pytest

import ttgpu
from oracle import amen as oamen
from oracle.builders import aniso_config, laplace_config
from oracle.tt import TT, tt_norm

pytestmark = pytest.mark.gpu


def _system(rng, rx1, n, rx2, ra1=3, ra2=2, eps=0.05):
    """Interfaces near 3 I and a Laplacian-like A core with small couplings:
    unpreconditioned GMRES stalls on the 1/n^2 end of the spectrum, the
    centre blocks carry it."""
    Phi1 = rng.standard_normal((rx1, rx1, ra1)) * eps
    Phi1[:, :, 0] += 3 * np.eye(rx1)
    A = rng.standard_normal((ra1, n, n, ra2)) * eps / n ** 2
    A[0, :, :, 0] += (n + 1) ** 2 * (2 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1)) / n ** 2
    Phi2 = rng.standard_normal((rx2, ra2, rx2)) * eps
    Phi2[:, 0, :] += 3 * np.eye(rx2)
    return Phi1, A, Phi2


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("rx1,n,rx2,tol", [(3, 5, 4, 1e-11), (12, 16, 9, 1e-9),
                                           (8, 64, 8, 1e-10), (5, 100, 3, 1e-10)])
def test_cjacobi_local_solve_parity(ctx, rx1, n, rx2, tol):
    rng = np.random.default_rng(rx1 * n)
    Phi1, A, Phi2 = _system(rng, rx1, n, rx2)
    sz = rx1 * n * rx2
    rhs = rng.standard_normal(sz)
    sol_prev = 0.01 * rng.standard_normal(sz)
    ref = oamen.solve3d_2(Phi1, A, Phi2, rhs, tol, sol_prev, 40, 2, prec=1)
    info1, info0 = {}, {}
    got = ttgpu.solve3d_2(Phi1, A, Phi2, rhs, tol, 1, sol_prev, 1, 40, 2, ctx=ctx, info=info1)
    assert rel(got, ref) < 1e-10
    ttgpu.solve3d_2(Phi1, A, Phi2, rhs, tol, 1, sol_prev, 0, 40, 2, ctx=ctx, info=info0)
    assert info1["iters"] < info0["iters"]
    res = np.linalg.norm(oamen.bfun3(Phi1, A, Phi2, got) - rhs) / np.linalg.norm(rhs)
    assert res <= 10 * tol


def test_cjacobi_amen_parity(ctx):
    A, y, x0, z0 = laplace_config(d=4, n=8)
    ref, info = oamen.amen_solve2(A, y, 1e-12, x0, z0, rmax=64, nswp=10, local_prec="cjacobi")
    st = {}
    got = ttgpu.amen_solve2(ttgpu.TTMatrix(A.n, A.m, A.r, A.flat()),
                            ttgpu.TensorTrain(y.n, y.r, y.flat()), 1e-12,
                            x0=ttgpu.TensorTrain(x0.n, x0.r, x0.flat()),
                            z0=ttgpu.TensorTrain(z0.n, z0.r, z0.flat()), ctx=ctx, stats=st,
                            rmax=64, nswp=10, local_prec="cjacobi")
    got = TT.from_flat(got.n, got.r, got.core)
    assert st["sweeps"] == info["sweeps"]
    assert list(got.r) == list(ref.r)
    assert tt_norm(got - ref) < 1e-10 * tt_norm(ref)


def test_cjacobi_reduces_iterations_on_aniso(ctx):
    """On the anisotropic rank-3 operator the preconditioned local solves need
    fewer Krylov iterations for the same tolerance."""
    A, y, x0, z0 = aniso_config(d=4, n=32)
    args = (ttgpu.TTMatrix(A.n, A.m, A.r, A.flat()), ttgpu.TensorTrain(y.n, y.r, y.flat()), 1e-8)
    kw = dict(x0=ttgpu.TensorTrain(x0.n, x0.r, x0.flat()), z0=ttgpu.TensorTrain(z0.n, z0.r,
              z0.flat()), ctx=ctx, rmax=32, nswp=4)
    s0, s1 = {}, {}
    ttgpu.amen_solve2(*args, stats=s0, **kw)
    ttgpu.amen_solve2(*args, stats=s1, local_prec="cjacobi", **kw)
    assert s1["gmres_iters"] < s0["gmres_iters"]


@pytest.mark.parametrize("prec", [2, 3])
@pytest.mark.parametrize("rx1,n,rx2,tol", [(3, 5, 4, 1e-11), (6, 16, 5, 1e-9), (9, 20, 7, 1e-10)])
def test_lr_jacobi_local_solve_parity(ctx, prec, rx1, n, rx2, tol):
    """Left / right block-Jacobi: blocks of rx1 n (ljacobi) or n rx2
    (rjacobi) rows; the last case has blocks above 128 rows (LU path)."""
    rng = np.random.default_rng(rx1 * n + prec)
    Phi1, A, Phi2 = _system(rng, rx1, n, rx2)
    sz = rx1 * n * rx2
    rhs = rng.standard_normal(sz)
    sol_prev = 0.01 * rng.standard_normal(sz)
    ref = oamen.solve3d_2(Phi1, A, Phi2, rhs, tol, sol_prev, 40, 2, prec=prec)
    info = {}
    got = ttgpu.solve3d_2(Phi1, A, Phi2, rhs, tol, 1, sol_prev, prec, 40, 2, ctx=ctx, info=info)
    assert rel(got, ref) < 1e-10
    res = np.linalg.norm(oamen.bfun3(Phi1, A, Phi2, got) - rhs) / np.linalg.norm(rhs)
    assert res <= 10 * tol


@pytest.mark.parametrize("name", ["ljacobi", "rjacobi"])
def test_lr_jacobi_amen_parity(ctx, name):
    A, y, x0, z0 = laplace_config(d=4, n=8)
    ref, info = oamen.amen_solve2(A, y, 1e-12, x0, z0, rmax=64, nswp=10, local_prec=name)
    st = {}
    got = ttgpu.amen_solve2(ttgpu.TTMatrix(A.n, A.m, A.r, A.flat()),
                            ttgpu.TensorTrain(y.n, y.r, y.flat()), 1e-12,
                            x0=ttgpu.TensorTrain(x0.n, x0.r, x0.flat()),
                            z0=ttgpu.TensorTrain(z0.n, z0.r, z0.flat()), ctx=ctx, stats=st,
                            rmax=64, nswp=10, local_prec=name)
    got = TT.from_flat(got.n, got.r, got.core)
    assert st["sweeps"] == info["sweeps"]
    assert list(got.r) == list(ref.r)
    assert tt_norm(got - ref) < 1e-10 * tt_norm(ref)


def test_preconditioner_errors(ctx):
    rng = np.random.default_rng(1)
    Phi1, A, Phi2 = _system(rng, 3, 4, 3)
    rhs = rng.standard_normal(36)
    with pytest.raises(ttgpu.TTGError, match="unknown"):
        ttgpu.solve3d_2(Phi1, A, Phi2, rhs, 1e-8, 1, np.zeros(36), 4, ctx=ctx)
    with pytest.raises(ttgpu.TTGError, match="cjacobi"):
        ttgpu.solve3d_2(Phi1, A, Phi2, rhs, 1e-8, 1, np.zeros(36), 2, ctx=ctx, precision="mixed")
    A0 = A.copy()
    A0[:] = 0.0  # every Jacobi block singular: the factorization error surfaces
    with pytest.raises(ttgpu.TTGError):
        ttgpu.solve3d_2(Phi1, A0, Phi2, rhs, 1e-8, 1, np.zeros(36), 1, ctx=ctx)
    # the failure does not leak into the next call on the context
    M = rng.standard_normal((8, 8))
    U, s, VT = ttgpu.dense_svd(M, ctx=ctx)
    assert np.allclose(U * s @ VT, M)


@pytest.mark.parametrize("rx1,n,rx2", [(6, 32, 5), (12, 64, 10)])
def test_cjacobi_mixed_local_solve(ctx, rx1, n, rx2):
    """'cjacobi' in the mixed-precision local solve (BF16 matvecs of B P in
    the FP32 Krylov solves, FP64 refinement): the FP64 residual target is
    met, with fewer Krylov steps than without the preconditioner."""
    rng = np.random.default_rng(rx1 * n + 11)
    Phi1, A, Phi2 = _system(rng, rx1, n, rx2)
    sz = rx1 * n * rx2
    rhs = rng.standard_normal(sz)
    sol_prev = np.zeros(sz)
    tol = 1e-9
    i1, i0 = {}, {}
    got = ttgpu.solve3d_2(Phi1, A, Phi2, rhs, tol, 1, sol_prev, 1, 40, 2, ctx=ctx,
                          precision="mixed", info=i1)
    ttgpu.solve3d_2(Phi1, A, Phi2, rhs, tol, 1, sol_prev, 0, 40, 2, ctx=ctx, precision="mixed",
                    info=i0)
    res = np.linalg.norm(oamen.bfun3(Phi1, A, Phi2, got) - rhs) / np.linalg.norm(rhs)
    assert res <= tol * 1.0001
    assert i1["iters"] < i0["iters"]


def test_cjacobi_mixed_amen(ctx):
    """AMEn in mixed precision with local_prec 'cjacobi' meets its stopping
    test with a true residual within the tolerance, like the FP64 solve."""
    from oracle.tt import true_residual
    A, y, x0, z0 = aniso_config(d=5, n=16)
    kw = dict(x0=ttgpu.TensorTrain(x0.n, x0.r, x0.flat()),
              z0=ttgpu.TensorTrain(z0.n, z0.r, z0.flat()), ctx=ctx, rmax=64, nswp=20)
    st = {}
    got = ttgpu.amen_solve2(ttgpu.TTMatrix(A.n, A.m, A.r, A.flat()),
                            ttgpu.TensorTrain(y.n, y.r, y.flat()), 1e-8, stats=st,
                            local_prec="cjacobi", precision="mixed", **kw)
    assert st["max_res"][st["sweeps"] - 1] < 1e-8
    assert true_residual(A, TT.from_flat(got.n, got.r, got.core), y) <= 1e-8

