"""Device TT algebra (ttg_tt_matvec / axpby / norm / dot) against the oracle's
restatements of @tt_matrix/mtimes.m, @tt_tensor/plus.m, @tt_tensor/norm.m and
@tt_tensor/dot.m: matvec and axpby cores bit-comparable (1e-13 relative,
identical ranks), norms and inner products to 1e-12, the device true
residual against the oracle's."""
import numpy as np
import pytest

import ttgpu
from golden_io import load_fixture
from oracle.builders import aniso_config
from oracle.tt import TT, TTMatrix, tt_dot, tt_matvec, tt_norm, tt_plus, tt_randn, true_residual

pytestmark = pytest.mark.gpu


def host_tt(t):
    return ttgpu.TensorTrain(t.n, t.r, t.flat())


def host_mat(A):
    return ttgpu.TTMatrix(A.n, A.m, A.r, A.flat())


def test_matvec_and_axpby_match_oracle(ctx):
    A, y, x0, _ = aniso_config(d=5, n=8)
    rng = np.random.default_rng(1)
    x = tt_randn(8, 5, 6, rng)
    got = ttgpu.tt_matvec(host_mat(A), host_tt(x), ctx=ctx)
    ref = tt_matvec(A, x)
    assert list(got.r) == list(ref.r)
    np.testing.assert_allclose(got.core, ref.flat(), rtol=1e-13, atol=1e-13 * abs(ref.flat()).max())
    s = ttgpu.tt_axpby(2.0, host_tt(x), -0.5, host_tt(y), ctx=ctx)
    sref = tt_plus(x * 2.0, y * -0.5)
    assert list(s.r) == list(sref.r)
    g = TT.from_flat(s.n, s.r, s.core)
    assert tt_norm(g - sref) <= 1e-13 * tt_norm(sref)


@pytest.mark.parametrize("d,n,r", [(1, 7, 1), (4, 5, 3), (12, 16, 40)])
def test_norm_and_dot(ctx, d, n, r):
    rng = np.random.default_rng(d * n)
    x = tt_randn(n, d, r, rng, scale=lambda r1, nn, r2: 1.0 / np.sqrt(r1 * nn))
    z = tt_randn(n, d, max(1, r // 2), rng, scale=lambda r1, nn, r2: 1.0 / np.sqrt(r1 * nn))
    assert ttgpu.tt_norm(host_tt(x), ctx=ctx) == pytest.approx(tt_norm(x), rel=1e-12)
    scale = tt_norm(x) * tt_norm(z)
    assert abs(ttgpu.tt_dot(host_tt(x), host_tt(z), ctx=ctx) - tt_dot(x, z)) <= 1e-12 * scale


@pytest.mark.parametrize("key", ["ex2", "ex6"])
def test_device_true_residual_on_reference_fixtures(ctx, key):
    """The stored solutions of the reference's tt-solve fixtures: the device
    true residual reproduces the published residuals."""
    A, rhs, x, stored = load_fixture(key)
    got = ttgpu.true_residual(host_mat(A), host_tt(x), host_tt(rhs), ctx=ctx)
    assert got == pytest.approx(true_residual(A, x, rhs), rel=1e-8)
    assert got == pytest.approx(stored, rel=1e-8)
