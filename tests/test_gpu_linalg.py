"""GPU tests of the device FP64 factorizations (one-CTA Householder QR,
one-sided Jacobi SVD, tall QR) against numpy/LAPACK, through the C ABI."""
import numpy as np
import pytest

import ttgpu

pytestmark = pytest.mark.gpu

SHAPES = [(64, 64), (132, 132), (4096, 64), (256, 4), (4, 256), (37, 53), (1, 5), (5, 1),
          (8448, 132), (160, 150), (256, 256), (1000, 201), (600, 600), (4096, 256),
          (301, 301), (2000, 384), (77, 77), (113, 113), (500, 90)]


@pytest.mark.parametrize("m,n", SHAPES)
def test_dense_svd_matches_lapack(ctx, m, n):
    rng = np.random.default_rng(m * 7 + n)
    A = rng.standard_normal((m, n))
    U, s, VT = ttgpu.dense_svd(A, ctx=ctx)
    s_ref = np.linalg.svd(A, compute_uv=False)
    k = min(m, n)
    # backward error of a one-sided Jacobi SVD grows like k * eps: 1e-13 up
    # to k = 256, 2.4e-13 at k = 600
    tol = max(1e-13, 4e-16 * k)
    # V is a product of some sweeps * k^2 / 2 plane rotations: each entry
    # takes a rounding error from each of the S k rotations that touch its
    # row, so the k^2 entries of V^T V - I grow like eps sqrt(S k) each and
    # the Frobenius norm like eps k^1.5 (3.7e-12 measured at k = 600)
    orth = max(1e-12, 4e-16 * k ** 1.5)
    assert np.allclose(s, s_ref, rtol=0, atol=tol * s_ref[0])
    assert np.linalg.norm(U * s @ VT - A) / np.linalg.norm(A) < tol
    assert np.linalg.norm(U.T @ U - np.eye(k)) < orth
    assert np.linalg.norm(VT @ VT.T - np.eye(k)) < orth
    assert np.all(np.diff(s) <= 0)


@pytest.mark.parametrize("m,n", [(300, 6), (8, 8), (6, 3), (2048, 8)])
def test_dense_svd_few_columns_rank_deficient(ctx, m, n):
    """Tall matrices with at most 8 columns take the one-CTA Jacobi SVD of A
    itself: zero and repeated columns must still give orthonormal U."""
    rng = np.random.default_rng(m + n)
    A = rng.standard_normal((m, n))
    A[:, 1] = 0.0
    A[:, n - 1] = A[:, 0]
    U, s, VT = ttgpu.dense_svd(A, ctx=ctx)
    s_ref = np.linalg.svd(A, compute_uv=False)
    assert np.allclose(s, s_ref, rtol=0, atol=1e-13 * s_ref[0])
    assert np.linalg.norm(U * s @ VT - A) / np.linalg.norm(A) < 1e-13
    assert np.linalg.norm(U.T @ U - np.eye(n)) < 1e-12
    assert np.linalg.norm(VT @ VT.T - np.eye(n)) < 1e-12
    assert s[-1] == 0.0 or s[-1] < 1e-14 * s[0]


def test_dense_svd_few_columns_graded(ctx):
    rng = np.random.default_rng(11)
    Q1, _ = np.linalg.qr(rng.standard_normal((512, 8)))
    Q2, _ = np.linalg.qr(rng.standard_normal((8, 8)))
    sv = 10.0 ** (-np.linspace(0, 14, 8))
    A = (Q1 * sv) @ Q2.T
    U, s, VT = ttgpu.dense_svd(A, ctx=ctx)
    assert np.allclose(s, sv, rtol=0, atol=4e-16 * 8)
    assert np.linalg.norm(U * s @ VT - A) / np.linalg.norm(A) < 1e-13
    assert np.linalg.norm(U.T @ U - np.eye(8)) < 1e-12


@pytest.mark.parametrize("n", [96, 180])
def test_dense_svd_graded_spectrum(ctx, n):
    """Singular values spanning 14 decades (the truncation regime of AMEn);
    n = 180 runs the grid-wide Jacobi rounds."""
    rng = np.random.default_rng(3)
    Q1, _ = np.linalg.qr(rng.standard_normal((512, n)))
    Q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
    sv = 10.0 ** (-np.linspace(0, 14, n))
    A = (Q1 * sv) @ Q2.T
    U, s, VT = ttgpu.dense_svd(A, ctx=ctx)
    # backward-stable bound |s_i - sv_i| <= p(n) eps ||A||, p(n) ~ n here
    assert np.allclose(s, sv, rtol=0, atol=4e-16 * n)
    assert np.linalg.norm(U * s @ VT - A) / np.linalg.norm(A) < 1e-13


@pytest.mark.parametrize("m,n", [(64, 64), (256, 4), (36, 9), (9, 36), (4096, 64), (130, 120)])
def test_dense_qr_matches_lapack(ctx, m, n):
    rng = np.random.default_rng(m + 11 * n)
    A = rng.standard_normal((m, n))
    Q, R = ttgpu.dense_qr(A, ctx=ctx)
    Qr, Rr = np.linalg.qr(A)
    k = min(m, n)
    assert np.linalg.norm(Q @ R - A) / np.linalg.norm(A) < 1e-13
    assert np.linalg.norm(Q.T @ Q - np.eye(k)) < 1e-12
    assert np.allclose(np.tril(R, -1), 0)
    # Same (LAPACK) sign convention as MATLAB's qr(A,0): R agrees entrywise.
    assert np.allclose(R, Rr, rtol=1e-10, atol=1e-12 * np.abs(Rr).max())


def test_dense_qr_rank_deficient(ctx):
    rng = np.random.default_rng(9)
    B = rng.standard_normal((200, 3))
    A = np.hstack([B, B[:, :1] * 2.0, B[:, 1:2] - B[:, 2:3]])
    Q, R = ttgpu.dense_qr(A, ctx=ctx)
    assert np.linalg.norm(Q @ R - A) / np.linalg.norm(A) < 1e-13
    assert np.linalg.norm(Q.T @ Q - np.eye(5)) < 1e-12


@pytest.mark.parametrize("m,n", [(8192, 4), (40000, 1), (9000, 8), (30000, 5)])
def test_skinny_qr_matches_lapack(ctx, m, n):
    """Skinny matrices too tall for one CTA's shared memory: the one-CTA
    Householder QR from global memory gives LAPACK's factors, signs included."""
    rng = np.random.default_rng(m + 3 * n)
    A = rng.standard_normal((m, n))
    Q, R = ttgpu.dense_qr(A, ctx=ctx)
    Qr, Rr = np.linalg.qr(A)
    assert np.linalg.norm(R - Rr) <= 1e-12 * np.linalg.norm(Rr)
    assert np.linalg.norm(Q.T @ Q - np.eye(n)) < 1e-12
    assert np.linalg.norm(Q @ R - A) <= 1e-13 * np.linalg.norm(A)
