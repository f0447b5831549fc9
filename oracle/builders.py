"""Seeded input generators for the five workloads of the hot path.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  The same generator
feeds the CPU oracle and the GPU library (``ttgpu.workloads`` holds a
byte-identical copy of the operator formulas for the product side), so both
see identical inputs.

Operators follow the reference's operator builders in spirit
(``exp/tt_qlaplace_dd.m``, ``misc/tt_laplacerep.m:6-125``): the Kronecker sum
``sum_k I x .. x L_k x .. x I`` with ``L = (n+1)^2 tridiag(-1, 2, -1)`` written
directly as rank-2 TT-matrix cores (first ``[L I]``, middle ``[[I 0];[L I]]``,
last ``[I; L]``).
"""
import numpy as np

from .tt import TT, TTMatrix, tt_ones, tt_randn, tt_rand, tt_plus


def lap1d(n):
    """``(n+1)^2 * tridiag(-1, 2, -1)``."""
    L = 2.0 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1)
    return (n + 1) ** 2 * L


def mass1d(n):
    """``tridiag(1, 4, 1) / 6`` (1D linear-element mass matrix, SPD)."""
    return (4.0 * np.eye(n) + np.eye(n, k=1) + np.eye(n, k=-1)) / 6.0


def kron_sum_operator(mats, react=None):
    """TT matrix of ``sum_k I x .. x mats[k] x .. x I`` (+ ``react[0] x react[1] x ...``).

    Without ``react`` the TT ranks are ``[1, 2, ..., 2, 1]``; with it they are
    ``[1, 3, ..., 3, 1]`` (block-diagonal extension by the separable term).
    """
    d = len(mats)
    R = 2 if react is None else 3
    cores = []
    for k in range(d):
        L = mats[k]
        n = L.shape[0]
        I = np.eye(n)
        if d == 1:
            c = np.zeros((1, n, n, 1))
            c[0, :, :, 0] = L + (react[k] if react is not None else 0)
        elif k == 0:
            c = np.zeros((1, n, n, R))
            c[0, :, :, 0] = L
            c[0, :, :, 1] = I
            if react is not None:
                c[0, :, :, 2] = react[k]
        elif k == d - 1:
            c = np.zeros((R, n, n, 1))
            c[0, :, :, 0] = I
            c[1, :, :, 0] = L
            if react is not None:
                c[2, :, :, 0] = react[k]
        else:
            c = np.zeros((R, n, n, R))
            c[0, :, :, 0] = I
            c[1, :, :, 0] = L
            c[1, :, :, 1] = I
            if react is not None:
                c[2, :, :, 2] = react[k]
        cores.append(np.asfortranarray(c))
    return TTMatrix(cores)


def laplace_config(d=8, n=32, x_rank=2, seed=1):
    """``d``-dim Laplacian (rank 2), RHS ``tt_ones``, x0 seeded N(0,1) rank-``x_rank``."""
    rng = np.random.default_rng(seed)
    A = kron_sum_operator([lap1d(n)] * d)
    y = tt_ones(n, d)
    x0 = tt_randn(n, d, x_rank, rng)
    z0 = tt_rand(n, d, 4, rng, -1)
    return A, y, x0, z0


def aniso_config(d=10, n=64, rhs_rank=4, seed=3, react_scale=1.0):
    """Anisotropic diffusion + separable reaction, operator rank 3.

    ``A = sum_k c_k (n+1)^2 tridiag(-1,2,-1)_k + sigma * (M x .. x M)`` with
    ``c_k ~ U[0.5, 2]`` seeded, ``M = tridiag(1,4,1)/6`` and
    ``sigma = react_scale * (n+1)^2``.  The Kronecker sum alone is rank 2; the
    separable reaction term is the genuine third TT rank.  RHS: seeded rank-4
    Gaussian TT; x0 seeded N(0,1) rank 2; z0 seeded right-orthogonal rank 4.
    """
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.5, 2.0, size=d)
    sigma = react_scale * (n + 1) ** 2
    M = mass1d(n)
    react = [M * (sigma if k == 0 else 1.0) for k in range(d)]
    A = kron_sum_operator([c[k] * lap1d(n) for k in range(d)], react)
    y = tt_randn(n, d, rhs_rank, rng)
    x0 = tt_randn(n, d, 2, rng)
    z0 = tt_rand(n, d, 4, rng, -1)
    return A, y, x0, z0


def round_config(d=20, n=16, r=64, terms=4, seed=2):
    """Sum of ``terms`` independent rank-``r`` Gaussian TTs (true rank <= terms*r).

    Core entries are N(0, sigma^2) with ``sigma = 1/sqrt(r_k * n)`` (the
    left rank of the core), so every term has O(1) norm growth per core.
    """
    rng = np.random.default_rng(seed)
    x = None
    for _ in range(terms):
        t = tt_randn(n, d, r, rng, scale=lambda r1, nn, r2: 1.0 / np.sqrt(r1 * nn))
        x = t if x is None else tt_plus(x, t)
    return x
