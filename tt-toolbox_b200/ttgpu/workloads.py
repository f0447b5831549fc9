"""Seeded synthetic inputs of the benchmark workloads (host side).

The reference publishes no benchmark data for this path; these generators
produce the operators/right-hand sides that its experiment scripts build
(``tests/test_amen_laplace.m:27-29``: a Laplacian in TT-matrix form and a TT
right-hand side) with explicit seeds, so the GPU library and the CPU oracle
see identical bytes.  Formulas:

* 1D stencil ``L = (n+1)^2 tridiag(-1, 2, -1)``; mass ``M = tridiag(1,4,1)/6``.
* Kronecker sum ``sum_k I x .. x L_k x .. x I`` as rank-2 TT-matrix cores
  (first ``[L I]``, middle ``[[I 0];[L I]]``, last ``[I; L]``); an optional
  separable term ``M_1 x .. x M_d`` extends every core block-diagonally to
  rank 3.
* Gaussian TT cores drawn from ``numpy.random.default_rng(seed)``.
"""
import numpy as np

from . import TensorTrain, TTMatrix


def lap1d(n):
    L = 2.0 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1)
    return (n + 1) ** 2 * L


def mass1d(n):
    return (4.0 * np.eye(n) + np.eye(n, k=1) + np.eye(n, k=-1)) / 6.0


def kron_sum_cores(mats, react=None):
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
        cores.append(c)
    return cores


def randn_cores(n, d, r, rng, scale=1.0):
    nn = [n] * d if np.isscalar(n) else list(n)
    rr = [1] + [r] * (d - 1) + [1] if np.isscalar(r) else list(r)
    cores = []
    for k in range(d):
        s = scale if not callable(scale) else scale(rr[k], nn[k], rr[k + 1])
        cores.append(rng.standard_normal((rr[k], nn[k], rr[k + 1])) * s)
    return cores


def rand_orth_cores(n, d, r, rng):
    """Right-to-left orthogonal random TT (``core/tt_rand.m:52-57``)."""
    nn = [n] * d if np.isscalar(n) else list(n)
    rr = [1] + [r] * (d - 1) + [1]
    cores = [None] * d
    for i in range(d - 1, -1, -1):
        g = rng.standard_normal((nn[i] * rr[i + 1], rr[i])).copy(order="F")
        q, _ = np.linalg.qr(g)
        q = q.T
        rr[i] = q.shape[0]
        cores[i] = q.reshape((rr[i], nn[i], rr[i + 1]), order="F")
    return cores


def laplace(d=8, n=32, x_rank=2, seed=1):
    """d-dim Laplacian (rank 2), RHS all-ones, x0 N(0,1) rank ``x_rank``, z0 rank 4."""
    rng = np.random.default_rng(seed)
    A = TTMatrix.from_cores(kron_sum_cores([lap1d(n)] * d))
    y = TensorTrain.from_cores([np.ones((1, n, 1)) for _ in range(d)])
    x0 = TensorTrain.from_cores(randn_cores(n, d, x_rank, rng))
    z0 = TensorTrain.from_cores(rand_orth_cores(n, d, 4, rng))
    return A, y, x0, z0


def aniso(d=10, n=64, rhs_rank=4, seed=3, react_scale=1.0):
    """Anisotropic diffusion ``sum_k c_k L_k`` (``c_k ~ U[0.5, 2]``) plus the
    separable reaction ``sigma M x .. x M`` (``sigma = (n+1)^2``): operator TT
    rank 3; RHS seeded rank-4 Gaussian TT; x0 rank 2; z0 rank 4."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.5, 2.0, size=d)
    sigma = react_scale * (n + 1) ** 2
    M = mass1d(n)
    react = [M * (sigma if k == 0 else 1.0) for k in range(d)]
    A = TTMatrix.from_cores(kron_sum_cores([c[k] * lap1d(n) for k in range(d)], react))
    y = TensorTrain.from_cores(randn_cores(n, d, rhs_rank, rng))
    x0 = TensorTrain.from_cores(randn_cores(n, d, 2, rng))
    z0 = TensorTrain.from_cores(rand_orth_cores(n, d, 4, rng))
    return A, y, x0, z0


def tt_sum_cores(a, b):
    d = len(a)
    out = []
    for k in range(d):
        ca, cb = a[k], b[k]
        r1a, n, r2a = ca.shape
        r1b, _, r2b = cb.shape
        if k == 0:
            c = np.zeros((r1a, n, r2a + r2b))
            c[:, :, :r2a] = ca
            c[:, :, r2a:] = cb
        elif k == d - 1:
            c = np.zeros((r1a + r1b, n, r2a))
            c[:r1a] = ca
            c[r1a:] = cb
        else:
            c = np.zeros((r1a + r1b, n, r2a + r2b))
            c[:r1a, :, :r2a] = ca
            c[r1a:, :, r2a:] = cb
        out.append(c)
    return out


def round_input(d=20, n=16, r=64, terms=4, seed=2):
    """Sum of ``terms`` independent rank-``r`` Gaussian TTs, entries
    N(0, 1/(r_k n)) (rank concatenation as ``@tt_tensor/plus.m:49-86``)."""
    rng = np.random.default_rng(seed)
    x = None
    for _ in range(terms):
        t = randn_cores(n, d, r, rng, scale=lambda r1, nn, r2: 1.0 / np.sqrt(r1 * nn))
        x = t if x is None else tt_sum_cores(x, t)
    return TensorTrain.from_cores(x)


def grad_inputs(d=12, n=32, r=64, rb=4, nsamples=1_000_000, hidden_rank=8, noise=1e-3,
                seed=9):
    """Differentiation workload: x rank ``r`` with N(0, 1/(r_k n)) entries;
    A the rank-3 operator of ``aniso`` with c_k = 1; b rank ``rb`` Gaussian;
    ``nsamples`` uniform 0-based multi-indices (int32 ``[S, d]``) and values
    of a hidden rank-``hidden_rank`` TT at them plus N(0, noise^2)."""
    rng = np.random.default_rng(seed)
    sc = lambda r1, nn, r2: 1.0 / np.sqrt(r1 * nn)  # noqa: E731
    x = TensorTrain.from_cores(randn_cores(n, d, r, rng, scale=sc))
    M = mass1d(n)
    sigma = (n + 1) ** 2
    react = [M * (sigma if k == 0 else 1.0) for k in range(d)]
    A = TTMatrix.from_cores(kron_sum_cores([lap1d(n)] * d, react))
    b = TensorTrain.from_cores(randn_cores(n, d, rb, rng, scale=sc))
    idx = rng.integers(0, n, size=(nsamples, d), dtype=np.int32)
    hidden = randn_cores(n, d, hidden_rank, rng, scale=sc)
    v = np.ones((nsamples, 1))
    for k in range(d):
        core = hidden[k]
        out = np.empty((nsamples, core.shape[2]))
        col = idx[:, k]
        for j in range(n):
            m = col == j
            out[m] = v[m] @ core[:, j, :]
        v = out
    y = v[:, 0] + noise * rng.standard_normal(nsamples)
    return x, A, b, idx, y


def batch_systems(count=512, seed=4, d_range=(6, 14), n_choices=(8, 16, 32, 64),
                  rmax_range=(8, 64)):
    """Batched-solve workload: ``count`` independent Laplacian systems
    (operator rank 2, RHS all-ones rank 1), d ~ U{d_range}, n from
    ``n_choices``, rmax ~ U{rmax_range}, all from one seeded generator.
    Returns (As, ys, rmaxs, shapes)."""
    rng = np.random.default_rng(seed)
    As, ys, rmaxs, shapes = [], [], [], []
    cache = {}
    for _ in range(count):
        d = int(rng.integers(d_range[0], d_range[1] + 1))
        n = int(rng.choice(n_choices))
        r = int(rng.integers(rmax_range[0], rmax_range[1] + 1))
        key = (d, n)
        if key not in cache:
            cache[key] = (TTMatrix.from_cores(kron_sum_cores([lap1d(n)] * d)),
                          TensorTrain.from_cores([np.ones((1, n, 1)) for _ in range(d)]))
        A, y = cache[key]
        As.append(A)
        ys.append(y)
        rmaxs.append(r)
        shapes.append((d, n, r))
    return As, ys, rmaxs, shapes
