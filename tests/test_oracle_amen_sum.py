"""CPU checks of the ``amen_sum`` oracle (``core/amen_sum.m``).

The reference has no tests or golden vectors for ``amen_sum``; the oracle is
pinned by what the algorithm must give: the exact linear combination when
the tolerance is tight (full-tensor comparison at small d), ranks no larger
than those of the exact result, and an error of the order of the tolerance
when it is loose.
"""
import numpy as np

from oracle.amen_sum import amen_sum
from oracle.tt import TT, tt_rand, tt_randn


def _full_with_outputs(y):
    """Full array of a TT whose last rank M indexes the outputs."""
    M = int(y.r[-1])
    return TT(y.cores + [np.eye(M).reshape(M, M, 1)]).full()


def _exact(X, c):
    return sum(np.multiply.outer(Xj.full(), c[j]) for j, Xj in enumerate(X))


def test_amen_sum_exact_combination_two_outputs():
    rng = np.random.default_rng(0)
    d, n = 5, 5
    X = [tt_randn(n, d, r, rng) for r in (2, 3, 2)]
    c = rng.standard_normal((3, 2))
    y, z, info = amen_sum(X, c, 1e-10, tt_randn(n, d, 2, rng), tt_rand(n, d, 4, rng))
    F = _exact(X, c)
    Y = _full_with_outputs(y)
    assert Y.shape == F.shape
    assert np.linalg.norm(Y - F) / np.linalg.norm(F) < 1e-12
    assert int(y.r[-1]) == 2
    assert max(y.r) <= 7                       # sum of the summands' ranks
    assert info["max_dx"][-1] < 1e-10


def test_amen_sum_cancelling_summands_keep_the_small_rank():
    rng = np.random.default_rng(1)
    d, n = 6, 4
    x = tt_randn(n, d, 3, rng)
    w = tt_randn(n, d, 2, rng)
    c = np.array([[1.0], [-1.0], [2.0]])
    y, _, _ = amen_sum([x, x, w], c, 1e-10, tt_randn(n, d, 2, rng), tt_rand(n, d, 4, rng))
    F = 2.0 * w.full()
    Y = _full_with_outputs(y)[..., 0]
    assert np.linalg.norm(Y - F) / np.linalg.norm(F) < 1e-12
    assert all(int(a) <= int(b) for a, b in zip(y.r[1:-1], w.r[1:-1]))


def test_amen_sum_loose_tolerance():
    """Summands of overall norms 3e3, 3e1, 3e-1, 3e-3: at tol 1e-3 the last two
    drop out (rank 3 + 3), at 1e-6 one more joins; the error follows tol."""
    rng = np.random.default_rng(2)
    d, n = 6, 6
    # overall scales 1, 1e-2, 1e-4, 1e-6 (the scale multiplies every core)
    X = [tt_randn(n, d, 3, rng, scale=s ** (1.0 / d)) for s in (1.0, 1e-2, 1e-4, 1e-6)]
    c = np.ones((4, 1))
    F = _exact(X, c)[..., 0]
    for tol, rank in ((1e-3, 6), (1e-6, 9)):
        y, _, _ = amen_sum(X, c, tol, tt_randn(n, d, 2, rng), tt_rand(n, d, 4, rng))
        Y = _full_with_outputs(y)[..., 0]
        err = np.linalg.norm(Y - F) / np.linalg.norm(F)
        assert err < 2 * tol
        assert max(int(r) for r in y.r) == rank
