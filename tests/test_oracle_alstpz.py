"""CPU tests of the ALS(t+z) oracle (``oracle/alstpz.py``, a restatement of
``solve/alstpz_solve.m``).  The reference has no tests or golden vectors
for this solver: the oracle is checked by what the algorithm guarantees --
convergence of the true residual on Laplacian systems, the zero-weight
enrichment leaving the tensor unchanged, and the dense and structured local
branches agreeing."""
import numpy as np
import pytest

from oracle.alstpz import als_sweep, alstpz_solve
from oracle.builders import aniso_config, laplace_config
from oracle.round import tt_round
from oracle.tt import tt_matvec, tt_norm, tt_plus, true_residual


@pytest.mark.parametrize("d,n", [(4, 8), (6, 16)])
def test_alstpz_converges_on_laplacian(d, n):
    A, y, x0, _ = laplace_config(d=d, n=n)
    x, info = alstpz_solve(A, y, 1e-8, x0)
    assert info["sweeps"] == 10                      # no stopping test (:138)
    assert true_residual(A, x, y) < 1e-8
    assert info["max_res"][-1] < info["max_res"][0]


def test_zero_weight_enrichment_keeps_the_tensor():
    A, y, x0, _ = laplace_config(d=4, n=8)
    x, _ = tt_round(x0, 1e-8)
    z, _ = tt_round(tt_plus(y, tt_matvec(A, x) * (-1.0)), 1e-8, 4)
    xe = tt_plus(x, z * 0.0)
    assert list(xe.r[1:-1]) == [int(a + b) for a, b in zip(x.r[1:-1], z.r[1:-1])]
    assert np.array_equal(xe.full(), x.full())


def test_dense_and_structured_local_solves_agree():
    A, y, x0, _ = aniso_config(d=4, n=8, seed=1)
    xa, ia = als_sweep(A, y, 1e-10, x0, max_full_size=10 ** 9)   # every core dense
    xb, ib = als_sweep(A, y, 1e-10, x0, max_full_size=0)         # every core GMRES
    assert list(xa.r) == list(xb.r)
    assert tt_norm(xa - xb) <= 1e-7 * tt_norm(xa)
