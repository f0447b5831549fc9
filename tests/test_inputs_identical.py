"""The GPU library's inputs are the oracle's inputs, byte for byte.

``bench.py`` feeds the device from ``ttgpu.workloads`` and the CPU arm from
``oracle.builders``: two copies of the same seeded formulas (the product
side may not import the oracle).  Every benchmark workload at its full size
is built both ways here and compared with ``array_equal`` (bitwise equality
of the float64 arrays)."""
import numpy as np
import pytest

from oracle import builders
from ttgpu import workloads


def _same_tt(a, b):
    assert list(a.n) == [int(v) for v in b.n]
    assert list(a.r) == [int(v) for v in b.r]
    assert np.array_equal(np.asarray(a.core, np.float64), b.flat())


def _same_mat(a, b):
    assert list(a.n) == [int(v) for v in b.n]
    assert list(a.m) == [int(v) for v in b.m]
    assert list(a.r) == [int(v) for v in b.r]
    assert np.array_equal(np.asarray(a.core, np.float64), b.flat())


@pytest.mark.parametrize("d,n", [(8, 32), (4, 8), (6, 16)])
def test_laplace_workload_identical(d, n):
    got = workloads.laplace(d=d, n=n)
    ref = builders.laplace_config(d=d, n=n)
    _same_mat(got[0], ref[0])
    for g, r in zip(got[1:], ref[1:]):
        _same_tt(g, r)


@pytest.mark.parametrize("d,n,seed", [(10, 64, 3), (5, 16, 3)])
def test_aniso_workload_identical(d, n, seed):
    got = workloads.aniso(d=d, n=n, seed=seed)
    ref = builders.aniso_config(d=d, n=n, seed=seed)
    _same_mat(got[0], ref[0])
    for g, r in zip(got[1:], ref[1:]):
        _same_tt(g, r)


def test_round_workload_identical():
    """The rounding input at full size: d=20, n=16, four rank-64 terms."""
    _same_tt(workloads.round_input(d=20, n=16, r=64, terms=4, seed=2),
             builders.round_config(d=20, n=16, r=64, terms=4, seed=2))
