"""Programmatic dependent launch changes only when kernels are scheduled,
never what they compute: a context created with ``TTG_PDL=0`` (plain
stream-ordered launches) must reproduce the default context's solve bit for
bit (every reduction of the library runs in a fixed order)."""
import os

import numpy as np
import pytest

import ttgpu
from ttgpu import workloads

pytestmark = pytest.mark.gpu


def _solve(precision, pdl):
    old = os.environ.get("TTG_PDL")
    os.environ["TTG_PDL"] = "1" if pdl else "0"
    try:
        ctx = ttgpu.Context(0)
    finally:
        if old is None:
            del os.environ["TTG_PDL"]
        else:
            os.environ["TTG_PDL"] = old
    try:
        A, y, x0, z0 = workloads.aniso(d=5, n=24, seed=7)
        dA, dy = ttgpu.DeviceTT.upload(ctx, A), ttgpu.DeviceTT.upload(ctx, y)
        dx0, dz0 = ttgpu.DeviceTT.upload(ctx, x0), ttgpu.DeviceTT.upload(ctx, z0)
        st = {}
        x = ttgpu.amen_solve2(dA, dy, 1e-9, x0=dx0, z0=dz0, ctx=ctx, stats=st, rmax=40,
                              nswp=20, precision=precision)
        h = x.download()
        for t in (x, dA, dy, dx0, dz0):
            t.free()
        return h, st
    finally:
        ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pdl_off_reproduces_default(precision):
    x1, s1 = _solve(precision, True)
    x0, s0 = _solve(precision, False)
    assert list(x1.r) == list(x0.r)
    assert s1["sweeps"] == s0["sweeps"]
    assert np.array_equal(np.asarray(x1.core), np.asarray(x0.core))
