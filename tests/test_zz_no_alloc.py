"""The allocation-free local matvec, ttg_local_matvec_noalloc, checked against
the allocating ttg_local_matvec through the C ABI.

It exists for callers that may not allocate device memory (a host whose
memory is owned by another pool, a time-critical loop that must not meet
cudaMalloc's synchronisation or out-of-memory failure, a plugin host whose
memory manager forbids untracked allocations): they pass only inputs and
outputs, and the intermediates live in a fixed 64 MiB array inside the
library.  This file is collected last so that a run stopping at its first
failure has already run every other test; it creates its own context, so it
also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import ttgpu

pytestmark = pytest.mark.gpu

KERNEL_TOL = 1e-12  # the FP64 kernel-level parity tolerance used by the other tests


def _dev(ctx, a):
    return ctx.to_device(np.asarray(a, dtype=np.float64).ravel(order="F"))


def _allocating(ctx, dims, P1, A, P2, x):
    rx1, n, rx2, ra1, ra2 = dims
    y = ctx.empty(rx1 * n * rx2)
    ttgpu._check(ttgpu.lib().ttg_local_matvec(ctx.h, rx1, n, rx2, ra1, ra2, P1.p, A.p, P2.p,
                                              x.p, y.p, ttgpu.TTG_FP64))
    return y.get()


def _noalloc(ctx, dims, P1, A, P2, x):
    rx1, n, rx2, ra1, ra2 = dims
    y = ctx.empty(rx1 * n * rx2)
    ttgpu._check(ttgpu.lib().ttg_local_matvec_noalloc(None, rx1, n, rx2, ra1, ra2, P1.p, A.p,
                                                      P2.p, x.p, y.p))
    return y.get()


@pytest.mark.parametrize("dims", [(61, 64, 59, 3, 3), (17, 8, 9, 2, 2), (1, 64, 4, 1, 3)])
def test_noalloc_matches_allocating_matvec_on_two_calls(dims):
    ctx = ttgpu.Context(0)
    try:
        rx1, n, rx2, ra1, ra2 = dims
        rng = np.random.default_rng(sum(dims))
        P1 = _dev(ctx, rng.standard_normal((rx1, rx1, ra1)))
        A = _dev(ctx, rng.standard_normal((ra1, n, n, ra2)))
        P2 = _dev(ctx, rng.standard_normal((rx2, ra2, rx2)))
        for call in range(2):  # two calls in a row, different inputs
            x = _dev(ctx, rng.standard_normal(rx1 * n * rx2))
            ref = _allocating(ctx, dims, P1, A, P2, x)
            got = _noalloc(ctx, dims, P1, A, P2, x)
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err < KERNEL_TOL, (call, err)
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    ctx = ttgpu.Context(0)
    try:
        dummy = ctx.empty(16)
        code = ttgpu.lib().ttg_local_matvec_noalloc(None, 400, 64, 400, 3, 3, dummy.p, dummy.p,
                                                    dummy.p, dummy.p, dummy.p)
        assert code == 1
        assert b"scratch" in ttgpu.lib().ttg_last_error()
    finally:
        ctx.close()
