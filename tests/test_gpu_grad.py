"""Gradients with respect to every core, through the C ABI and the
``torch.autograd.Function`` harness.

Checks (FP64): the value against the oracle (1e-12 relative), the gradient
against the FP64 oracle gradient (1e-11 relative per core), and against
central finite differences with h = 1e-6 of the library's own value on
random entries (|fd - g| <= 1e-6 |g| + 1e-8 max(1, |f|)).
"""
import numpy as np
import pytest

import ttgpu
from oracle import grad as og

pytestmark = pytest.mark.gpu

VAL_TOL = 1e-12
GRAD_TOL = 1e-11
FD_H = 1e-6
FD_TOL = 1e-6


def rand_cores(rng, n, r, scale=None):
    cs = []
    for k in range(len(n)):
        s = 1.0 / np.sqrt(r[k] * n[k]) if scale is None else scale
        cs.append(np.asfortranarray(rng.standard_normal((r[k], n[k], r[k + 1])) * s))
    return cs


def to_tt(cs):
    return ttgpu.TensorTrain.from_cores(cs)


def to_mat(cs):
    return ttgpu.TTMatrix.from_cores(cs)


def split(tt, cs):
    out, p = [], 0
    for c in cs:
        out.append(tt.core[p:p + c.size].reshape(c.shape, order="F"))
        p += c.size
    return out


def grad_rel(G, Gref):
    num = np.sqrt(sum(np.sum((g - h) ** 2) for g, h in zip(G, Gref)))
    den = np.sqrt(sum(np.sum(h ** 2) for h in Gref))
    return num / den


def fd_check(ctx, f, cs, G, rng, nprobe=12):
    """Worst ratio |fd - g| / (FD_TOL |g| + 1e-8 max(1, |f|)) over random
    entries (<= 1 passes).  The functionals are at most quadratic in each
    entry, so central differences carry rounding error only, about
    eps |f| / h = 1e-10 |f|."""
    f0 = abs(f(cs))
    worst = 0.0
    for _ in range(nprobe):
        k = int(rng.integers(len(cs)))
        i = tuple(int(rng.integers(s)) for s in cs[k].shape)
        cp = [c.copy() for c in cs]
        cm = [c.copy() for c in cs]
        cp[k][i] += FD_H
        cm[k][i] -= FD_H
        fd = (f(cp) - f(cm)) / (2 * FD_H)
        worst = max(worst, abs(fd - G[k][i]) / (FD_TOL * abs(G[k][i]) + 1e-8 * max(1.0, f0)))
    return worst


def lap_cores(n, d, c=None, nonsym=False, rng=None):
    """Rank-3 operator: Laplacian Kronecker sum plus a separable term
    (nonsymmetric when asked, to exercise both adjoint terms)."""
    cores = []
    for k in range(d):
        L = (n + 1) ** 2 * (2 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1))
        if c is not None:
            L = L * c[k]
        I = np.eye(n)
        M = rng.standard_normal((n, n)) / n if nonsym else np.diag(np.linspace(1, 2, n))
        if k == 0:
            core = np.zeros((1, n, n, 3))
            core[0, :, :, 0], core[0, :, :, 1], core[0, :, :, 2] = L, I, M
        elif k == d - 1:
            core = np.zeros((3, n, n, 1))
            core[0, :, :, 0], core[1, :, :, 0], core[2, :, :, 0] = I, L, M
        else:
            core = np.zeros((3, n, n, 3))
            core[0, :, :, 0] = I
            core[1, :, :, 0] = L
            core[1, :, :, 1] = I
            core[2, :, :, 2] = M
        cores.append(np.asfortranarray(core))
    return cores


@pytest.mark.parametrize("d,n,r,nonsym", [(4, 5, 3, True), (6, 8, 6, False), (5, 7, 9, True)])
def test_grad_xAx(ctx, d, n, r, nonsym):
    rng = np.random.default_rng(d * 100 + r)
    rr = [1] + [r] * (d - 1) + [1]
    xs = rand_cores(rng, [n] * d, rr)
    As = lap_cores(n, d, rng=rng, nonsym=nonsym)
    v, G = ttgpu.grad_xAx(to_tt(xs), to_mat(As), ctx=ctx)
    Gd = split(G, xs)
    vref, Gref = og.xAx(xs, As)
    assert abs(v - vref) <= VAL_TOL * abs(vref)
    assert grad_rel(Gd, Gref) <= GRAD_TOL
    if d * np.log(n) < np.log(5000):  # full-tensor anchor on the tiny case
        assert abs(og.full_xAx(xs, As) - vref) <= 1e-10 * abs(vref)

    def f(cs):
        return ttgpu.grad_xAx(to_tt(cs), to_mat(As), ctx=ctx)[0]
    assert fd_check(ctx, f, xs, Gd, rng) <= 1.0


@pytest.mark.parametrize("d,n,r,rb", [(3, 4, 2, 3), (7, 6, 5, 4), (12, 8, 16, 4)])
def test_grad_xb(ctx, d, n, r, rb):
    rng = np.random.default_rng(d + 7 * r)
    xs = rand_cores(rng, [n] * d, [1] + [r] * (d - 1) + [1])
    bs = rand_cores(rng, [n] * d, [1] + [rb] * (d - 1) + [1])
    v, G = ttgpu.grad_xb(to_tt(xs), to_tt(bs), ctx=ctx)
    Gd = split(G, xs)
    vref, Gref = og.xb(xs, bs)
    # <x,b> of independent Gaussian TTs cancels heavily: bound by |x| |b|
    scale = np.sqrt(og.xb(xs, xs)[0] * og.xb(bs, bs)[0])
    assert abs(v - vref) <= VAL_TOL * scale
    assert grad_rel(Gd, Gref) <= GRAD_TOL

    def f(cs):
        return ttgpu.grad_xb(to_tt(cs), to_tt(bs), ctx=ctx)[0]
    assert fd_check(ctx, f, xs, Gd, rng) <= 1.0


@pytest.mark.parametrize("d,n,r,S", [(3, 4, 2, 50), (5, 7, 9, 3000), (6, 32, 20, 20000),
                                     (4, 3, 70, 5000)])
def test_grad_sampled(ctx, d, n, r, S):
    rng = np.random.default_rng(S + d)
    xs = rand_cores(rng, [n] * d, [1] + [r] * (d - 1) + [1])
    idx = np.stack([rng.integers(0, n, S) for _ in range(d)], axis=1)
    y = og.entries(rand_cores(rng, [n] * d, [1] + [3] * (d - 1) + [1]), idx)
    y = y + 1e-3 * rng.standard_normal(S)
    v, G = ttgpu.grad_sampled(to_tt(xs), idx, y, ctx=ctx)
    Gd = split(G, xs)
    vref, Gref = og.sampled(xs, idx, y)
    assert abs(v - vref) <= VAL_TOL * abs(vref)
    assert grad_rel(Gd, Gref) <= GRAD_TOL
    if S <= 100:
        assert abs(og.full_sampled(xs, idx, y) - vref) <= 1e-12 * abs(vref)

    def f(cs):
        return ttgpu.grad_sampled(to_tt(cs), idx, y, ctx=ctx)[0]
    assert fd_check(ctx, f, xs, Gd, rng, nprobe=8) <= 1.0


def test_grad_sampled_repeatable_and_edges(ctx):
    rng = np.random.default_rng(3)
    n, d, r = 6, 4, 5
    xs = rand_cores(rng, [n] * d, [1] + [r] * (d - 1) + [1])
    # all samples in one bucket of core 2, an empty bucket elsewhere
    idx = np.stack([rng.integers(0, n - 1, 777) for _ in range(d)], axis=1)
    idx[:, 2] = 4
    y = rng.standard_normal(777)
    v1, G1 = ttgpu.grad_sampled(to_tt(xs), idx, y, ctx=ctx)
    v2, G2 = ttgpu.grad_sampled(to_tt(xs), idx, y, ctx=ctx)
    assert v1 == v2 and np.array_equal(G1.core, G2.core)  # bitwise repeatable
    vref, Gref = og.sampled(xs, idx, y)
    assert grad_rel(split(G1, xs), Gref) <= GRAD_TOL
    assert np.all(split(G1, xs)[0][:, n - 1, :] == 0.0)  # empty bucket
    # no samples: zero loss and gradient
    v0, G0 = ttgpu.grad_sampled(to_tt(xs), np.zeros((0, d), np.int64), np.zeros(0), ctx=ctx)
    assert v0 == 0.0 and not np.any(G0.core)
    # out-of-range index fails loudly
    bad = idx.copy()
    bad[5, 1] = n
    with pytest.raises(ttgpu.TTGError, match="out of range"):
        ttgpu.grad_sampled(to_tt(xs), bad, y, ctx=ctx)
    bad[5, 1] = -1
    with pytest.raises(ttgpu.TTGError, match="out of range"):
        ttgpu.grad_sampled(to_tt(xs), bad, y, ctx=ctx)


def test_grad_shape_errors(ctx):
    rng = np.random.default_rng(4)
    xs = rand_cores(rng, [4] * 3, [1, 2, 2, 1])
    As = lap_cores(5, 3, rng=rng)
    with pytest.raises(ttgpu.TTGError, match="A is"):
        ttgpu.grad_xAx(to_tt(xs), to_mat(As), ctx=ctx)
    bs = rand_cores(rng, [4] * 2, [1, 2, 1])
    with pytest.raises(ttgpu.TTGError, match="cores"):
        ttgpu.grad_xb(to_tt(xs), to_tt(bs), ctx=ctx)


def test_torch_autograd_harness(ctx):
    import ttgpu.autograd as ta
    import torch
    rng = np.random.default_rng(11)
    d, n, r = 5, 6, 4
    xs = rand_cores(rng, [n] * d, [1] + [r] * (d - 1) + [1])
    As = lap_cores(n, d, rng=rng, nonsym=True)
    bs = rand_cores(rng, [n] * d, [1] + [2] * (d - 1) + [1])
    idx = np.stack([rng.integers(0, n, 400) for _ in range(d)], axis=1)
    y = rng.standard_normal(400)
    x = to_tt(xs)
    core = torch.tensor(x.core, dtype=torch.float64, device="cuda", requires_grad=True)
    loss = (ta.xAx(core, x.n, x.r, to_mat(As)) - 2.0 * ta.xb(core, x.n, x.r, to_tt(bs))
            + 0.5 * ta.sampled_loss(core, x.n, x.r, idx, y))
    loss.backward()
    ga = core.grad.cpu().numpy()
    ref = (np.concatenate([g.ravel(order="F") for g in og.xAx(xs, As)[1]])
           - 2.0 * np.concatenate([g.ravel(order="F") for g in og.xb(xs, bs)[1]])
           + 0.5 * np.concatenate([g.ravel(order="F") for g in og.sampled(xs, idx, y)[1]]))
    assert np.linalg.norm(ga - ref) <= GRAD_TOL * np.linalg.norm(ref)
    # torch's own finite-difference checker on the xb functional (linear in core)
    core2 = torch.tensor(x.core, dtype=torch.float64, device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(lambda c: ta.xb(c, x.n, x.r, to_tt(bs)), (core2,),
                                    eps=FD_H, atol=1e-7, rtol=1e-6)


def test_grad_d12_n32_r64_full_size(ctx):
    """The differentiation workload at its full size (d=12, n=32, rank-64 x,
    rank-3 operator, rank-4 b, 1e6 samples from a hidden rank-8 TT plus
    N(0, 1e-3^2) noise) against the FP64 oracle."""
    from ttgpu import workloads
    x, A, b, idx, y = workloads.grad_inputs()
    xc = x.cores()
    Ac, p = [], 0
    for k in range(A.d):
        shp = (int(A.r[k]), int(A.n[k]), int(A.m[k]), int(A.r[k + 1]))
        Ac.append(A.core[p:p + int(np.prod(shp))].reshape(shp, order="F"))
        p += int(np.prod(shp))
    for name, call, ref in [
            ("xAx", lambda: ttgpu.grad_xAx(x, A, ctx=ctx), lambda: og.xAx(xc, Ac)),
            ("xb", lambda: ttgpu.grad_xb(x, b, ctx=ctx), lambda: og.xb(xc, b.cores())),
            ("sampled", lambda: ttgpu.grad_sampled(x, idx, y, ctx=ctx),
             lambda: og.sampled(xc, idx, y))]:
        v, G = call()
        vr, Gr = ref()
        scale = abs(vr) if name != "xb" else np.sqrt(og.xb(xc, xc)[0] * og.xb(b.cores(),
                                                                             b.cores())[0])
        assert abs(v - vr) <= 1e-11 * scale, name
        assert grad_rel(split(G, xc), Gr) <= GRAD_TOL, name
