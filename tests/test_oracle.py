"""CPU tests of the FP64 oracle, pinned against the reference's fixtures.

The reference's own MATLAB path cannot run here; its known-answer fixtures
(``tests/tt-solve/*.mat``, converted to ``tests/golden/*.npz``) and
mathematical invariants pin the oracle.
"""
import os

import numpy as np
import pytest

from golden_io import load_fixture
from oracle.amen import amen_solve2, bfun3, compute_next_Phi, dgmresr_hh, solve3d_2
from oracle.builders import aniso_config, kron_sum_operator, lap1d, laplace_config, round_config
from oracle.round import my_chop2, tt_round
from oracle.tt import (TT, TTMatrix, tt_dot, tt_matvec, tt_norm, tt_plus, tt_rand, tt_randn,
                       true_residual)

# Relative residuals of the stored solutions, as listed for the reference's
# fixtures (recomputed with the QR-based TT norm).
FIXTURE_RESIDUALS = {"ex2": 2.10e-6, "ex2_1": 2.81e-6, "ex6": 3.12e-4}


@pytest.mark.parametrize("key", sorted(FIXTURE_RESIDUALS))
def test_fixture_residuals(key):
    A, rhs, x, stored = load_fixture(key)
    res = true_residual(A, x, rhs)
    assert res == pytest.approx(stored, rel=1e-8)
    assert res == pytest.approx(FIXTURE_RESIDUALS[key], rel=2e-2)


def test_tt_algebra_vs_full():
    rng = np.random.default_rng(0)
    a = tt_randn([3, 4, 2, 3], 4, 3, rng)
    b = tt_randn([3, 4, 2, 3], 4, 2, rng)
    fa, fb = a.full(), b.full()
    assert np.allclose((a + b).full(), fa + fb)
    assert tt_norm(a) == pytest.approx(np.linalg.norm(fa), rel=1e-12)
    assert tt_dot(a, b) == pytest.approx(np.sum(fa * fb), rel=1e-12)
    A = kron_sum_operator([lap1d(k) for k in [3, 4, 2, 3]])
    Ax = tt_matvec(A, a).full().ravel(order="F")
    assert np.allclose(Ax, A.full() @ fa.ravel(order="F"))


def test_my_chop2_cases():
    s = np.array([10.0, 1.0, 0.1, 0.01])
    assert my_chop2(s, 0.0) == 4
    assert my_chop2(np.zeros(3), 1.0) == 1
    # sqrt(0.01^2) < 0.05 -> drop one; sqrt(0.1^2+0.01^2) > 0.05 -> keep 3
    assert my_chop2(s, 0.05) == 3
    assert my_chop2(s, 0.2) == 2
    assert my_chop2(s, 100.0) == 0


def test_round_exact_rank_and_bound():
    x = round_config(d=6, n=4, r=3, terms=3, seed=7)
    assert list(x.r) == [1, 9, 9, 9, 9, 9, 1]
    y, info = tt_round(x, 1e-12)
    # exact ranks of a sum of three rank-3 terms, capped by the mode products
    assert list(y.r) == [1, 4, 9, 9, 9, 4, 1]
    assert tt_norm(y - x) / tt_norm(x) < 1e-12
    z, _ = tt_round(x, 0.3)
    assert tt_norm(z - x) / tt_norm(x) <= 0.3
    w, _ = tt_round(x, 1e-12, 2)
    assert max(w.r) <= 2


def test_bfun3_matches_dense():
    rng = np.random.default_rng(1)
    rx1, n, rx2, ra1, ra2 = 3, 4, 5, 2, 3
    Phi1 = rng.standard_normal((rx1, rx1, ra1))
    A = rng.standard_normal((ra1, n, n, ra2))
    Phi2 = rng.standard_normal((rx2, ra2, rx2))
    x = rng.standard_normal(rx1 * n * rx2)
    y = bfun3(Phi1, A, Phi2, x)
    ref = np.einsum("iaq,qjmb,cbk,amc->ijk", Phi1, A, Phi2,
                    x.reshape(rx1, n, rx2, order="F")).ravel(order="F")
    assert np.allclose(y, ref, rtol=1e-12, atol=1e-12)


def test_next_phi_matches_einsum():
    rng = np.random.default_rng(2)
    rx1, n, rx2, ry1, ry2, ra1, ra2 = 3, 4, 5, 2, 3, 2, 3
    x = rng.standard_normal((rx1, n, rx2))
    y = rng.standard_normal((ry1, n, ry2))
    A = rng.standard_normal((ra1, n, n, ra2))
    P = rng.standard_normal((rx1, ry1, ra1))
    out, _ = compute_next_Phi(P, x, A, y, "lr")
    assert np.allclose(out, np.einsum("anc,abq,qnmr,bme->cer", x, P, A, y))
    P = rng.standard_normal((ry2, ra2, rx2))
    out, _ = compute_next_Phi(P, x, A, y, "rl")
    assert np.allclose(out, np.einsum("yme,erc,qjmr,ajc->yqa", y, P, A, x))
    out, nrm = compute_next_Phi(rng.standard_normal((rx1, ry1)), x, None, y, "lr", want_norm=True)
    assert np.linalg.norm(out) == pytest.approx(1.0)


def test_gmres_hh_solves_small_system():
    rng = np.random.default_rng(3)
    N = 60
    B = np.eye(N) * 4 + rng.standard_normal((N, N)) * 0.3
    b = rng.standard_normal(N)
    st = {}
    x = dgmresr_hh(lambda v: B @ v, b, 40, 1e-12, 3, st)
    assert np.linalg.norm(B @ x - b) / np.linalg.norm(b) < 1e-10
    assert st["matvecs"] > 1


def test_amen_oracle_matches_dense_solve():
    rng = np.random.default_rng(0)
    d, n = 4, 6
    mats = [lap1d(n) + 30 * rng.standard_normal((n, n)) for _ in range(d)]
    A = kron_sum_operator(mats)
    y = tt_randn(n, d, 2, rng)
    x0 = tt_rand(n, d, 2, rng, -1)
    x, info = amen_solve2(A, y, 1e-10, x0, nswp=30, max_full_size=0)
    xe = np.linalg.solve(A.full(), y.full().ravel(order="F"))
    err = np.linalg.norm(x.full().ravel(order="F") - xe) / np.linalg.norm(xe)
    assert err < 1e-9


def test_amen_oracle_laplace_config():
    A, y, x0, z0 = laplace_config(d=6, n=16)
    x, info = amen_solve2(A, y, 1e-6, x0, z0, rmax=20)
    assert info["max_res"][-1] < 1e-6
    assert true_residual(A, x, y) < 1e-5


def test_amen_oracle_refines_fixture_solution():
    """Started from the reference's stored solution of ex2, AMEn keeps (and
    improves) the published residual."""
    A, rhs, xs, stored = load_fixture("ex2")
    x, info = amen_solve2(A, rhs, 1e-6, xs, nswp=2)
    assert true_residual(A, x, rhs) < stored


def test_solve3d_2_oracle_reduces_residual():
    A, y, x0, z0 = laplace_config(d=4, n=8)
    rng = np.random.default_rng(4)
    rx1, rx2 = 3, 4
    ra1, ra2 = 2, 2
    Phi1 = rng.standard_normal((rx1, rx1, ra1))
    Phi1 = Phi1 + np.transpose(Phi1, (1, 0, 2))
    Phi1[:, :, 0] += 10 * np.eye(rx1)
    Phi2 = rng.standard_normal((rx2, ra2, rx2))
    Phi2[:, 1, :] = np.eye(rx2)
    Ak = A.cores[1]
    rhs = rng.standard_normal(rx1 * 8 * rx2)
    sol0 = np.zeros_like(rhs)
    sol = solve3d_2(Phi1, Ak, Phi2, rhs, 1e-8, sol0, 40, 2)
    r0 = np.linalg.norm(rhs)
    r1 = np.linalg.norm(bfun3(Phi1, Ak, Phi2, sol) - rhs)
    assert r1 < 0.5 * r0


def test_aniso_operator_rank3_matches_dense():
    A, y, x0, z0 = aniso_config(d=3, n=5)
    assert list(A.r) == [1, 3, 3, 1]
    from oracle.builders import mass1d
    rng = np.random.default_rng(3)
    c = rng.uniform(0.5, 2.0, size=3)
    I = np.eye(5)
    L = lap1d(5)
    M = mass1d(5)
    # column-major multi-index: first mode fastest -> kron(A3, A2, A1)
    dense = (np.kron(I, np.kron(I, c[0] * L)) + np.kron(I, np.kron(c[1] * L, I)) +
             np.kron(c[2] * L, np.kron(I, I)) + 36.0 * np.kron(M, np.kron(M, M)))
    assert np.allclose(A.full(), dense)


def _fd_grad_check(f, cs, G, rng, nprobe=10, h=1e-6):
    f0 = abs(f(cs))
    for _ in range(nprobe):
        k = int(rng.integers(len(cs)))
        i = tuple(int(rng.integers(s)) for s in cs[k].shape)
        cp = [c.copy() for c in cs]
        cm = [c.copy() for c in cs]
        cp[k][i] += h
        cm[k][i] -= h
        fd = (f(cp) - f(cm)) / (2 * h)
        assert abs(fd - G[k][i]) <= 1e-6 * abs(G[k][i]) + 1e-8 * max(1.0, f0)


def test_grad_oracle_vs_full_tensor_and_fd():
    """The oracle's sweep gradients against the full-tensor functionals
    (value) and central differences (h = 1e-6) on a nonsymmetric operator."""
    from oracle import grad as og
    rng = np.random.default_rng(21)
    n, r, ra, rb = [3, 4, 2, 3], [1, 2, 3, 2, 1], [1, 2, 3, 2, 1], [1, 3, 2, 2, 1]
    xs = [rng.standard_normal((r[k], n[k], r[k + 1])) for k in range(4)]
    As = [rng.standard_normal((ra[k], n[k], n[k], ra[k + 1])) for k in range(4)]
    bs = [rng.standard_normal((rb[k], n[k], rb[k + 1])) for k in range(4)]
    idx = np.stack([rng.integers(0, n[k], 60) for k in range(4)], axis=1)
    y = rng.standard_normal(60)
    for f_sweep, f_full, arg in [(og.xAx, og.full_xAx, As), (og.xb, og.full_xb, bs)]:
        v, G = f_sweep(xs, arg)
        assert v == pytest.approx(f_full(xs, arg), rel=1e-12)
        _fd_grad_check(lambda cs: f_full(cs, arg), xs, G, rng)
    v, G = og.sampled(xs, idx, y)
    assert v == pytest.approx(og.full_sampled(xs, idx, y), rel=1e-12)
    assert np.allclose(og.entries(xs, idx), og.full_tensor(xs)[tuple(idx.T)], rtol=1e-13)
    _fd_grad_check(lambda cs: og.full_sampled(cs, idx, y), xs, G, rng)


@pytest.mark.parametrize("prec", [1, 2, 3])
def test_jacobi_preconditioners_invert_their_blocks(prec):
    """jac_gen/jac_apply (solve3d_2ml.m:21-70,120-146): P inverts the chosen
    diagonal blocks of the dense local matrix B, and the preconditioned local
    solve reaches the same solution as the plain one."""
    from oracle.amen import assemble_local, jac_apply, jac_gen, solve3d_2
    rng = np.random.default_rng(prec)
    rx1, n, rx2, ra1, ra2 = 3, 4, 2, 2, 3
    Phi1 = rng.standard_normal((rx1, rx1, ra1)) + 4 * np.eye(rx1)[:, :, None]
    Phi2 = rng.standard_normal((rx2, ra2, rx2)) + 4 * np.eye(rx2)[:, None, :]
    A = rng.standard_normal((ra1, n, n, ra2)) + 4 * np.eye(n)[None, :, :, None]
    B = assemble_local(Phi1, A, Phi2)
    N = rx1 * n * rx2
    P = np.stack([jac_apply(jac_gen(Phi1, A, Phi2, prec), prec, e, rx1, n, rx2)
                  for e in np.eye(N)], axis=1)
    idx = np.arange(N).reshape(rx1, n, rx2, order="F")
    if prec == 1:
        groups = [idx[i, :, k] for i in range(rx1) for k in range(rx2)]
    elif prec == 2:
        groups = [idx[:, :, k].ravel(order="F") for k in range(rx2)]
    else:
        groups = [idx[i, :, :].ravel(order="F") for i in range(rx1)]
    for g in groups:  # P restricted to a block is the inverse of B's block
        np.testing.assert_allclose(P[np.ix_(g, g)] @ B[np.ix_(g, g)], np.eye(len(g)), atol=1e-10)
    mask = np.zeros((N, N), bool)
    for g in groups:
        mask[np.ix_(g, g)] = True
    assert not np.any(P[~mask])  # and zero elsewhere
    rhs = rng.standard_normal(N)
    x0 = np.zeros(N)
    xs = np.linalg.solve(B, rhs)
    for p in (0, prec):
        x = solve3d_2(Phi1, A, Phi2, rhs, 1e-12, x0, nrestart=N, niters=2, prec=p)
        assert np.linalg.norm(x - xs) <= 1e-9 * np.linalg.norm(xs)


@pytest.mark.parametrize("name", ["A", "b"])
def test_sdv_fixture_rebuilds_reference_bytes(name):
    """The oracle's SDV writer, fed the parsed contents of the reference's own
    fmex/{A,b}.sdv, reproduces the file byte for byte (SHA-256 pinned)."""
    from golden_io import load_sdv
    from oracle import sdv
    hd, g, data = load_sdv(name)
    f = sdv.parse(data)
    assert f["d"] == 80 and np.array_equal(f["core"], g["core"])


def test_amen_mv_oracle_reaches_exact_product():
    """oracle.amen_mv (core/amen_mv.m default path) at tight tolerance gives the
    exact TT matvec; at loose tolerance an error near tol."""
    from oracle.amen_mv import amen_mv
    A, _, _, _ = aniso_config(d=5, n=6)
    rng = np.random.default_rng(8)
    x = tt_randn(6, 5, 4, rng)
    ex = tt_matvec(A, x)
    y0 = tt_rand(6, 5, 2, np.random.default_rng(1))
    z0 = tt_rand(6, 5, 4, np.random.default_rng(2))
    y, z, info = amen_mv(A, x, 1e-12, y0, z0)
    assert tt_norm(y - ex) <= 1e-11 * tt_norm(ex)
    y, z, info = amen_mv(A, x, 1e-3, y0, z0)
    assert tt_norm(y - ex) <= 1e-2 * tt_norm(ex)
