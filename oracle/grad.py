"""Gradients of TT functionals with respect to every core -- FP64 oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

TT-Toolbox has no derivative code, so there is nothing of the reference to
restate here beyond the forward maps it defines:

* ``<x, A x>``: ``@tt_matrix/mtimes.m:38-65`` (TT matrix times TT tensor)
  followed by ``@tt_tensor/dot.m:92-111`` (left-to-right sweep of interface
  matrices);
* ``<x, b>``: ``@tt_tensor/dot.m:92-111``;
* an entry ``X[i_1, ..., i_d]``: ``@tt_tensor/subsref.m:93-123`` (the product
  of the core slices ``x_k(:, i_k, :)``).

Each functional is multilinear in the cores; the gradient with respect to
core k is the functional with that core taken out, i.e. the left and right
interface sweeps contracted with what touched core k.  This module computes
those sweeps with ``numpy.einsum`` in its own index convention (bra rank,
operator rank, ket rank), independent of the CUDA library's layouts.
``full_*`` evaluate the functionals on the full tensor for tiny cases and
anchor the sweeps (and finite differences) in the tests.

Parity unpinned by the reference: there is no reference gradient.
"""
import numpy as np


def _e(spec, a, b):
    """Pairwise contraction through BLAS (numpy.einsum with a tensordot path)."""
    return np.einsum(spec, a, b, optimize=True)


def xAx(xc, Ac):
    """``(f, [G_k])`` for ``f = <x, A x>``; ``xc`` cores ``[r, n, r']``,
    ``Ac`` cores ``[ra, n, n, ra']`` (row index first, as ``tt_matrix``).
    Interfaces ``L[a, A, b]`` / ``R[c, B, e]``: bra rank, operator rank,
    ket rank."""
    d = len(xc)
    L = [np.ones((1, 1, 1))]
    for k in range(d):
        t = _e("aAb,aic->Abic", L[k], xc[k])
        t = _e("Abic,AijB->bjcB", t, Ac[k])
        L.append(_e("bjcB,bje->cBe", t, xc[k]))
    R = [None] * (d + 1)
    R[d] = np.ones((1, 1, 1))
    for k in range(d - 1, -1, -1):
        t = _e("cBe,bje->cBbj", R[k + 1], xc[k])
        t = _e("cBbj,AijB->cAib", t, Ac[k])
        R[k] = _e("cAib,aic->aAb", t, xc[k])
    G = []
    for k in range(d):
        t = _e("aAb,bje->aAje", L[k], xc[k])
        t = _e("aAje,AijB->aiBe", t, Ac[k])
        gb = _e("aiBe,cBe->aic", t, R[k + 1])  # through the bra copy of x_k
        t = _e("aAb,aic->Abic", L[k], xc[k])
        t = _e("Abic,AijB->bcjB", t, Ac[k])
        gk = _e("bcjB,cBe->bje", t, R[k + 1])  # through the ket copy
        G.append(gb + gk)
    return float(L[d][0, 0, 0]), G


def xb(xc, bc):
    """``(f, [G_k])`` for ``f = <x, b>``; interfaces ``[x rank, b rank]``."""
    d = len(xc)
    PL = [np.ones((1, 1))]
    for k in range(d):
        PL.append(_e("aiq,aic->cq", _e("ap,piq->aiq", PL[k], bc[k]), xc[k]))
    PR = [None] * (d + 1)
    PR[d] = np.ones((1, 1))
    for k in range(d - 1, -1, -1):
        PR[k] = _e("pic,aic->ap", _e("cq,piq->pic", PR[k + 1], bc[k]), xc[k])
    G = [_e("aiq,cq->aic", _e("ap,piq->aiq", PL[k], bc[k]), PR[k + 1]) for k in range(d)]
    return float(PL[d][0, 0]), G


def _buckets(col, n):
    """Sample positions grouped by index value: (order, start) with the
    samples of value j at order[start[j]:start[j+1]]."""
    order = np.argsort(col, kind="stable")
    start = np.zeros(n + 1, dtype=np.int64)
    start[1:] = np.cumsum(np.bincount(col, minlength=n))
    return order, start


def entries(xc, idx):
    """``X[idx[s]]`` for every row of ``idx`` ([S, d], 0-based)."""
    S = idx.shape[0]
    v = np.ones((S, 1))
    for k, core in enumerate(xc):
        out = np.empty((S, core.shape[2]))
        order, start = _buckets(idx[:, k], core.shape[1])
        for j in range(core.shape[1]):
            sel = order[start[j]:start[j + 1]]
            out[sel] = v[sel] @ core[:, j, :]
        v = out
    return v[:, 0]


def sampled(xc, idx, y):
    """``(f, [G_k])`` for ``f = sum_s (X[idx[s]] - y[s])^2``.

    Left row vectors ``l_k(s)`` (product of the slices left of k) and right
    column vectors ``rho_k(s) = 2 e_s * (product of the slices right of k)``;
    ``G_k[:, j, :] = sum_{s: i_k(s) = j} l_k(s)^T rho_k(s)^T``."""
    d = len(xc)
    S = idx.shape[0]
    groups = [_buckets(idx[:, k], xc[k].shape[1]) for k in range(d)]
    left = [np.ones((S, 1))]
    for k in range(d):
        core = xc[k]
        out = np.empty((S, core.shape[2]))
        order, start = groups[k]
        for j in range(core.shape[1]):
            sel = order[start[j]:start[j + 1]]
            out[sel] = left[k][sel] @ core[:, j, :]
        left.append(out)
    e = left[d][:, 0] - y
    rho = (2.0 * e)[:, None]
    G = [None] * d
    for k in range(d - 1, -1, -1):
        core = xc[k]
        order, start = groups[k]
        g = np.zeros(core.shape)
        nxt = np.empty((S, core.shape[0]))
        for j in range(core.shape[1]):
            sel = order[start[j]:start[j + 1]]
            g[:, j, :] = left[k][sel].T @ rho[sel]
            nxt[sel] = rho[sel] @ core[:, j, :].T
        G[k] = g
        rho = nxt
    return float(e @ e), G


# ---- full-tensor forms (tiny cases only) ---------------------------------

def full_tensor(xc):
    """Full tensor with C-order axes (i_1, ..., i_d)."""
    t = np.ones((1, 1))
    for core in xc:
        t = np.einsum("pa,aic->pic", t, core).reshape(-1, core.shape[2])
    return t[:, 0].reshape([c.shape[1] for c in xc])


def full_matrix(Ac):
    """Full operator as an (N x N) matrix in the C-order flattening of full_tensor."""
    t = np.ones((1, 1, 1))  # (rows, cols, rank)
    for core in Ac:
        ra1, n, m, ra2 = core.shape
        t = np.einsum("xya,aijb->xiyjb", t, core).reshape(t.shape[0] * n, t.shape[1] * m, ra2)
    return t[:, :, 0]


def full_xAx(xc, Ac):
    v = full_tensor(xc).ravel()
    return float(v @ (full_matrix(Ac) @ v))


def full_xb(xc, bc):
    return float(full_tensor(xc).ravel() @ full_tensor(bc).ravel())


def full_sampled(xc, idx, y):
    X = full_tensor(xc)
    e = X[tuple(idx.T)] - y
    return float(e @ e)
