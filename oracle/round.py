"""TT rounding oracle (FP64).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates ``@tt_tensor/round.m:20-108`` and ``core/my_chop2.m:18-35``:
a left-to-right QR sweep with the R-factor norms extracted, a right-to-left
truncated SVD sweep with the per-core threshold ``eps/sqrt(d-1) * ||s||``,
then the norm re-balancing ``exp(mean(log nrm))`` into every core.
"""
import numpy as np

from .tt import TT, rs


def my_chop2(sv, eps):
    """Smallest r with ``sqrt(sum(sv[r:]**2)) < eps`` (``core/my_chop2.m:18-35``)."""
    sv = np.asarray(sv, dtype=np.float64)
    if np.linalg.norm(sv) == 0:                       # my_chop2.m:18-21
        return 1
    if eps <= 0:                                      # my_chop2.m:23-26
        return sv.size
    sv0 = np.cumsum(sv[::-1] ** 2)                    # my_chop2.m:28
    ff = np.nonzero(sv0 < eps ** 2)[0]                # my_chop2.m:29
    if ff.size == 0:
        return sv.size
    return sv.size - (ff[-1] + 1)                     # my_chop2.m:33 (1-based ff(end))


def chop_margin(sv, eps):
    """How close ``my_chop2(sv, eps)`` is to a different answer: the smallest
    ``|tail/eps^2 - 1|`` of the two cumulative tail sums ``sum(sv[k:]**2)``
    on either side of the cut (the test ``sv0 < eps^2``, ``my_chop2.m:29``).
    ``inf`` when there is no decision (zero tensor, ``eps <= 0``)."""
    sv = np.asarray(sv, dtype=np.float64)
    if np.linalg.norm(sv) == 0 or eps <= 0:
        return np.inf
    sv0 = np.cumsum(sv[::-1] ** 2)
    below = np.nonzero(sv0 < eps ** 2)[0]
    k = below[-1] if below.size else -1       # last tail under the threshold
    cand = [k, k + 1]
    return min(abs(sv0[j] / eps ** 2 - 1.0) for j in cand if 0 <= j < sv0.size)


def tt_round(x, eps, rmax=None):
    """``round(tt, eps[, rmax])`` (``@tt_tensor/round.m:1-110``).

    Returns ``(y, info)`` where ``info`` holds the singular values seen at
    every step of the SVD sweep and the margin of every rank decision
    (``margins[i]``, ``chop_margin``) for rank/threshold parity checks.
    """
    d = x.d
    n = [int(v) for v in x.n]
    r = [int(v) for v in x.r]
    if rmax is None:                                  # round.m:20-22
        rmax = [np.iinfo(np.int64).max] * (d + 1)
    elif np.isscalar(rmax):                           # round.m:30-32
        rmax = [int(rmax)] * (d + 1)
    cores = [c.copy(order="F") for c in x.cores]
    nrm = np.zeros(d)
    # Left-to-right QR sweep (round.m:39-53).
    for i in range(d - 1):
        c0 = rs(cores[i], r[i] * n[i], r[i + 1])
        q, ru = np.linalg.qr(c0)                      # round.m:41 qr(core0,0)
        nrm[i + 1] = np.linalg.norm(ru)
        if nrm[i + 1] != 0:                           # round.m:42-44
            ru = ru / nrm[i + 1]
        c1 = rs(cores[i + 1], r[i + 1], n[i + 1] * r[i + 2])
        c1 = ru @ c1                                  # round.m:47
        r[i + 1] = q.shape[1]                         # round.m:48
        cores[i] = rs(q, r[i], n[i], r[i + 1])
        cores[i + 1] = rs(c1, r[i + 1], n[i + 1], r[i + 2])
    ep = eps / np.sqrt(d - 1) if d > 1 else eps       # round.m:56
    svals = [None] * (d + 1)
    margins = [None] * (d + 1)
    # Right-to-left SVD sweep (round.m:59-89).
    for i in range(d - 1, 0, -1):
        c0 = rs(cores[i], r[i], n[i] * r[i + 1])
        c1 = rs(cores[i - 1], r[i - 1] * n[i - 1], r[i])
        u, s, vt = np.linalg.svd(c0, full_matrices=False)   # round.m:65
        svals[i] = s.copy()
        margins[i] = chop_margin(s, np.linalg.norm(s) * ep)
        r1 = my_chop2(s, np.linalg.norm(s) * ep)      # round.m:77
        r1 = min(r1, rmax[i])                         # round.m:78
        u = u[:, :r1] * s[:r1]                        # round.m:80-81
        r[i] = r1
        c1 = c1 @ u                                   # round.m:83
        cores[i] = rs(vt[:r1, :], r[i], n[i], r[i + 1])     # round.m:84
        cores[i - 1] = rs(c1, r[i - 1], n[i - 1], r[i])
    # Norm balancing (round.m:94-107).
    nrm[0] = np.linalg.norm(cores[0])
    if nrm[0] != 0:
        cores[0] = cores[0] / nrm[0]
    with np.errstate(divide="ignore"):
        nrm0 = np.exp(np.sum(np.log(np.abs(nrm))) / d)
    cores = [c * nrm0 for c in cores]
    return TT(cores), {"svals": svals, "ranks": list(r), "margins": margins}
