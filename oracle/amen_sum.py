"""AMEn approximation of linear combinations of TT tensors -- FP64 oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates ``core/amen_sum.m:1-483`` on its default option path for TT
inputs (``can = false``, ``renorm = 'direct'``, ``fkick = false``,
``kickrank2 = 0``, ``multrank = false``): ``y(:, m) ~ sum_j X{j} c(j, m)``
for ``m = 1..M`` is kept as one TT whose current core carries the extra
index ``m``; every core is, in turn, the projection of the sum onto the
interfaces of the other cores of ``y`` (``proj_sum``, ``:647-684``),
truncated by an SVD to ``tol ||s|| / sqrt(d)`` and, in the backward
half-sweep, enriched by the projected residual of a rank-``kickrank``
auxiliary TT ``z``.  The result is a TT whose last rank is ``M``.

MATLAB draws the initial ``y`` and ``z`` from its RNG, which
cannot be reproduced here (``:152-187``, ``gen_rand`` ``:633-644``), so both
are arguments.
"""
import numpy as np

from .round import my_chop2
from .tt import TT, rs


def _phi_lr(prev, ycore, xcores, want_norm=False, extnrm=None):
    """``compute_next_Phi(..., 'lr')`` (``amen_sum.m:557-594``), one interface
    per summand: ``Phi_j[b, beta] = sum y[a,k,b] prev_j[a,alpha] X_j[alpha,k,beta]``."""
    out = [np.einsum("akb,al,lkm->bm", ycore, p, x) for p, x in zip(prev, xcores)]
    return _scale(out, want_norm, extnrm)


def _phi_rl(prev, ycore, xcores, want_norm=False, extnrm=None):
    """``compute_next_Phi(..., 'rl')`` (``amen_sum.m:595-627``):
    ``Phi_j[alpha, a] = sum X_j[alpha,k,beta] prev_j[beta,b] y[a,k,b]``."""
    out = [np.einsum("lkm,mb,akb->la", x, p, ycore) for p, x in zip(prev, xcores)]
    return _scale(out, want_norm, extnrm)


def _scale(phis, want_norm, extnrm):
    """The largest Frobenius norm is taken out when asked for
    (``:580-588``), else an external norm divides (``:589-593``)."""
    if want_norm:
        nrm = max(np.linalg.norm(p) for p in phis)
        if nrm > 0:
            phis = [p / nrm for p in phis]
        else:
            nrm = 1.0
        return phis, nrm
    if extnrm is not None:
        phis = [p / extnrm for p in phis]
    return phis


def _proj_sum(phi1, xcores, phi2, c):
    """``proj_sum`` (``amen_sum.m:647-684``, TT branch): the local core of
    ``sum_j X_j c(j, :)``, shape ``(ry1 n ry2, M)``."""
    out = 0.0
    for j, (p1, x, p2) in enumerate(zip(phi1, xcores, phi2)):
        t = np.einsum("al,lkm,mb->akb", p1, x, p2)
        out = out + np.outer(rs(t, t.size), c[j])
    return out


def _qr_normalized(core, r1, n, r2, nxt, rn2):
    """Initial orthogonalisation step (``amen_sum.m:196-209``)."""
    q, R = np.linalg.qr(rs(core, r1 * n, r2))
    nrm = np.linalg.norm(R)
    if nrm > 0:
        R = R / nrm
    return q, R @ rs(nxt, r2, rn2)


def amen_sum(X, c, tol, y0, z0=None, nswp=20, kickrank=4, init_qr=True, rmax=np.inf):
    """``[y, z] = amen_sum(X, c, tol, 'y0', y0, 'z0', z0, ...)`` for a list of
    TT tensors ``X`` of equal mode sizes and coefficients ``c`` (``N x M``);
    returns ``(y, z, info)`` with ``y`` of last rank ``M``."""
    c = np.asarray(c, dtype=np.float64)
    if c.ndim == 1:
        c = c[:, None]
    N, M = c.shape
    assert len(X) == N
    d = X[0].d
    n = [int(v) for v in X[0].n]
    Xc = [[X[j].cores[i] for j in range(N)] for i in range(d)]
    y = [np.asfortranarray(cr.copy()) for cr in y0.cores]
    ry = [int(v) for v in y0.r]
    kick = kickrank > 0
    one = np.ones((1, 1))
    phiyx = [None] * (d + 1)
    phiyx[0] = [one] * N
    phiyx[d] = [one] * N
    if kick:
        z = [np.asfortranarray(cr.copy()) for cr in z0.cores]
        rz = [int(v) for v in z0.r]
        phizx = [None] * (d + 1)
        phizx[0] = [one] * N
        phizx[d] = [one] * N
        phizy = [None] * (d + 1)
        phizy[0] = one
        phizy[d] = one
    nrms = np.ones(d)
    for i in range(d - 1):                                                       # :194-241
        if init_qr:
            q, cr2 = _qr_normalized(y[i], ry[i], n[i], ry[i + 1], y[i + 1], n[i + 1] * ry[i + 2])
            ry[i + 1] = q.shape[1]
            y[i] = rs(q, ry[i], n[i], ry[i + 1])
            y[i + 1] = rs(cr2, ry[i + 1], n[i + 1], ry[i + 2])
        phiyx[i + 1], nrms[i] = _phi_lr(phiyx[i], y[i], Xc[i], want_norm=True)
        if kick:
            q, cr2 = _qr_normalized(z[i], rz[i], n[i], rz[i + 1], z[i + 1], n[i + 1] * rz[i + 2])
            rz[i + 1] = q.shape[1]
            z[i] = rs(q, rz[i], n[i], rz[i + 1])
            z[i + 1] = rs(cr2, rz[i + 1], n[i + 1], rz[i + 2])
            phizx[i + 1] = _phi_lr(phizx[i], z[i], Xc[i], extnrm=nrms[i])
            phizy[i + 1] = _phi_lr([phizy[i]], z[i], [y[i]])[0]

    # The last core carries the output index (:247-251).
    last = rs(y[d - 1], ry[d - 1] * n[d - 1], ry[d])
    padded = np.zeros((ry[d - 1] * n[d - 1], M))
    k = min(ry[d], M)
    padded[:, :k] = last[:, :k]
    y[d - 1] = rs(padded, ry[d - 1], n[d - 1], 1, M)
    ry[d] = 1

    i, direction, swp, max_dx = d - 1, -1, 1, 0.0
    info = dict(max_dx=[], sweeps=0)
    cry = None
    while swp <= nswp:                                                           # :253
        cry = _proj_sum(phiyx[i], Xc[i], phiyx[i + 1], c)                        # :255
        nrms[i] = np.linalg.norm(cry)
        if nrms[i] > 0:
            cry = cry / nrms[i]
        else:
            nrms[i] = 1.0
        yi = rs(y[i], ry[i] * n[i] * ry[i + 1], M)                              # :265-268
        dx = np.linalg.norm(cry - yi) / np.linalg.norm(cry)
        max_dx = max(max_dx, dx)
        ni = n[i]
        if direction > 0 and i < d - 1:                                          # :271
            u, s, vh = np.linalg.svd(rs(cry, ry[i] * ni, ry[i + 1] * M), full_matrices=False)
            r = min(my_chop2(s, tol * np.linalg.norm(s) / np.sqrt(d)), rmax)    # :288-289
            u = u[:, :r]
            v = vh[:r].T * s[:r]                                                 # :291
            if kick:                                                             # :301-327
                cry2 = rs(u @ v.T, ry[i] * ni * ry[i + 1], M)
                crys = rs(cry2.T, M * ry[i] * ni, ry[i + 1]) @ phizy[i + 1]
                crys = rs(crys, M, ry[i] * ni * rz[i + 1]).T
                cryz = phizy[i] @ rs(crys, ry[i], ni * rz[i + 1] * M)
                cryz = rs(cryz, rz[i] * ni * rz[i + 1], M)
                crz = _proj_sum(phizx[i], Xc[i], phizx[i + 1], c) / nrms[i] - cryz
                uz = np.linalg.svd(rs(crz, rz[i] * ni, rz[i + 1] * M), full_matrices=False)[0]
                crz = uz[:, :min(uz.shape[1], kickrank)]
            y[i] = rs(u, ry[i], ni, r)                                           # :342
            cr2 = rs(v, ry[i + 1], M * r).T @ rs(y[i + 1], ry[i + 1], n[i + 1] * ry[i + 2])
            cr2 = rs(cr2, M, r * n[i + 1] * ry[i + 2]).T                         # :344-348
            y[i + 1] = rs(cr2, r, n[i + 1], ry[i + 2], M)
            ry[i + 1] = r
            phiyx[i + 1], nrms[i] = _phi_lr(phiyx[i], y[i], Xc[i], want_norm=True)   # :352
            if kick:                                                             # :354-360
                rz[i + 1] = crz.shape[1]
                z[i] = rs(crz, rz[i], ni, rz[i + 1])
                phizx[i + 1] = _phi_lr(phizx[i], z[i], Xc[i], extnrm=nrms[i])
                phizy[i + 1] = _phi_lr([phizy[i]], z[i], [y[i]])[0]
        elif direction < 0 and i > 0:                                            # :361
            u, s, vh = np.linalg.svd(rs(cry.T, M * ry[i], ni * ry[i + 1]), full_matrices=False)
            r = min(my_chop2(s, tol * np.linalg.norm(s) / np.sqrt(d)), rmax)    # :369-370
            u = u[:, :r] * s[:r]
            v = vh[:r].T
            if kick:                                                             # :382-420
                cry2 = rs(u @ v.T, M, ry[i] * ni * ry[i + 1])
                crys = phizy[i] @ rs(cry2.T, ry[i], ni * ry[i + 1] * M)
                crys = rs(crys, rz[i] * ni * ry[i + 1], M)
                cryz = rs(crys.T, M * rz[i] * ni, ry[i + 1]) @ phizy[i + 1]
                cryz = rs(cryz, M, rz[i] * ni * rz[i + 1]).T
                crz = _proj_sum(phizx[i], Xc[i], phizx[i + 1], c) / nrms[i] - cryz
                vz = np.linalg.svd(rs(crz.T, M * rz[i], ni * rz[i + 1]), full_matrices=False)[2]
                crz = vz[:min(vz.shape[0], kickrank)]                           # (kz, n rz)
                crs = _proj_sum(phizx[i], Xc[i], phiyx[i + 1], c) / nrms[i] - crys
                vs = np.linalg.svd(rs(crs.T, M * rz[i], ni * ry[i + 1]), full_matrices=False)[2]
                crs = vs[:min(vs.shape[0], kickrank)].T
                v, R = np.linalg.qr(np.hstack([v, crs]))                         # :412-418
                u = np.hstack([u, np.zeros((M * ry[i], crs.shape[1]))]) @ R.T
                r = v.shape[1]
            y[i] = rs(np.ascontiguousarray(v.T), r, ni, ry[i + 1])               # :421
            uu = rs(rs(u, M, ry[i] * r).T, ry[i], r * M)                         # :423-429
            cr2 = rs(y[i - 1], ry[i - 1] * n[i - 1], ry[i]) @ uu
            y[i - 1] = rs(cr2, ry[i - 1], n[i - 1], r, M)
            ry[i] = r
            phiyx[i], nrms[i] = _phi_rl(phiyx[i + 1], y[i], Xc[i], want_norm=True)   # :433
            if kick:                                                             # :435-441
                rz[i] = crz.shape[0]
                z[i] = rs(crz, rz[i], ni, rz[i + 1])
                phizx[i] = _phi_rl(phizx[i + 1], z[i], Xc[i], extnrm=nrms[i])
                phizy[i] = _phi_rl([phizy[i + 1]], z[i], [y[i]])[0]
        else:
            y[i] = rs(y[i], ry[i], ni, ry[i + 1], M)                             # :443
        if (direction > 0 and i == d - 1) or (direction < 0 and i == 0):        # :451-463
            if direction > 0:
                info["max_dx"].append(max_dx)
                info["sweeps"] = swp
            if (max_dx < tol or swp == nswp) and direction > 0:
                break
            max_dx = 0.0
            if direction > 0:
                swp += 1
            direction = -direction
        else:
            i += direction
    y[d - 1] = rs(cry, ry[d - 1], n[d - 1], M)                                   # :466
    nrm = np.exp(np.sum(np.log(nrms)) / d)                                       # :469-473
    y = TT([cr * nrm for cr in y])
    return y, (TT(z) if kick else None), info
