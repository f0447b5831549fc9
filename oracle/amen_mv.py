"""AMEn approximate matrix-by-vector product -- FP64 oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates ``core/amen_mv.m:1-419`` on its default option path (tt_matrix
operator, ``renorm = 'direct'``, ``fkick = false``, ``kickrank2 = 0``,
``init_qr = true``): y ~ A x is kept as a TT whose every core is, in turn, the
projection of A x onto the interfaces of the other cores of y (the local
matvec ``bfun3`` with bra y and ket x), truncated by an SVD to
``tol ||s|| / sqrt(d)`` and, in the backward half-sweep, enriched by the
projected residual of a rank-``kickrank`` auxiliary TT z.  The helpers
``bfun3`` and ``compute_next_Phi`` are the ones of ``oracle.amen`` (the local
functions of ``amen_mv.m:421-621`` compute the same quantities).

MATLAB draws the initial ``y`` and ``z`` from its RNG (``:130-137``), which
cannot be reproduced here, so both are arguments.
"""
import numpy as np

from .amen import bfun3, compute_next_Phi
from .round import my_chop2
from .tt import TT, rs


def _qr(a):
    q, r = np.linalg.qr(a)
    return q, r


def amen_mv(A, x, tol, y0, z0=None, nswp=20, kickrank=4, init_qr=True):
    """``[y, z] = amen_mv(A, x, tol, 'y0', y0, 'z0', z0, ...)``; returns
    ``(y, z, info)`` with ``info['sweeps']`` and per-sweep ``max_dx``."""
    d = x.d
    n = [int(v) for v in A.n]
    Ac = A.cores
    xc = x.cores
    y = [np.asfortranarray(c.copy()) for c in y0.cores]
    ry = [int(v) for v in y0.r]
    use_z = kickrank > 0
    ones3 = np.ones((1, 1, 1), order="F")
    ones2 = np.ones((1, 1), order="F")
    if use_z:
        z = [np.asfortranarray(c.copy()) for c in z0.cores]
        rz = [int(v) for v in z0.r]
        phizax = [None] * (d + 1); phizax[0] = ones3; phizax[d] = ones3          # :142-147
        phizy = [None] * (d + 1); phizy[0] = ones2; phizy[d] = ones2
    phiyax = [None] * (d + 1); phiyax[0] = ones3; phiyax[d] = ones3              # :150-155
    nrms = np.ones(d)                                                            # :157
    for i in range(d - 1):                                                       # :160-214
        if init_qr:
            cr, R = _qr(rs(y[i], ry[i] * n[i], ry[i + 1]))
            nrmr = np.linalg.norm(R)
            if nrmr > 0:
                R = R / nrmr
            cr2 = R @ rs(y[i + 1], ry[i + 1], n[i + 1] * ry[i + 2])
            ry[i + 1] = cr.shape[1]
            y[i] = rs(cr, ry[i], n[i], ry[i + 1])
            y[i + 1] = rs(cr2, ry[i + 1], n[i + 1], ry[i + 2])
        phiyax[i + 1], nrms[i] = compute_next_Phi(phiyax[i], y[i], Ac[i], xc[i], "lr",
                                                  want_norm=True)
        if use_z:
            cr, R = _qr(rs(z[i], rz[i] * n[i], rz[i + 1]))
            nrmr = np.linalg.norm(R)
            if nrmr > 0:
                R = R / nrmr
            cr2 = R @ rs(z[i + 1], rz[i + 1], n[i + 1] * rz[i + 2])
            rz[i + 1] = cr.shape[1]
            z[i] = rs(cr, rz[i], n[i], rz[i + 1])
            z[i + 1] = rs(cr2, rz[i + 1], n[i + 1], rz[i + 2])
            phizax[i + 1], _ = compute_next_Phi(phizax[i], z[i], Ac[i], xc[i], "lr",
                                                extnrm=nrms[i])
            phizy[i + 1], _ = compute_next_Phi(phizy[i], z[i], None, y[i], "lr")

    i = d - 1                                                                    # :216-219
    direction = -1
    swp = 1
    max_dx = 0.0
    info = dict(max_dx=[], sweeps=0)
    cry = None
    while swp <= nswp:                                                           # :221
        crx = rs(xc[i], xc[i].size)
        cry = bfun3(phiyax[i], Ac[i], phiyax[i + 1], crx)                        # :224
        nrms[i] = np.linalg.norm(cry)                                            # :225
        if nrms[i] > 0:
            cry = cry / nrms[i]
        else:
            nrms[i] = 1.0
        dx = np.linalg.norm(cry - rs(y[i], y[i].size))                           # :232-233
        max_dx = max(max_dx, dx)
        if direction > 0 and i < d - 1:                                          # :237
            cry = rs(cry, ry[i] * n[i], ry[i + 1])
            u, s, vh = np.linalg.svd(cry, full_matrices=False)                   # :244
            r = my_chop2(s, tol * np.linalg.norm(s) / np.sqrt(d))                # :246
            u = u[:, :r]
            v = vh[:r].T * s[:r]                                                 # :248
            if use_z:
                cry = u @ v.T                                                    # :253
                crz = bfun3(phizax[i], Ac[i], phizax[i + 1], crx)                # :256
                crz = rs(crz, rz[i] * n[i], rz[i + 1])
                ys = cry @ phizy[i + 1]                                          # :258
                yz = rs(ys, ry[i], n[i] * rz[i + 1])
                yz = phizy[i] @ yz
                yz = rs(yz, rz[i] * n[i], rz[i + 1])
                crz = crz / nrms[i] - yz                                         # :262
            y[i] = rs(u, ry[i], n[i], r)                                         # :287
            cr2 = rs(v, ry[i + 1], r).T @ rs(y[i + 1], ry[i + 1], n[i + 1] * ry[i + 2])
            y[i + 1] = rs(cr2, r, n[i + 1], ry[i + 2])                           # :292
            ry[i + 1] = r
            phiyax[i + 1], nrms[i] = compute_next_Phi(phiyax[i], y[i], Ac[i], xc[i], "lr",
                                                      want_norm=True)            # :296
            if use_z:
                crz, _ = _qr(crz)                                                # :302
                rz[i + 1] = crz.shape[1]
                z[i] = rs(crz, rz[i], n[i], rz[i + 1])
                phizax[i + 1], _ = compute_next_Phi(phizax[i], z[i], Ac[i], xc[i], "lr",
                                                    extnrm=nrms[i])
                phizy[i + 1], _ = compute_next_Phi(phizy[i], z[i], None, y[i], "lr")
        elif direction < 0 and i > 0:                                            # :311
            cry = rs(cry, ry[i], n[i] * ry[i + 1])
            u, s, vh = np.linalg.svd(cry, full_matrices=False)                   # :318
            r = my_chop2(s, tol * np.linalg.norm(s) / np.sqrt(d))
            v = vh[:r].T                                                         # :321
            u = u[:, :r] * s[:r]
            if use_z:
                cry = u @ v.T                                                    # :327
                crz = bfun3(phizax[i], Ac[i], phizax[i + 1], crx)
                crz = rs(crz, rz[i], n[i] * rz[i + 1])
                ys = phizy[i] @ cry                                              # :332
                yz = rs(ys, rz[i] * n[i], ry[i + 1])
                yz = yz @ phizy[i + 1]
                yz = rs(yz, rz[i], n[i] * rz[i + 1])
                crz = crz / nrms[i] - yz                                         # :336
                crs = bfun3(phizax[i], Ac[i], phiyax[i + 1], crx)                # :344
                crs = rs(crs, rz[i], n[i] * ry[i + 1])
                crs = crs / nrms[i] - ys
                v = np.hstack([v, crs.T])                                        # :347
                v, R = _qr(v)                                                    # :351
                u = np.hstack([u, np.zeros((ry[i], rz[i]))]) @ R.T               # :353-354
                r = v.shape[1]
            cr2 = rs(y[i - 1], ry[i - 1] * n[i - 1], ry[i]) @ u                  # :357-358
            y[i - 1] = rs(cr2, ry[i - 1], n[i - 1], r)
            y[i] = rs(np.ascontiguousarray(v.T), r, n[i], ry[i + 1])
            ry[i] = r
            phiyax[i], nrms[i] = compute_next_Phi(phiyax[i + 1], y[i], Ac[i], xc[i], "rl",
                                                  want_norm=True)                # :364
            if use_z:
                crz, _ = _qr(crz.T)                                              # :370
                rz[i] = crz.shape[1]
                z[i] = rs(np.ascontiguousarray(crz.T), rz[i], n[i], rz[i + 1])
                phizax[i], _ = compute_next_Phi(phizax[i + 1], z[i], Ac[i], xc[i], "rl",
                                                extnrm=nrms[i])
                phizy[i], _ = compute_next_Phi(phizy[i + 1], z[i], None, y[i], "rl")
        if (direction > 0 and i == d - 1) or (direction < 0 and i == 0):         # :387
            if direction > 0:
                info["max_dx"].append(max_dx)
                info["sweeps"] = swp
            if (max_dx < tol or swp == nswp) and direction > 0:
                break
            y[i] = rs(cry, ry[i], n[i], ry[i + 1])                               # :396
            if direction > 0:
                swp += 1
            max_dx = 0.0
            direction = -direction
        else:
            i += direction
    y[d - 1] = rs(cry, ry[d - 1], n[d - 1], ry[d])                               # :408
    nrm = np.exp(np.sum(np.log(nrms)) / d)                                       # :414
    y = [np.asfortranarray(c * nrm) for c in y]
    return TT(y), (TT(z) if use_z else None), info
