"""ALS(t+z) linear-solver oracle (FP64).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates ``solve/alstpz_solve.m`` on its default option path (kicktype
``'svd'``: the residual ``y - A x`` rounded to rank ``kickrank``; the MEX
local solver ``solve3d_2``; no symmetrisation):

* ``alstpz_solve`` -- ``solve/alstpz_solve.m:1-215``: each of ``nswp`` sweeps
  rounds x to ``tol`` (:140), rounds the exact residual to rank ``kickrank``
  (:189-195), appends it to x with weight zero (:199-201) and runs one ALS
  sweep (:204-208).  There is no convergence test: every sweep runs.
* ``als_sweep``   -- ``als_solve``, ``solve/alstpz_solve.m:217-428``:
  right-to-left QR orthogonalisation with interfaces (:286-299), then one
  left-to-right pass of local solves (dense below ``max_full_size``,
  :316-336; else ``solve3d_2``, :338-362), each solution split by QR into the
  next core (:380-407).

The local kernels (``bfun3``, ``compute_next_Phi``, ``solve3d_2``, the dense
local matrix) are those of ``oracle/amen.py``: ``alstpz_solve.m`` carries its
own copies of ``compute_next_Phi`` (:429-500) and ``bfun3`` (:502-530) with
the same contractions.  The interfaces are not normalised here (the
reference calls ``compute_next_Phi`` with one output).
"""
import numpy as np

from .amen import assemble_local, bfun3, compute_next_Phi, solve3d_2
from .round import tt_round
from .tt import TT, rs, tt_matvec, tt_plus

DEFAULTS = dict(nswp=10, max_full_size=50, local_restart=40, local_iters=2, kickrank=4,
                resid_damp=2.0, local_prec=0)


def als_sweep(A, y, tol, x, max_full_size=50, local_restart=40, local_iters=2, resid_damp=2.0,
              local_prec=0):
    """One ALS sweep (``als_solve``, ``solve/alstpz_solve.m:217-428``).

    Returns ``(x, info)`` with ``info = {max_res, max_dx, res_prev: [..]}``."""
    d = y.d
    n = [int(v) for v in A.n]
    crx = [c.copy(order="F") for c in x.cores]
    rx = [int(v) for v in x.r]
    ry = [int(v) for v in y.r]
    cry = y.cores
    crA = A.cores
    ones3 = np.ones((1, 1, 1), order="F")
    ones2 = np.ones((1, 1), order="F")
    phia = [None] * (d + 1); phia[0] = ones3; phia[d] = ones3          # :270
    phiy = [None] * (d + 1); phiy[0] = ones2; phiy[d] = ones2          # :271
    for i in range(d - 1, 0, -1):                                       # :286-299
        cr = rs(crx[i], rx[i], n[i] * rx[i + 1])
        q, rv = np.linalg.qr(cr.T)                                      # :288
        cr2 = rs(crx[i - 1], rx[i - 1] * n[i - 1], rx[i]) @ rv.T        # :289-291
        rx[i] = q.shape[1]                                              # :292
        crx[i] = rs(q.T, rx[i], n[i], rx[i + 1])                        # :293
        crx[i - 1] = rs(cr2, rx[i - 1], n[i - 1], rx[i])                # :294
        phia[i] = compute_next_Phi(phia[i + 1], crx[i], crA[i], crx[i], "rl")[0]   # :297
        phiy[i] = compute_next_Phi(phiy[i + 1], crx[i], None, cry[i], "rl")[0]     # :298
    info = dict(max_res=0.0, max_dx=0.0, res_prev=[], ranks=None)
    real_tol = (tol / np.sqrt(d)) / resid_damp                          # :318
    for i in range(d):                                                  # :305
        Phi1, Phi2 = phia[i], phia[i + 1]
        A1 = crA[i]
        rhs = phiy[i] @ rs(cry[i], ry[i], n[i] * ry[i + 1])             # :311-313
        rhs = rs(rhs, rx[i] * n[i], ry[i + 1]) @ phiy[i + 1]            # :314-315
        rhs = rhs.ravel(order="F")
        norm_rhs = np.linalg.norm(rhs)                                  # :317
        sol_prev = crx[i].ravel(order="F")                              # :319
        N = rx[i] * n[i] * rx[i + 1]
        if N < max_full_size:                                           # :321-336
            B = assemble_local(Phi1, A1, Phi2)
            res_prev = np.linalg.norm(B @ sol_prev - rhs) / norm_rhs
            if res_prev > real_tol:
                sol = np.linalg.solve(B, rhs)
            else:
                sol = sol_prev
        else:                                                           # :338-362
            res_prev = np.linalg.norm(bfun3(Phi1, A1, Phi2, sol_prev) - rhs) / norm_rhs
            if res_prev > real_tol:
                sol = solve3d_2(Phi1, A1, Phi2, rhs, real_tol, sol_prev, local_restart,
                                local_iters, prec=local_prec)
            else:
                sol = sol_prev
        nsol = np.linalg.norm(sol)
        dx = np.linalg.norm(sol - sol_prev) / nsol if nsol > 0 else 0.0     # :371
        info["max_dx"] = max(info["max_dx"], dx)                        # :372
        info["max_res"] = max(info["max_res"], res_prev)                # :373
        info["res_prev"].append(res_prev)
        sol = rs(sol, rx[i] * n[i], rx[i + 1])
        if i < d - 1:                                                   # :387-402
            u, v = np.linalg.qr(sol)                                    # :380
            r = u.shape[1]
            v = v @ rs(crx[i + 1], rx[i + 1], n[i + 1] * rx[i + 2])     # :390
            crx[i] = rs(u, rx[i], n[i], r)
            crx[i + 1] = rs(v, r, n[i + 1], rx[i + 2])
            rx[i + 1] = r
            phia[i + 1] = compute_next_Phi(phia[i], crx[i], crA[i], crx[i], "lr")[0]   # :396
            phiy[i + 1] = compute_next_Phi(phiy[i], crx[i], None, cry[i], "lr")[0]     # :397
        else:
            crx[i] = rs(sol, rx[i], n[i], rx[i + 1])                    # :405
    x = TT(crx)
    info["ranks"] = [int(v) for v in x.r]
    return x, info


def alstpz_solve(A, y, tol, x0, **opts):
    """``[x, testdata] = alstpz_solve(A, y, tol, ...)`` with kicktype 'svd'.

    ``x0`` is required (the reference draws ``tt_rand(n, d, 2)``, :117, from
    MATLAB's RNG).  Returns ``(x, info)`` with per-sweep ``max_res`` and
    ``max_dx`` of the ALS sweeps and the ranks after each sweep."""
    o = dict(DEFAULTS)
    for k, v in opts.items():
        if k not in o:
            raise ValueError("Unrecognized option: %s" % k)
        o[k] = v
    if np.any(A.n != A.m):
        raise ValueError("alstpz_solve needs a square operator")
    x = x0.copy()
    info = dict(max_res=[], max_dx=[], ranks=[], sweeps=0)
    kickrank = o["kickrank"]
    for _ in range(o["nswp"]):                                          # :138
        x, _ = tt_round(x, tol)                                         # :140
        if kickrank > 0:
            zz = tt_plus(y, tt_matvec(A, x) * (-1.0))                   # :193 y - A*x
            z, _ = tt_round(zz, tol, kickrank)
            x = tt_plus(x, z * 0.0)                                     # :199-201 x + 0*z
        x, si = als_sweep(A, y, tol, x, o["max_full_size"], o["local_restart"],
                          o["local_iters"], o["resid_damp"], o["local_prec"])
        info["max_res"].append(si["max_res"])
        info["max_dx"].append(si["max_dx"])
        info["ranks"].append(si["ranks"])
        info["sweeps"] += 1
    return x, info
