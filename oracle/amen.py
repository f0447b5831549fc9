"""AMEn linear-solver oracle (FP64).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates, on the default option path of ``solve/amen_solve2.m``
(kicktype ``'als'``, trunc_norm ``'residual'``, the MEX local solver
``solve3d_2``, with or without the block-Jacobi local preconditioners):

* ``bfun3``            -- ``solve/amen_solve2.m:924-951``
* ``compute_next_Phi`` -- ``solve/amen_solve2.m:834-920``
* ``dgmresr_hh``       -- ``fmex/solve3d.c:339-518`` (Householder Arnoldi +
  Givens; the readable twin of the tt-fort routine that ``fmex/solve3d_2.c:267``
  calls; tt-fort itself is an un-vendored submodule, pinned version unknown)
* ``solve3d_2``        -- ``fmex/solve3d_2.c:121-300`` (residual branch)
* ``amen_solve2``      -- ``solve/amen_solve2.m:67-831``

Array layouts are the reference's (column-major): ``Phi1 [ry1, rx1, ra1]``,
``A [ra1, n, m, ra2]``, ``Phi2 [rx2, ra2, ry2]``, ``x [rx1, m, rx2]``.
"""
import numpy as np

from .tt import TT, TTMatrix, rs


# ---------------------------------------------------------------------------
# Local kernels
# ---------------------------------------------------------------------------

def bfun3(Phi1, A, Phi2, x):
    """Local matvec ``y = (Phi1 x A x Phi2) x`` (``amen_solve2.m:924-951``)."""
    ry1, rx1, ra1 = Phi1.shape[0], Phi1.shape[1], (Phi1.shape[2] if Phi1.ndim > 2 else 1)
    rx2, ra2, ry2 = Phi2.shape[0], (Phi2.shape[1] if Phi2.ndim > 1 else 1), (Phi2.shape[2] if Phi2.ndim > 2 else 1)
    n, m = A.shape[1], A.shape[2]
    y = rs(x, rx1 * m, rx2)                                   # :937
    y = y @ rs(Phi2, rx2, ra2 * ry2)                          # :938-939
    y = rs(y, rx1, m * ra2 * ry2).T                           # :940-941
    y = rs(y, m * ra2, ry2 * rx1)                             # :942
    y = rs(A, ra1 * n, m * ra2) @ y                           # :943-944
    y = rs(y, ra1 * n * ry2, rx1).T                           # :945-946
    y = rs(y, rx1 * ra1, n * ry2)                             # :947
    y = rs(Phi1, ry1, rx1 * ra1) @ y                          # :948-949
    return rs(y, ry1 * n * ry2)                               # :950


def compute_next_Phi(Phi_prev, x, A, y, direction, extnrm=None, want_norm=False):
    """Interface update (``amen_solve2.m:834-920``).

    ``'lr'``: ``Phi_prev [rx1, ry1, ra1]`` -> ``[rx2, ry2, ra2]``;
    ``'rl'``: ``Phi_prev [ry2, ra2, rx2]`` -> ``[ry1, ra1, rx1]``.
    ``A is None`` gives the X'Y variant (no ``ra`` index).
    Returns ``(Phi, nrm)``; ``nrm`` is the Frobenius norm divided out when
    ``want_norm`` (``:907-914``), otherwise ``extnrm`` divides (``:915-918``).
    """
    rx1, n, rx2 = x.shape
    ry1, m, ry2 = y.shape
    if A is not None:
        ra1, ra2 = A.shape[0], A.shape[3]
    else:
        ra1 = ra2 = 1
    if direction == "lr":
        xx = rs(x, rx1, n * rx2)
        Phi = rs(Phi_prev, rx1, ry1 * ra1)
        Phi = xx.T @ Phi                                        # :861
        if A is not None:
            Phi = rs(Phi, n * rx2 * ry1, ra1).T                 # :863-864
            Phi = rs(Phi, ra1 * n, rx2 * ry1)
            Phi = rs(A, ra1 * n, m * ra2).T @ Phi               # :866-867
            Phi = rs(Phi, m, ra2 * rx2 * ry1)
        else:
            Phi = rs(Phi, n, rx2 * ry1)
        Phi = Phi.T                                             # :872
        Phi = rs(Phi, ra2 * rx2, ry1 * m)
        Phi = Phi @ rs(y, ry1 * m, ry2)                         # :875-876
        if A is not None:
            Phi = rs(Phi, ra2, rx2 * ry2).T
        Phi = rs(Phi, rx2, ry2, ra2)
        if A is None:
            Phi = rs(Phi, rx2, ry2)
    else:
        yy = rs(y, ry1 * m, ry2)
        Phi = rs(Phi_prev, ry2, ra2 * rx2)
        Phi = yy @ Phi                                          # :886
        if A is not None:
            Phi = rs(Phi, ry1, m * ra2 * rx2).T                 # :888-889
            Phi = rs(Phi, m * ra2, rx2 * ry1)
            Phi = rs(A, ra1 * n, m * ra2) @ Phi                 # :891-892
            Phi = rs(Phi, ra1 * n * rx2, ry1).T                 # :893-894
        Phi = rs(Phi, ry1 * ra1, n * rx2)
        Phi = Phi @ rs(x, rx1, n * rx2).T                       # :898-899
        if A is not None:
            Phi = rs(Phi, ry1, ra1, rx1)
        else:
            Phi = rs(Phi, ry1, rx1)
    nrm = None
    if want_norm:
        nrm = np.linalg.norm(Phi)
        if nrm > 0:
            Phi = Phi / nrm
        else:
            nrm = 1.0
    elif extnrm is not None:
        Phi = Phi / extnrm
    return np.asfortranarray(Phi), nrm


def _phi3(P):
    """View an X'Y Phi ``[r, r']`` as ``[r, r', 1]`` (MATLAB trailing singleton)."""
    return P if P.ndim == 3 else P.reshape(P.shape[0], P.shape[1], 1, order="F")


def _phi3_right(P):
    """View an X'Y right Phi ``[r, r']`` as ``[r, 1, r']``."""
    return P if P.ndim == 3 else P.reshape(P.shape[0], 1, P.shape[1], order="F")


# ---------------------------------------------------------------------------
# Local GMRES (Householder Arnoldi + Givens), fmex/solve3d.c:339-518
# ---------------------------------------------------------------------------

def dgmresr_hh(mv, rhs, nrestart, tol, niters, stats=None, force_iters=None):
    """Right-preconditioned GMRES with Householder orthogonalisation.

    Restates ``fmex/solve3d.c:339-518`` (no preconditioner).  Starts from
    ``sol = 0`` (``:366``); ``tol`` is relative to the initial residual norm
    of the first restart (``:383,473``).  ``mv`` applies the local operator.
    Returns the solution.  ``stats`` (a dict) receives ``matvecs``,
    ``gmres_calls``, and for this call ``iters`` (Krylov steps over all
    restarts), ``hist`` (the residual estimate after every step) and
    ``gm_tol``.  ``force_iters`` replaces the stopping test ``curres < tol``
    (``:476,508``) by "stop after that many steps": a checker uses it to
    follow another implementation's step count, after it has compared the
    estimates in ``hist`` with ``tol``.
    """
    sz = rhs.size
    U = np.zeros((sz, nrestart + 1))
    tau = np.zeros(nrestart + 1)
    J = np.zeros((2, nrestart))
    R = np.zeros((nrestart, nrestart), order="F")
    sol = np.zeros(sz)
    nrmrhs = None
    curres = np.inf
    nmv = 0
    j = 0
    hist = []

    def stop():
        if force_iters is None:
            return curres < tol
        return len(hist) >= force_iters

    for it in range(niters):
        w = mv(sol)                                     # :376
        nmv += 1
        w = rhs - w                                     # :378-380
        nrmr = np.linalg.norm(w)                        # :381
        if it == 0:
            nrmrhs = nrmr                               # :383
        if nrmr == 0.0:
            # Exact solution already; the reference would divide by zero here.
            curres = 0.0
            break
        beta = -nrmr if w[0] < 0.0 else nrmr            # :385-386
        w[0] += beta                                    # :387
        tau[:] = 0.0
        tau[0] = -beta                                  # :388
        w = w / np.linalg.norm(w)                       # :389-391
        U[:, 0] = w                                     # :392
        broke = False
        for j in range(nrestart):
            w = U[:, j] * (-2.0 * U[j, j])              # :396-398
            w[j] += 1.0                                 # :399
            for i in range(j - 1, -1, -1):              # :400-403
                w -= 2.0 * np.dot(U[:, i], w) * U[:, i]
            w = w / np.linalg.norm(w)                   # :404-406
            w = mv(w)                                   # :417
            nmv += 1
            for i in range(j + 1):                      # :421-424
                w -= 2.0 * np.dot(U[:, i], w) * U[:, i]
            if j < sz - 1:                              # :427-442
                U[: j + 1, j + 1] = 0.0
                U[j + 1:, j + 1] = w[j + 1:]
                alpha = np.linalg.norm(U[j + 1:, j + 1])
                if alpha != 0.0:
                    if w[j + 1] < 0.0:
                        alpha = -alpha
                    U[j + 1, j + 1] += alpha
                    U[j + 1:, j + 1] /= np.linalg.norm(U[j + 1:, j + 1])
                    w[j + 1] = -alpha
                    w[j + 2:] = 0.0
            for i in range(j):                          # :445-449
                b = w[i]
                w[i] = J[0, i] * w[i] + J[1, i] * w[i + 1]
                w[i + 1] = -J[1, i] * b + J[0, i] * w[i + 1]
            if j < sz - 1:                              # :454-465
                rho = np.sqrt(w[j] * w[j] + w[j + 1] * w[j + 1])
                J[0, j] = w[j] / rho
                J[1, j] = w[j + 1] / rho
                tau[j + 1] = -J[1, j] * tau[j]
                tau[j] = J[0, j] * tau[j]
                w[j] = rho
                w[j + 1] = 0.0
            R[:, j] = w[:nrestart]                      # :469
            curres = abs(tau[j + 1]) / nrmrhs           # :473
            hist.append(curres)
            if stop():                                  # :476
                broke = True
                break
        if not broke:                                   # :482-486
            j = nrestart - 1
            ni = nrestart
        else:
            ni = j + 1
        # dtrsv upper, in place on tau[0:ni]            # :487
        y = np.zeros(ni)
        for row in range(ni - 1, -1, -1):
            y[row] = (tau[row] - np.dot(R[row, row + 1:ni], y[row + 1:ni])) / R[row, row]
        tau[:ni] = y
        # Correction (:496-507)
        w = U[:, j] * (-2.0 * U[j, j] * tau[j])
        w[j] += tau[j]
        for i in range(j - 1, -1, -1):
            w[i] += tau[i]
            w -= 2.0 * np.dot(U[:, i], w) * U[:, i]
        sol = sol + w
        if stop():                                      # :508
            break
    if stats is not None:
        stats["matvecs"] = stats.get("matvecs", 0) + nmv
        stats["gmres_calls"] = stats.get("gmres_calls", 0) + 1
        stats["iters"] = len(hist)
        stats["hist"] = hist
        stats["gm_tol"] = tol
    return sol


def jac_gen(Phi1, A, Phi2, prec):
    """Block-Jacobi local preconditioners (``solve/solve3d_2ml.m:21-70``; the
    centre variant also in ``fmex/solve3d.c:47-112``).

    prec 1 ('cjacobi'): for every rank pair (i, k) the n x n diagonal block
      ``J[:, :, i, k] = sum_{al,be} Phi1[i,i,al] A[al,:,:,be] Phi2[k,be,k]``,
      inverted; returned as ``[n, n, rx1, rx2]``.
    prec 2 ('ljacobi'): for every k the (rx1 n) x (rx1 n) block
      ``sum_{al,be} Phi1[:,:,al] (x) A[al,:,:,be] Phi2[k,be,k]``, inverted:
      ``[rx1 n, rx1 n, rx2]``.
    prec 3 ('rjacobi'): for every i the (n rx2) x (n rx2) block
      ``sum_{al,be} Phi1[i,i,al] A[al,:,:,be] (x) Phi2[:,be,:]``, inverted:
      ``[n rx2, n rx2, rx1]``."""
    rx1, ra1 = Phi1.shape[1], Phi1.shape[2]
    n = A.shape[1]
    rx2, ra2 = Phi2.shape[0], Phi2.shape[1]
    d1 = np.stack([np.diag(Phi1[:, :, a]) for a in range(ra1)], axis=1)     # [rx1, ra1]
    d2 = np.stack([np.diag(Phi2[:, b, :]) for b in range(ra2)], axis=0)     # [ra2, rx2]
    if prec == 1:
        J = np.einsum("ia,ajmb,bk->jmik", d1, A, d2)                      # [n, n, rx1, rx2]
        out = np.empty_like(J)
        for i in range(rx1):
            for k in range(rx2):
                out[:, :, i, k] = np.linalg.inv(J[:, :, i, k])
        return out
    if prec == 2:
        J = np.einsum("ipa,ajmb,bk->ijpmk", Phi1, A, d2)                  # [rx1,n,rx1,n,rx2]
        J = J.reshape(rx1 * n, rx1 * n, rx2, order="F")
        return np.stack([np.linalg.inv(J[:, :, k]) for k in range(rx2)], axis=2)
    if prec == 3:
        J = np.einsum("ia,ajmb,qbk->jkmqi", d1, A, Phi2)                  # [n,rx2,n,rx2,rx1]
        J = J.reshape(n * rx2, n * rx2, rx1, order="F")
        return np.stack([np.linalg.inv(J[:, :, i]) for i in range(rx1)], axis=2)
    raise ValueError("unknown preconditioner %r" % (prec,))


def jac_apply(jacs, prec, x, rx1, n, rx2):
    """``y = P x`` for the preconditioners of ``jac_gen``
    (``solve/solve3d_2ml.m:120-146``, ``fmex/solve3d.c:115-128``)."""
    X = rs(x, rx1, n, rx2)
    if prec == 1:
        Y = np.einsum("jmik,imk->ijk", jacs, X)
    elif prec == 2:
        Y = np.einsum("pqk,qk->pk", jacs, rs(X, rx1 * n, rx2))
    elif prec == 3:
        Xt = rs(np.transpose(X, (1, 2, 0)), n * rx2, rx1)
        Yt = np.einsum("pqi,qi->pi", jacs, Xt)
        Y = np.transpose(rs(Yt, n, rx2, rx1), (2, 0, 1))
    else:
        raise ValueError("unknown preconditioner %r" % (prec,))
    return np.asfortranarray(Y).ravel(order="F")


def solve3d_2(Phi1, A, Phi2, rhs, tol, sol_prev, nrestart=40, niters=2, stats=None, prec=0,
              force_iters=None):
    """MEX local solver, residual branch (``fmex/solve3d_2.c:121-300``).

    ``tol`` is relative to ``||rhs||``.  Computes ``dres = rhs - B sol_prev``,
    runs ``dgmresr_hh`` with tolerance ``tol/max(||dres||/||rhs||, tol)`` and
    returns ``sol_prev + dsol`` (``:254-279``).  ``prec`` 1/2/3 (cjacobi,
    ljacobi, rjacobi) right-preconditions the Krylov solve with ``jac_gen``:
    the matvec is ``B P`` and ``dsol = P y`` (``:226-231,272-274``)."""
    rx1, n, rx2 = Phi1.shape[1], A.shape[1], Phi2.shape[0]
    sz = rx1 * n * rx2
    if nrestart > sz:                                   # :184
        nrestart = sz
    dres = rhs - bfun3(Phi1, A, Phi2, sol_prev)         # :257-262
    if stats is not None:
        stats["matvecs"] = stats.get("matvecs", 0) + 1
    tol_prev = np.linalg.norm(dres) / np.linalg.norm(rhs)   # :263
    if tol_prev < tol:
        tol_prev = tol                                  # :264
    if prec:
        jacs = jac_gen(Phi1, A, Phi2, prec)
        mv = lambda v: bfun3(Phi1, A, Phi2, jac_apply(jacs, prec, v, rx1, n, rx2))
    else:
        mv = lambda v: bfun3(Phi1, A, Phi2, v)
    dsol = dgmresr_hh(mv, dres, nrestart, tol / tol_prev, niters, stats,
                      force_iters)                                          # :267
    if prec:
        dsol = jac_apply(jacs, prec, dsol, rx1, n, rx2)                    # :272-274
    return dsol + sol_prev                              # :277-278


def assemble_local(Phi1, A1, Phi2):
    """Dense local matrix ``B`` for the full-solve branch (``amen_solve2.m:472-480``)."""
    rx1, ra1 = Phi1.shape[0], Phi1.shape[2]
    n = A1.shape[1]
    rx2, ra2 = Phi2.shape[0], Phi2.shape[1]
    B = rs(Phi1, rx1 * rx1, ra1) @ rs(A1, ra1, n * n * ra2)
    B = rs(B, rx1, rx1, n, n * ra2)
    B = np.transpose(B, (0, 2, 1, 3))
    B = rs(B, rx1 * n * rx1 * n, ra2)
    B = B @ rs(np.transpose(Phi2, (1, 2, 0)), ra2, rx2 * rx2)
    B = rs(B, rx1 * n, rx1 * n, rx2, rx2)
    B = np.transpose(B, (0, 2, 1, 3))
    return rs(B, rx1 * n * rx2, rx1 * n * rx2)


# ---------------------------------------------------------------------------
# AMEn driver, solve/amen_solve2.m
# ---------------------------------------------------------------------------

DEFAULTS = dict(nswp=50, rmax=1000, max_full_size=50, local_restart=40, local_iters=2,
                kickrank=4, resid_damp=2.0, tol_exit=None, verb=0, local_prec="")

# local_prec names -> the MEX prec code (solve/amen_solve2.m:205-207)
LOCAL_PREC = {"": 0, "cjacobi": 1, "ljacobi": 2, "rjacobi": 3}


def _near(v, ref, near_tie):
    """``v`` lies within relative ``near_tie`` of the threshold ``ref``."""
    return ref > 0 and abs(v / ref - 1.0) < near_tie


class _Follow:
    """Decision checker: compares this solve's discrete decisions with those
    another implementation recorded (``steps``: one dict per local step with
    ``rank``, ``iters``, ``res_prev`` and ``res_new``, as ``ttg_amen_step``;
    ``max_res``: its per-sweep maxima).  Where the two differ and the
    compared quantity lies near its threshold (a near tie: rounding decides),
    the other implementation's choice is adopted and the step is listed in
    ``flips``; otherwise the difference is listed in ``mismatches`` (and the
    choice adopted as well, so that the comparison can go on).  "Near" is
    relative ``near_tie``, or four times the relative difference of the two
    implementations' own local residuals of that step when that is larger:
    the residuals that set the thresholds carry that much rounding noise
    (it grows where a local solve ends close to the FP64 floor)."""

    def __init__(self, steps, max_res, near_tie):
        self.steps = {(s["sweep"], s["core"]): s for s in steps}
        self.max_res = list(max_res)
        self.near_tie = near_tie
        self.flips = []
        self.mismatches = []

    def step(self, swp, i):
        s = self.steps.get((swp, i))
        if s is None:
            self.mismatches.append(dict(kind="missing step", sweep=swp, core=i))
        return s

    def noise(self, step, res_prev, res_new=None):
        """Tie bound of a step: near_tie, or 4x the relative difference of
        the two sides' local residuals of the step."""
        d = 0.0
        for mine, key in ((res_prev, "res_prev"), (res_new, "res_new")):
            other = step.get(key) if step is not None else None
            if mine is not None and other is not None and mine > 0:
                d = max(d, abs(other / mine - 1.0))
        return max(self.near_tie, 4.0 * d)

    def gmres(self, swp, i, hist, gm_tol, iters_o, iters_g, cap, tie=None):
        """Krylov step count: the other side stopped after ``iters_g`` steps,
        i.e. its estimate stayed >= tol before and fell below at that step
        (unless it hit the cap)."""
        if iters_g == iters_o:
            return
        near = self.near_tie if tie is None else tie
        bad = []
        for k, cr in enumerate(hist[:iters_g], start=1):
            implied = (k == iters_g)
            if k == iters_g and iters_g >= cap:
                continue
            if (cr < gm_tol) != implied and not _near(cr, gm_tol, near):
                bad.append(k)
        lo, hi = min(iters_o, iters_g), max(iters_o, iters_g)
        rec = dict(kind="gmres steps", sweep=swp, core=i, own=iters_o, other=iters_g,
                   ratio_to_tol=[float(v / gm_tol) for v in hist[max(lo - 2, 0):hi + 1]])
        (self.mismatches if bad or len(hist) < iters_g else self.flips).append(rec)

    def rank(self, swp, i, r_own, r_g, K, cap, thr, res_of, tie=None):
        """Truncation rank: the other side kept ``r_g`` (after the caps
        ``min(., K, rmax)``), i.e. its candidate residuals stayed <= thr for
        candidates >= r_g and exceeded thr at r_g - 1 (when r_g is not
        capped and not the loop's fall-through value 2)."""
        if r_g == r_own:
            return
        near = self.near_tie if tie is None else tie
        bad = []
        capped = r_g >= cap
        for rr in range(K - 1, max(r_g - 1, 1) - 1, -1):
            if rr >= r_g:
                implied = False
            elif capped or r_g == 2:
                continue
            else:
                implied = True
            v = res_of(rr)
            if (v > thr) != implied and not _near(v, thr, near):
                bad.append(rr)
        if capped and r_g > r_own:
            # the other side's exceeding candidate lies somewhere >= r_g - 1
            if not any(_near(res_of(rr), thr, near) for rr in range(r_g - 1, K)):
                bad.append(r_g - 1)
        lo = max(min(r_own, r_g) - 1, 1)
        rec = dict(kind="rank", sweep=swp, core=i, own=r_own, other=r_g,
                   ratio_to_thr={rr: float(res_of(rr) / thr)
                                 for rr in range(lo, min(max(r_own, r_g) + 1, K))})
        (self.mismatches if bad else self.flips).append(rec)

    def stop(self, swp, max_res, tol_exit):
        if swp - 1 >= len(self.max_res):
            self.mismatches.append(dict(kind="missing sweep", sweep=swp))
            return max_res < tol_exit
        own = max_res < tol_exit
        other = self.max_res[swp - 1] < tol_exit
        if own != other:
            tie = max(self.near_tie, 4.0 * abs(self.max_res[swp - 1] / max_res - 1.0))
            rec = dict(kind="sweep stop", sweep=swp, own=own, other=other)
            (self.flips if _near(max_res, tol_exit, tie) else self.mismatches).append(rec)
        return other


def amen_solve2(A, y, tol, x0, z0=None, trace=None, follow=None, near_tie=1e-6, **opts):
    """``[x, testdata, z] = amen_solve2(A, y, tol, ...)`` on the default path.

    ``x0`` is required (the reference draws ``tt_rand(n,d,2,-1)`` from
    MATLAB's RNG, ``:222-224``, which cannot be reproduced); ``z0`` likewise
    (``:250-252``; defaults to the rank-``kickrank`` right-orthogonal TT drawn
    from ``numpy`` with seed 0 when omitted).  Returns ``(x, info)``; ``info``
    holds per-sweep ``max_res``, ``max_dx``, ranks and operation counts.

    ``trace`` (a list) receives one dict per local step: sweep, core, kept
    rank, Krylov steps, local residuals, the truncation threshold and the
    step's decision margins (``rank_margin``: the smallest
    ``|res/thr - 1|`` over the candidates the rank loop examined;
    ``gmres_margin``: the smallest ``|curres/tol - 1|`` over the Krylov
    steps).  ``follow`` (dict with ``steps`` and ``max_res`` recorded by
    another implementation) checks every discrete decision against the
    other implementation's and adopts the other's choice at near ties
    (relative distance to the threshold below ``near_tie``); ``info``
    then holds ``flips`` (adopted near ties) and ``mismatches`` (differences
    that were not near ties).
    """
    o = dict(DEFAULTS)
    for k, v in opts.items():
        if k not in o:
            raise ValueError("Unrecognized option: %s" % k)   # :200-201
        o[k] = v
    nswp, rmax = o["nswp"], o["rmax"]
    max_full_size = o["max_full_size"]
    local_restart, local_iters = o["local_restart"], o["local_iters"]
    kickrank, resid_damp = o["kickrank"], float(o["resid_damp"])
    tol_exit = tol if o["tol_exit"] is None else o["tol_exit"]       # :156-158
    verb = o["verb"]
    prec = LOCAL_PREC[o["local_prec"]]                                 # :205-207

    if np.any(A.n != A.m):
        raise ValueError("AMEn does not know how to solve rectangular systems!")  # :216-218
    d = y.d
    n = [int(v) for v in A.n]
    crx = [c.copy(order="F") for c in x0.cores]                       # :226-227
    rx = [int(v) for v in x0.r]
    ry = [int(v) for v in y.r]
    ra = [int(v) for v in A.r]
    cry = [c for c in y.cores]                                         # :236-239
    crA = [c for c in A.cores]

    ones3 = np.ones((1, 1, 1), order="F")
    ones2 = np.ones((1, 1), order="F")
    phia = [None] * (d + 1); phia[0] = ones3; phia[d] = ones3         # :243
    phiy = [None] * (d + 1); phiy[0] = ones2; phiy[d] = ones2         # :244
    use_z = kickrank > 0                                               # :246 (kicktype 'als')
    if use_z:
        phiza = [None] * (d + 1); phiza[0] = ones3; phiza[d] = ones3  # :248
        phizy = [None] * (d + 1); phizy[0] = ones2; phizy[d] = ones2  # :249
        if z0 is None:
            from .tt import tt_rand
            z0 = tt_rand(n, d, kickrank, np.random.default_rng(0), -1)
        crz = [c.copy(order="F") for c in z0.cores]                    # :250-254
        rz = [int(v) for v in z0.r]

    nrmsa = np.ones(d - 1)                                             # :277-279
    nrmsy = np.ones(d - 1)
    nrmsx = np.ones(d - 1)
    nrmsc = 1.0                                                        # :282

    info = dict(max_res=[], max_dx=[], max_rank=[], matvecs=0, local_solves=0, sweeps=0,
                res_prev=[])
    fol = _Follow(follow["steps"], follow["max_res"], near_tie) if follow is not None else None
    st = {"matvecs": 0}
    last_sweep = False

    def mv_count(k=1):
        st["matvecs"] += k

    for swp in range(1, nswp + 1):                                     # :296
        # ---------------- right-to-left orthogonalisation (:299-438)
        for i in range(d - 1, 0, -1):
            if use_z and not last_sweep:                               # :301-324
                if swp > 1:
                    crzAt = bfun3(phiza[i], crA[i], phiza[i + 1],
                                  rs(crx[i], rx[i] * n[i] * rx[i + 1]))
                    mv_count()
                    crzAt = rs(crzAt, rz[i] * n[i], rz[i + 1])
                    crzy = phizy[i] @ rs(cry[i], ry[i], n[i] * ry[i + 1])
                    crzy = rs(crzy, rz[i] * n[i], ry[i + 1])
                    crzy = crzy @ phizy[i + 1]
                    crznew = crzy * nrmsc - crzAt
                    crznew = rs(crznew, rz[i], n[i] * rz[i + 1])
                    _, _, vh = np.linalg.svd(crznew, full_matrices=False)
                    crznew = vh.T[:, :min(kickrank, vh.shape[0])]
                else:
                    crznew = rs(crz[i], rz[i], n[i] * rz[i + 1]).T
                crznew, _ = np.linalg.qr(crznew)                       # :320
                rznew = crznew.shape[1]
                crz[i] = rs(crznew.T, rznew, n[i], rz[i + 1])          # :322-323
            if swp > 1:                                                # :325-328
                nrmsc = nrmsc / (nrmsy[i - 1] / (nrmsa[i - 1] * nrmsx[i - 1]))
            cr = rs(crx[i], rx[i], n[i] * rx[i + 1]).T                 # :331-333
            cr, rv = np.linalg.qr(cr)                                  # :342
            cr2 = rs(crx[i - 1], rx[i - 1] * n[i - 1], rx[i])
            cr2 = cr2 @ rv.T                                           # :349
            curnorm = np.linalg.norm(cr2)                              # :351-357
            if curnorm > 0:
                cr2 = cr2 / curnorm
            else:
                curnorm = 1.0
            nrmsx[i - 1] *= curnorm
            rx[i] = cr.shape[1]                                        # :359
            cr = rs(cr.T, rx[i], n[i], rx[i + 1])
            crx[i - 1] = rs(cr2, rx[i - 1], n[i - 1], rx[i])
            crx[i] = cr
            phia[i], nrmsa[i - 1] = compute_next_Phi(phia[i + 1], cr, crA[i], cr, "rl", want_norm=True)  # :364
            phiy[i], nrmsy[i - 1] = compute_next_Phi(phiy[i + 1], cr, None, cry[i], "rl", want_norm=True)  # :365
            nrmsc = nrmsc * (nrmsy[i - 1] / (nrmsa[i - 1] * nrmsx[i - 1]))  # :372
            if use_z and not last_sweep:                               # :432-436
                rz[i] = rznew
                phiza[i], _ = compute_next_Phi(phiza[i + 1], crz[i], crA[i], crx[i], "rl", extnrm=nrmsa[i - 1])
                phizy[i], _ = compute_next_Phi(phizy[i + 1], crz[i], None, cry[i], "rl", extnrm=nrmsy[i - 1])

        # ---------------- left-to-right solve sweep (:444-791)
        max_res = 0.0
        max_dx = 0.0
        res_list = []
        for i in range(d):
            Phi1 = phia[i]
            Phi2 = phia[i + 1]
            A1 = crA[i]
            other = fol.step(swp, i) if fol is not None else None
            step_iters, gm_margin = -1, None
            sol_prev = rs(crx[i], rx[i] * n[i] * rx[i + 1])            # :451
            y1 = cry[i] * nrmsc                                        # :453
            rhs = phiy[i] @ rs(y1, ry[i], n[i] * ry[i + 1])            # :456-458
            rhs = rs(rhs, rx[i] * n[i], ry[i + 1]) @ phiy[i + 1]       # :459-460
            rhs = rs(rhs, rx[i] * n[i] * rx[i + 1])
            norm_rhs = np.linalg.norm(rhs)                             # :462
            real_tol = (tol / np.sqrt(d)) / resid_damp                 # :466
            full = rx[i] * n[i] * rx[i + 1] < max_full_size            # :468
            if full:
                B = assemble_local(Phi1, A1, Phi2)                     # :472-480
                res_prev = np.linalg.norm(B @ sol_prev - rhs) / norm_rhs   # :482
                sol = np.linalg.solve(B, rhs)                          # :486
                res_new = np.linalg.norm(B @ sol - rhs) / norm_rhs     # :487
            else:
                res_prev = np.linalg.norm(bfun3(Phi1, A1, Phi2, sol_prev) - rhs) / norm_rhs  # :495
                mv_count()
                if norm_rhs > 0:                                       # :497
                    gst = {}
                    force = None
                    if other is not None and other["iters"] >= 0:
                        # the step count this solve takes on its own (same
                        # arithmetic, no side effects), then the check
                        solve3d_2(Phi1, A1, Phi2, rhs, real_tol, sol_prev, local_restart,
                                  local_iters, gst, prec)
                        cap = min(local_restart, sol_prev.size) * local_iters
                        fol.gmres(swp, i, gst["hist"], gst["gm_tol"], gst["iters"],
                                  other["iters"], cap, fol.noise(other, res_prev))
                        force = other["iters"]
                        gst = {}
                    sol = solve3d_2(Phi1, A1, Phi2, rhs, real_tol, sol_prev,
                                    local_restart, local_iters, gst, prec, force)  # :501
                    st["matvecs"] += gst.get("matvecs", 0)
                    step_iters = gst["iters"]
                    gm_margin = min((abs(v / gst["gm_tol"] - 1.0) for v in gst["hist"]),
                                    default=None)
                    info["local_solves"] += 1
                    res_new = np.linalg.norm(bfun3(Phi1, A1, Phi2, sol) - rhs) / norm_rhs   # :504
                    mv_count()
                else:
                    sol = np.zeros(sol_prev.size)
                    res_new = 0.0
            nsol = np.linalg.norm(sol)
            dx = np.linalg.norm(sol - sol_prev) / nsol if nsol > 0 else 0.0   # :519
            max_dx = max(max_dx, dx)
            max_res = max(max_res, res_prev)                           # :521
            res_list.append(res_prev)

            sol = rs(sol, rx[i] * n[i], rx[i + 1])                     # :530
            thr, rank_margin = None, None
            if kickrank >= 0 and i < d - 1:                            # :532
                u, s, vh = np.linalg.svd(sol, full_matrices=False)     # :533
                v = vh.T
                K = min(rx[i] * n[i], rx[i + 1])
                thr = max(real_tol * resid_damp, res_new)
                cand = {}

                def res_of(rr):
                    if rr not in cand:
                        cursol = (u[:, :rr] * s[:rr]) @ v[:, :rr].T
                        if full:
                            cand[rr] = np.linalg.norm(B @ rs(cursol, cursol.size) - rhs) / norm_rhs
                        else:
                            cand[rr] = np.linalg.norm(bfun3(Phi1, A1, Phi2, rs(cursol, cursol.size))
                                                      - rhs) / norm_rhs
                            mv_count()
                    return cand[rr]

                r = None
                for r in range(K - 1, 0, -1):                          # :539-550
                    res = res_of(r)
                    if res > thr:
                        break
                rank_margin = min((abs(v_ / thr - 1.0) for v_ in cand.values()), default=None)
                # MATLAB leaves r at the last loop value (1) when no break
                # happens; an empty loop (K == 1) leaves r empty, treated as K-1.
                r = (K - 1 if r is None else r) + 1                    # :551
                r = min(r, s.size)                                     # :593
                r = min(r, rmax)                                       # :594
                if other is not None:
                    r_own = r
                    r = other["rank"]
                    fol.rank(swp, i, r_own, r, K, min(s.size, rmax), thr, res_of,
                             fol.noise(other, res_prev, res_new))
            else:                                                      # :596-601
                u, v = np.linalg.qr(sol)
                v = v.T
                r = u.shape[1]
                s = np.ones(r)
            u = u[:, :r]                                               # :603
            v = v[:, :r] * s[:r]                                       # :604
            if trace is not None:
                trace.append(dict(sweep=swp, core=i, rank=r if i < d - 1 else -1,
                                  iters=step_iters, res_prev=res_prev, res_new=res_new,
                                  thr=thr, rank_margin=rank_margin, gmres_margin=gm_margin))

            if use_z and not last_sweep:                               # :605-623
                crzAt = bfun3(phiza[i], A1, phiza[i + 1], rs(u @ v.T, u.shape[0] * v.shape[0]))
                mv_count()
                crzAt = rs(crzAt, rz[i] * n[i], rz[i + 1])
                crzy = phizy[i] @ rs(y1, ry[i], n[i] * ry[i + 1])
                crzy = rs(crzy, rz[i] * n[i], ry[i + 1])
                crzy = crzy @ phizy[i + 1]
                crznew = crzy - crzAt
                uz, _, _ = np.linalg.svd(crznew, full_matrices=False)
                crznew = uz[:, :min(kickrank, uz.shape[1])]
                crznew, _ = np.linalg.qr(crznew)                       # :619
                rznew = crznew.shape[1]
                crz[i] = rs(crznew, rz[i], n[i], rznew)

            if i < d - 1:                                              # :625
                if kickrank > 0 and not last_sweep:                    # :626
                    leftresid = bfun3(Phi1, A1, phiza[i + 1], rs(u @ v.T, u.shape[0] * v.shape[0]))  # :702
                    mv_count()
                    leftresid = rs(leftresid, rx[i] * n[i], rz[i + 1])
                    lefty = phiy[i] @ rs(y1, ry[i], n[i] * ry[i + 1])
                    lefty = rs(lefty, rx[i] * n[i], ry[i + 1])
                    lefty = lefty @ phizy[i + 1]
                    uk = lefty - leftresid                             # :707
                    u, rv = np.linalg.qr(np.hstack([u, uk]))           # :713
                    radd = uk.shape[1]
                    v = np.hstack([v, np.zeros((rx[i + 1], radd))])    # :715
                    v = v @ rv.T                                       # :716
                r = u.shape[1]                                         # :718
                cr2 = rs(crx[i + 1], rx[i + 1], n[i + 1] * rx[i + 2])
                v = v.T @ cr2                                          # :734
                nrmsc = nrmsc / (nrmsy[i] / (nrmsa[i] * nrmsx[i]))     # :737
                curnorm = np.linalg.norm(v)                            # :739-745
                if curnorm > 0:
                    v = v / curnorm
                else:
                    curnorm = 1.0
                nrmsx[i] *= curnorm
                u = rs(u, rx[i], n[i], r)                              # :747-748
                v = rs(v, r, n[i + 1], rx[i + 2])
                phia[i + 1], nrmsa[i] = compute_next_Phi(phia[i], u, crA[i], u, "lr", want_norm=True)   # :751
                phiy[i + 1], nrmsy[i] = compute_next_Phi(phiy[i], u, None, cry[i], "lr", want_norm=True)  # :752
                nrmsc = nrmsc * (nrmsy[i] / (nrmsa[i] * nrmsx[i]))     # :754
                rx[i + 1] = r                                          # :765
                crx[i] = u
                crx[i + 1] = v
                if use_z and not last_sweep:                           # :770-774
                    rz[i + 1] = rznew
                    phiza[i + 1], _ = compute_next_Phi(phiza[i], crz[i], crA[i], crx[i], "lr", extnrm=nrmsa[i])
                    phizy[i + 1], _ = compute_next_Phi(phizy[i], crz[i], None, cry[i], "lr", extnrm=nrmsy[i])
            else:
                crx[i] = rs(sol, rx[i], n[i], rx[i + 1])               # :778-779

        info["max_res"].append(max_res)
        info["max_dx"].append(max_dx)
        info["max_rank"].append(max(rx))
        info["res_prev"].append(res_list)
        info["sweeps"] = swp
        if verb > 0:
            print("=amen_solve= sweep %d, max_dx: %3.3e, max_res: %3.3e, max_rank: %g"
                  % (swp, max_dx, max_res, max(rx)))                   # :793-795
        if last_sweep:                                                 # :797-799
            break
        stop = max_res < tol_exit                                      # :806-808
        if fol is not None:
            stop = fol.stop(swp, max_res, tol_exit)
        if stop:
            last_sweep = True

    nx = np.exp(np.sum(np.log(nrmsx)) / d)                             # :816
    crx = [c * nx for c in crx]                                        # :818-820
    info["matvecs"] = st["matvecs"]
    info["ranks"] = list(rx)
    if fol is not None:
        info["flips"] = fol.flips
        info["mismatches"] = fol.mismatches
    return TT(crx), info
