"""The oracle's local kernels against the reference's own C.

``oracle/build_ref.py`` compiles TT-Toolbox's ``fmex/solve3d.c`` (where it
lies in the reference tree) against MEX/BLAS stand-ins into
``oracle/_ref/libsolve3d_ref.so``; this file calls its ``bfun3``,
``dgmresr_hh`` (Householder GMRES, ``fmex/solve3d.c:339-518``) and
``dcjacgen``/``dcjacapply`` (``:47-139``) through ctypes and requires the
oracle's restatements (``oracle/amen.py``) to agree.  ``fmex/solve3d.c``
takes Phi2 as ``[rx2', rx2, ra2]`` (``:836-838``), the transpose of
amen_solve2's ``[rx2, ra2, rx2']``; the arrays are permuted accordingly.
Without the reference tree and no prebuilt library the tests are skipped.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import amen as oamen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# The reference tree is read only here, in the CPU suite of the build
# container; elsewhere a library built earlier is used, or the tests skip.
REF_TREE = os.environ.get("TTG_REFERENCE_TREE", "/root/reference")

_pd = C.POINTER(C.c_double)
_l = C.c_long


def _lib():
    from oracle import build_ref
    path = build_ref.LIB
    if os.path.isdir(REF_TREE):
        path = build_ref.build(REF_TREE) or path
    if not os.path.exists(path):
        pytest.skip("reference checker library not built (no reference tree here)")
    L = C.CDLL(path)
    L.bfun3.argtypes = [_pd, _pd, _pd, _l, _l, _l, _l, _l, _pd, _pd]
    L.bfun3.restype = None
    L.dgmresr_hh.argtypes = [_pd, _pd, _pd, _pd, _l, _l, _l, _l, _l, _l, C.c_double, _l, _pd,
                             _pd, C.c_char]
    L.dgmresr_hh.restype = None
    L.dcjacgen.argtypes = [_pd, _pd, _pd, _l, _l, _l, _l, _l, _pd]
    L.dcjacgen.restype = None
    L.dcjacapply.argtypes = [_pd, _l, _l, _l, _pd, _pd]
    L.dcjacapply.restype = None
    return L


def _p(a):
    return a.ctypes.data_as(_pd)


def _f(a):
    """Column-major contiguous copy (what the C code indexes)."""
    return np.asfortranarray(a, dtype=np.float64).ravel(order="F").copy()


def _system(rng, rx1, n, rx2, ra1=2, ra2=3, shift=8.0):
    Phi1 = rng.standard_normal((rx1, rx1, ra1)) * 0.1
    Phi1[:, :, 0] += shift * np.eye(rx1)
    A = rng.standard_normal((ra1, n, n, ra2)) * 0.1
    A[0, :, :, 0] += np.eye(n) * 2.0
    Phi2 = rng.standard_normal((rx2, ra2, rx2)) * 0.1
    Phi2[:, 0, :] += shift * np.eye(rx2)
    return Phi1, A, Phi2


def _phi2_c(Phi2):
    return np.transpose(Phi2, (2, 0, 1))


@pytest.mark.parametrize("rx1,n,rx2,ra1,ra2", [(1, 4, 2, 1, 2), (3, 5, 7, 2, 3), (9, 6, 4, 3, 2)])
def test_bfun3_matches_reference_c(rx1, n, rx2, ra1, ra2):
    L = _lib()
    rng = np.random.default_rng(rx1 * 13 + n)
    Phi1, A, Phi2 = _system(rng, rx1, n, rx2, ra1, ra2)
    x = rng.standard_normal(rx1 * n * rx2)
    y = np.zeros_like(x)
    P1, AA, P2, xx = _f(Phi1), _f(A), _f(_phi2_c(Phi2)), x.copy()
    L.bfun3(_p(P1), _p(AA), _p(P2), rx1, n, rx2, ra1, ra2, _p(xx), _p(y))
    ref = oamen.bfun3(Phi1, A, Phi2, x)
    assert np.linalg.norm(y - ref) <= 1e-13 * np.linalg.norm(ref)


@pytest.mark.parametrize("rx1,n,rx2,nrestart,tol,niters",
                         [(3, 4, 5, 40, 1e-10, 2), (6, 8, 5, 12, 1e-8, 3), (8, 10, 7, 20, 1e-12, 2),
                          (2, 3, 2, 5, 1e-14, 1)])
def test_dgmresr_hh_matches_reference_c(rx1, n, rx2, nrestart, tol, niters):
    L = _lib()
    rng = np.random.default_rng(rx1 + 100 * n)
    Phi1, A, Phi2 = _system(rng, rx1, n, rx2)
    ra1, ra2 = A.shape[0], A.shape[3]
    sz = rx1 * n * rx2
    nrestart = min(nrestart, sz)
    rhs = rng.standard_normal(sz)
    sol = np.zeros(sz)
    P1, AA, P2, rr = _f(Phi1), _f(A), _f(_phi2_c(Phi2)), rhs.copy()
    L.dgmresr_hh(_p(P1), _p(AA), _p(P2), _p(rr), rx1, n, rx2, ra1, ra2, nrestart, tol, niters,
                 None, _p(sol), b"\0")
    st = {}
    ref = oamen.dgmresr_hh(lambda v: oamen.bfun3(Phi1, A, Phi2, v), rhs, nrestart, tol, niters,
                           st)
    assert np.linalg.norm(sol - ref) <= 1e-11 * np.linalg.norm(ref)


@pytest.mark.parametrize("rx1,n,rx2", [(3, 4, 5), (5, 7, 2)])
def test_cjacobi_matches_reference_c(rx1, n, rx2):
    L = _lib()
    rng = np.random.default_rng(7 * rx1 + n)
    Phi1, A, Phi2 = _system(rng, rx1, n, rx2)
    ra1, ra2 = A.shape[0], A.shape[3]
    jacs = np.zeros(n * n * rx1 * rx2)
    L.dcjacgen(_p(_f(Phi1)), _p(_f(A)), _p(_f(_phi2_c(Phi2))), rx1, n, rx2, ra1, ra2, _p(jacs))
    ref = oamen.jac_gen(Phi1, A, Phi2, 1)
    assert np.linalg.norm(jacs - _f(ref)) <= 1e-12 * np.linalg.norm(ref)
    x = rng.standard_normal(rx1 * n * rx2)
    y = np.zeros_like(x)
    xx = x.copy()
    L.dcjacapply(_p(jacs), n, rx1, rx2, _p(xx), _p(y))
    yref = oamen.jac_apply(ref, 1, x, rx1, n, rx2)
    assert np.linalg.norm(y - yref) <= 1e-12 * np.linalg.norm(yref)
