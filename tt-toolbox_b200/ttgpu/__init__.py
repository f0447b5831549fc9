"""Python host side of libttgpu (ctypes over the C ABI in include/ttgpu.h).

Mirrors the reference's MATLAB interface for the hot path, with the same
argument meaning and error behaviour:

* ``round(tt, eps, rmax=None)``            -- ``@tt_tensor/round.m:1``
* ``amen_solve2(A, y, tol, **opts)``       -- ``solve/amen_solve2.m:1`` (options :161-203)
* ``solve3d_2(Phi1, A, Phi2, rhs, tol, trunc_norm, sol_prev, prec, nrestart, niters, verb)``
                                            -- MEX gateway ``fmex/solve3d_2.c:121-122``
* ``bfun3(Phi1, A, Phi2, x)``              -- ``solve/amen_solve2.m:924-951``
* ``compute_next_Phi(Phi_prev, x, A, y, direction, extnrm=None)``
                                            -- ``solve/amen_solve2.m:834-920``

Host arrays are numpy FP64 in column-major reference layouts.  There is no
CPU fallback: loading fails loudly when ``libttgpu.so`` (or a GPU) is missing.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libttgpu.so")

TTG_FP64, TTG_MIXED = 0, 1
_PREC = {"fp64": TTG_FP64, "mixed": TTG_MIXED, TTG_FP64: TTG_FP64, TTG_MIXED: TTG_MIXED}

_i64 = C.c_int64
_p64 = C.POINTER(C.c_int64)
_pd = C.POINTER(C.c_double)
_vp = C.c_void_p


class TTGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("libttgpu error %d: %s" % (code, msg))
        self.code = code


class AmenStep(C.Structure):
    """``ttg_amen_step``: the decisions of one local step of a sweep."""
    _fields_ = [("sweep", _i64), ("core", _i64), ("rank", _i64), ("iters", _i64),
                ("res_prev", C.c_double), ("res_new", C.c_double)]

    def to_dict(self):
        return dict(sweep=int(self.sweep), core=int(self.core), rank=int(self.rank),
                    iters=int(self.iters), res_prev=float(self.res_prev),
                    res_new=float(self.res_new))


class AmenOpts(C.Structure):
    _fields_ = [("nswp", _i64), ("rmax", _i64), ("max_full_size", _i64),
                ("local_restart", _i64), ("local_iters", _i64), ("kickrank", _i64),
                ("resid_damp", C.c_double), ("tol_exit", C.c_double),
                ("trunc_norm", C.c_int32), ("local_prec", C.c_int32),
                ("precision", C.c_int32), ("verb", C.c_int32), ("seed", C.c_uint64),
                ("timing", C.c_int32), ("reserved", C.c_int32),
                ("trace", C.POINTER(AmenStep)), ("trace_cap", _i64)]


MAX_SWEEPS = 64


class AmenStats(C.Structure):
    _fields_ = [("sweeps", _i64), ("matvecs", _i64), ("matvecs_fp64", _i64),
                ("local_solves", _i64), ("gmres_iters", _i64), ("max_rank", _i64),
                ("max_res", C.c_double * MAX_SWEEPS), ("max_dx", C.c_double * MAX_SWEEPS),
                ("ms_total", C.c_double), ("ms_matvec", C.c_double),
                ("matvec_gflop", C.c_double), ("launches", _i64), ("matvecs_lp", _i64),
                ("gflop_lp", C.c_double), ("ms_lp", C.c_double), ("gflop_fp64", C.c_double),
                ("ms_fp64", C.c_double), ("trace_len", _i64), ("gbyte_lp", C.c_double)]

    def to_dict(self):
        s = int(self.sweeps)
        k = min(s, MAX_SWEEPS)
        return dict(sweeps=s, matvecs=int(self.matvecs), matvecs_fp64=int(self.matvecs_fp64),
                    local_solves=int(self.local_solves), gmres_iters=int(self.gmres_iters),
                    max_rank=int(self.max_rank), max_res=list(self.max_res[:k]),
                    max_dx=list(self.max_dx[:k]), ms_total=float(self.ms_total),
                    matvec_gflop=float(self.matvec_gflop), launches=int(self.launches),
                    ms_matvec=float(self.ms_matvec), matvecs_lp=int(self.matvecs_lp),
                    gflop_lp=float(self.gflop_lp), ms_lp=float(self.ms_lp),
                    gflop_fp64=float(self.gflop_fp64), ms_fp64=float(self.ms_fp64),
                    trace_len=int(self.trace_len), gbyte_lp=float(self.gbyte_lp))


class GroupStats(C.Structure):
    _fields_ = [("flushes", _i64), ("launches", _i64), ("records", _i64),
                ("grouped_records", _i64), ("ms_plan", C.c_double),
                ("ms_issue_wait", C.c_double), ("ms_total", C.c_double),
                ("lanes_max", _i64), ("ms_record", C.c_double), ("allocs", _i64),
                ("device_mallocs", _i64), ("ms_alloc", C.c_double),
                ("ms_issue", C.c_double), ("tc_launches", _i64), ("tc_records", _i64),
                ("tc_gflop", C.c_double), ("tc_ms", C.c_double)]

    def to_dict(self):
        return {k: (float(getattr(self, k)) if t is C.c_double else int(getattr(self, k)))
                for k, t in self._fields_}


class AmenMvOpts(C.Structure):
    _fields_ = [("nswp", _i64), ("kickrank", _i64), ("init_qr", C.c_int32),
                ("verb", C.c_int32), ("seed", C.c_uint64), ("reserved", _i64 * 4)]


class AmenSumOpts(C.Structure):
    _fields_ = [("nswp", _i64), ("kickrank", _i64), ("init_qr", C.c_int32),
                ("verb", C.c_int32), ("seed", C.c_uint64), ("rmax", _i64),
                ("reserved", _i64 * 3)]


class RoundStats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_qr_sweep", C.c_double),
                ("ms_svd_sweep", C.c_double), ("max_rank", _i64), ("svd_fallbacks", _i64)]


_lib = None


def lib():
    """Load libttgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libttgpu.so not found at %s; run `python -m ttgpu.build` in "
                          "tt-toolbox_b200/" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    L.ttg_last_error.restype = C.c_char_p
    L.ttg_version.restype = C.c_int
    sigs = {
        "ttg_context_create": [C.c_int, C.POINTER(_vp)],
        "ttg_context_destroy": [_vp],
        "ttg_context_sync": [_vp],
        "ttg_malloc": [_vp, C.c_size_t, C.POINTER(_vp)],
        "ttg_free": [_vp, _vp],
        "ttg_memcpy_h2d": [_vp, _vp, _vp, C.c_size_t],
        "ttg_memcpy_d2h": [_vp, _vp, _vp, C.c_size_t],
        "ttg_memset": [_vp, _vp, C.c_int, C.c_size_t],
        "ttg_launch_count": [_vp, _p64],
        "ttg_tt_upload": [_vp, _i64, _p64, _p64, _p64, _pd, C.POINTER(_vp)],
        "ttg_tt_shape": [_vp, _p64, _p64, _p64, _p64, _p64],
        "ttg_tt_download": [_vp, _pd],
        "ttg_tt_free": [_vp],
        "ttg_round": [_vp, C.c_double, _p64, _i64, C.c_int32, C.POINTER(_vp),
                      C.POINTER(RoundStats)],
        "ttg_amen_solve": [_vp, _vp, C.c_double, C.POINTER(AmenOpts), _vp, _vp,
                           C.POINTER(_vp), C.POINTER(AmenStats)],
        "ttg_local_matvec": [_vp, _i64, _i64, _i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp,
                             C.c_int32],
        "ttg_next_phi": [_vp, C.c_int32, _i64, _i64, _i64, _i64, _i64, _i64, _i64, _vp, _vp,
                         _vp, _vp, _vp, _pd],
        "ttg_local_solve": [_vp, _i64, _i64, _i64, _i64, _i64, _vp, _vp, _vp, _vp, C.c_double,
                            C.c_int32, _vp, C.c_int32, _i64, _i64, _vp, C.c_int32, _p64],
    }
    sigs["ttg_local_matvec_noalloc"] = [_vp, _i64, _i64, _i64, _i64, _i64, _vp, _vp, _vp, _vp,
                                        _vp]
    sigs["ttg_dense_qr"] = [_vp, _i64, _i64, _vp, _vp, _vp]
    sigs["ttg_dense_svd"] = [_vp, _i64, _i64, _vp, _vp, _vp, _vp]
    sigs["ttg_grad_xAx"] = [_vp, _vp, _vp, _pd]
    sigs["ttg_tt_read_sdv"] = [_vp, C.c_char_p, C.POINTER(_vp)]
    sigs["ttg_tt_matvec"] = [_vp, _vp, C.POINTER(_vp)]
    sigs["ttg_amen_mv"] = [_vp, _vp, C.c_double, C.POINTER(AmenMvOpts), _vp, _vp,
                           C.POINTER(_vp), C.POINTER(_vp), _p64]
    sigs["ttg_tt_axpby"] = [C.c_double, _vp, C.c_double, _vp, C.POINTER(_vp)]
    sigs["ttg_tt_norm"] = [_vp, _pd]
    sigs["ttg_tt_dot"] = [_vp, _vp, _pd]
    sigs["ttg_tt_write_sdv"] = [_vp, C.c_char_p, C.c_int32]
    sigs["ttg_amen_solve_batch"] = [_vp, _i64, C.POINTER(_vp), C.POINTER(_vp), _pd,
                                    C.POINTER(AmenOpts), C.POINTER(_vp), C.POINTER(_vp),
                                    C.c_int32, C.POINTER(_vp), C.POINTER(AmenStats),
                                    C.POINTER(C.c_int32)]
    sigs["ttg_amen_solve_grouped"] = [_vp, _i64, C.POINTER(_vp), C.POINTER(_vp), _pd,
                                      C.POINTER(AmenOpts), C.POINTER(_vp), C.POINTER(_vp),
                                      C.c_int32, C.POINTER(_vp), C.POINTER(AmenStats),
                                      C.POINTER(C.c_int32), C.POINTER(GroupStats)]
    sigs["ttg_grad_xb"] = [_vp, _vp, _vp, _pd]
    sigs["ttg_grad_sampled"] = [_vp, _i64, _vp, _vp, _vp, _pd]
    sigs["ttg_context_set_option"] = [_vp, C.c_int32, _i64]
    sigs["ttg_amen_sum"] = [_i64, C.POINTER(_vp), _pd, _i64, C.c_double,
                            C.POINTER(AmenSumOpts), _vp, _vp, C.POINTER(_vp), C.POINTER(_vp),
                            _p64]
    sigs["ttg_selftest_wait"] = [_vp, C.c_int32]
    sigs["ttg_alstpz_solve"] = [_vp, _vp, C.c_double, C.POINTER(AmenOpts), _vp, C.POINTER(_vp),
                                C.POINTER(AmenStats)]
    for name, args in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.ttg_amen_sum_opts_default.argtypes = [C.POINTER(AmenSumOpts)]
    L.ttg_amen_sum_opts_default.restype = C.c_int
    L.ttg_amen_mv_opts_default.argtypes = [C.POINTER(AmenMvOpts)]
    L.ttg_amen_mv_opts_default.restype = C.c_int
    L.ttg_amen_opts_default.argtypes = [C.POINTER(AmenOpts)]
    L.ttg_amen_opts_default.restype = None
    L.ttg_alstpz_opts_default.argtypes = [C.POINTER(AmenOpts)]
    L.ttg_alstpz_opts_default.restype = None
    _lib = L
    return L


def _check(code):
    if code != 0:
        raise TTGError(code, lib().ttg_last_error().decode(errors="replace"))


def _i64arr(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int64))


def _ptr64(a):
    return a.ctypes.data_as(_p64)


def _ptrd(a):
    return a.ctypes.data_as(_pd)


# ---------------------------------------------------------------------------
# Host containers (flat-core layout of @tt_tensor/tt_tensor.m:33-41)
# ---------------------------------------------------------------------------

class TensorTrain:
    """Host TT tensor: mode sizes ``n[d]``, ranks ``r[d+1]``, flat column-major ``core``."""

    def __init__(self, n, r, core):
        self.n = _i64arr(n)
        self.r = _i64arr(r)
        self.core = np.ascontiguousarray(np.asarray(core, dtype=np.float64).ravel())
        need = int(np.sum(self.n * self.r[:-1] * self.r[1:]))
        if self.core.size != need or self.r.size != self.n.size + 1:
            raise ValueError("inconsistent TT sizes")

    @property
    def d(self):
        return int(self.n.size)

    @classmethod
    def from_cores(cls, cores):
        n = [c.shape[1] for c in cores]
        r = [cores[0].shape[0]] + [c.shape[2] for c in cores]
        return cls(n, r, np.concatenate([np.asarray(c).ravel(order="F") for c in cores]))

    def cores(self):
        out, pos = [], 0
        for k in range(self.d):
            sz = int(self.r[k] * self.n[k] * self.r[k + 1])
            out.append(self.core[pos:pos + sz].reshape(
                (int(self.r[k]), int(self.n[k]), int(self.r[k + 1])), order="F"))
            pos += sz
        return out


class TTMatrix:
    """Host TT matrix: row sizes ``n``, column sizes ``m``, ranks ``r``, flat core
    with cores ``[r_k, n_k, m_k, r_{k+1}]`` (``@tt_matrix/tt_matrix.m:33-40``)."""

    def __init__(self, n, m, r, core):
        self.n = _i64arr(n)
        self.m = _i64arr(m)
        self.r = _i64arr(r)
        self.core = np.ascontiguousarray(np.asarray(core, dtype=np.float64).ravel())
        need = int(np.sum(self.n * self.m * self.r[:-1] * self.r[1:]))
        if self.core.size != need:
            raise ValueError("inconsistent TT-matrix sizes")

    @property
    def d(self):
        return int(self.n.size)

    @classmethod
    def from_cores(cls, cores):
        n = [c.shape[1] for c in cores]
        m = [c.shape[2] for c in cores]
        r = [cores[0].shape[0]] + [c.shape[3] for c in cores]
        return cls(n, m, r, np.concatenate([np.asarray(c).ravel(order="F") for c in cores]))


# ---------------------------------------------------------------------------
# Device context / handles
# ---------------------------------------------------------------------------

class Context:
    """One device + one CUDA stream (``ttg_context``)."""

    def __init__(self, device=0):
        h = _vp()
        _check(lib().ttg_context_create(int(device), C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            lib().ttg_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        _check(lib().ttg_context_sync(self.h))

    # ttg_context_set_option keys
    OPT_JACOBI_MAX_SWEEPS = 1
    OPT_GROUP_SMS = 2

    def set_option(self, key, value):
        """``ttg_context_set_option`` (e.g. the Jacobi SVD sweep limit)."""
        _check(lib().ttg_context_set_option(self.h, int(key), int(value)))

    def selftest_wait(self, which):
        """``ttg_selftest_wait``: runs one bounded device wait on a condition
        that nothing satisfies; raises ``TTGError`` (code 6, TTG_ERR_TIMEOUT)
        when the wait gave up as designed."""
        _check(lib().ttg_selftest_wait(self.h, int(which)))

    def launch_count(self):
        v = _i64(0)
        _check(lib().ttg_launch_count(self.h, C.byref(v)))
        return v.value

    def flush_l2(self, nbytes=256 << 20):
        """Overwrite ``nbytes`` of device memory (larger than the 126 MB L2)."""
        if getattr(self, "_flush", None) is None or self._flush.n * 8 < nbytes:
            self._flush = DeviceArray(self, None, nbytes // 8)
        _check(lib().ttg_memset(self.h, self._flush.p, 0, self._flush.n * 8))

    # device memory helpers
    def to_device(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F")
                                 if np.asarray(a).ndim > 1 else np.asarray(a, dtype=np.float64))
        return DeviceArray(self, a)

    def empty(self, n):
        return DeviceArray(self, None, n)


class DeviceArray:
    """Flat FP64 device buffer owned by a context."""

    def __init__(self, ctx, host=None, n=None):
        self.ctx = ctx
        self.n = int(host.size if host is not None else n)
        p = _vp()
        _check(lib().ttg_malloc(ctx.h, max(self.n, 1) * 8, C.byref(p)))
        self.p = p
        if host is not None and self.n:
            _check(lib().ttg_memcpy_h2d(ctx.h, self.p, host.ctypes.data_as(_vp), self.n * 8))

    def get(self):
        out = np.empty(self.n, dtype=np.float64)
        if self.n:
            _check(lib().ttg_memcpy_d2h(self.ctx.h, out.ctypes.data_as(_vp), self.p, self.n * 8))
        return out

    def free(self):
        if self.p:
            lib().ttg_free(self.ctx.h, self.p)
            self.p = None

    def __del__(self):
        try:
            if self.ctx.h:
                self.free()
        except Exception:
            pass


class DeviceTT:
    """Device-resident TT tensor or matrix (``ttg_tt``)."""

    def __init__(self, ctx, h):
        self.ctx = ctx
        self.h = h

    @classmethod
    def upload(cls, ctx, t):
        h = _vp()
        n = _i64arr(t.n)
        r = _i64arr(t.r)
        core = np.ascontiguousarray(t.core, dtype=np.float64)
        if isinstance(t, TTMatrix):
            m = _i64arr(t.m)
            _check(lib().ttg_tt_upload(ctx.h, t.d, _ptr64(n), _ptr64(m), _ptr64(r), _ptrd(core),
                                       C.byref(h)))
        else:
            _check(lib().ttg_tt_upload(ctx.h, t.d, _ptr64(n), None, _ptr64(r), _ptrd(core),
                                       C.byref(h)))
        return cls(ctx, h)

    def shape(self):
        d = _i64()
        _check(lib().ttg_tt_shape(self.h, C.byref(d), None, None, None, None))
        d = d.value
        n = np.zeros(d, np.int64)
        m = np.zeros(d, np.int64)
        r = np.zeros(d + 1, np.int64)
        numel = _i64()
        _check(lib().ttg_tt_shape(self.h, None, _ptr64(n), _ptr64(m), _ptr64(r), C.byref(numel)))
        return n, m, r, numel.value

    def download(self):
        n, m, r, numel = self.shape()
        core = np.empty(numel, np.float64)
        _check(lib().ttg_tt_download(self.h, _ptrd(core)))
        return TensorTrain(n, r, core)

    def free(self):
        if self.h:
            lib().ttg_tt_free(self.h)
            self.h = None

    def __del__(self):
        try:
            if self.ctx.h:
                self.free()
        except Exception:
            pass


_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(int(os.environ.get("TTG_DEVICE", "0")))
    return _default_ctx


# ---------------------------------------------------------------------------
# Reference-facing operations
# ---------------------------------------------------------------------------

def round(tt, eps, rmax=None, precision="fp64", ctx=None, stats=None):
    """``tt = round(tt, eps[, rmax])`` (``@tt_tensor/round.m:1-110``).

    ``tt`` is a host ``TensorTrain`` or a ``DeviceTT``; the result has the same
    kind.  ``rmax``: scalar or ``d+1`` values (``round.m:20-32``).
    """
    ctx = ctx or (tt.ctx if isinstance(tt, DeviceTT) else default_context())
    dev_in = tt if isinstance(tt, DeviceTT) else DeviceTT.upload(ctx, tt)
    if rmax is None:
        rp, nr = None, 0
    else:
        rm = _i64arr(np.atleast_1d(rmax))
        rp, nr = _ptr64(rm), rm.size
    out = _vp()
    st = RoundStats()
    _check(lib().ttg_round(dev_in.h, float(eps), rp, nr, _PREC[precision], C.byref(out),
                           C.byref(st)))
    res = DeviceTT(ctx, out)
    if stats is not None:
        stats.update(ms_total=st.ms_total, ms_qr_sweep=st.ms_qr_sweep,
                     ms_svd_sweep=st.ms_svd_sweep, max_rank=int(st.max_rank),
                     svd_fallbacks=int(st.svd_fallbacks))
    if isinstance(tt, DeviceTT):
        return res
    host = res.download()
    res.free()
    dev_in.free()
    return host


# local_prec names -> MEX prec codes (solve/amen_solve2.m:205-207).
_LOCAL_PREC = {"": 0, None: 0, 0: 0, "cjacobi": 1, 1: 1, "ljacobi": 2, 2: 2, "rjacobi": 3, 3: 3}

_AMEN_KEYS = {"nswp", "rmax", "x0", "z0", "verb", "local_prec", "local_restart", "local_iters",
              "kickrank", "kicktype", "ismex", "max_full_size", "resid_damp", "trunc_norm",
              "tol_exit", "precision", "seed", "timing"}


def _check_amen_opts(opts):
    for k in opts:
        if k.lower() not in _AMEN_KEYS:
            raise ValueError("Unrecognized option: %s" % k)
    opts = {k.lower(): v for k, v in opts.items()}
    if opts.get("kicktype", "als") != "als":
        raise TTGError(7, "kicktype %r is not implemented (only 'als')" % opts["kicktype"])
    if opts.get("trunc_norm", "residual") not in ("residual", "resid", 1):
        raise TTGError(7, "trunc_norm %r is not implemented (only 'residual')" % opts["trunc_norm"])
    lp = opts.get("local_prec", "")
    if lp not in _LOCAL_PREC:
        raise TTGError(7, "local_prec %r is unknown ('', 'cjacobi', 'ljacobi', 'rjacobi')"
                       % (lp,))
    return opts


def _amen_opts(opts):
    """``ttg_amen_opts`` from checked name/value options (defaults of
    ``amen_solve2.m:75-107`` for the rest)."""
    o = AmenOpts()
    lib().ttg_amen_opts_default(C.byref(o))
    for k in ("nswp", "rmax", "max_full_size", "local_restart", "local_iters", "kickrank"):
        if k in opts:
            setattr(o, k, int(opts[k]))
    if "resid_damp" in opts:
        o.resid_damp = float(opts["resid_damp"])
    if "tol_exit" in opts and opts["tol_exit"] is not None:
        o.tol_exit = float(opts["tol_exit"])
    if "verb" in opts:
        o.verb = int(opts["verb"])
    if "seed" in opts:
        o.seed = int(opts["seed"])
    if "timing" in opts:
        o.timing = 1 if opts["timing"] else 0
    o.local_prec = _LOCAL_PREC[opts.get("local_prec", "")]
    o.precision = _PREC[opts.get("precision", "fp64")]
    return o


def amen_solve2(A, y, tol, ctx=None, stats=None, trace=None, **opts):
    """``[x] = amen_solve2(A, y, tol, 'name', value, ...)`` (``solve/amen_solve2.m:1``).

    Options follow ``amen_solve2.m:161-203``; unknown names raise
    ``ValueError('Unrecognized option')`` as the reference errors (``:200-201``).
    ``A``: host ``TTMatrix`` or ``DeviceTT``; ``y``/``x0``/``z0``: host
    ``TensorTrain`` or ``DeviceTT``.  Returns a host ``TensorTrain`` when ``y``
    is a host tensor, else a ``DeviceTT``.  ``trace``: optional list that
    receives one dict per local step (``ttg_amen_step``: sweep, core, kept
    rank, Krylov steps, local residuals before and after).
    """
    opts = _check_amen_opts(opts)
    ctx = ctx or (A.ctx if isinstance(A, DeviceTT) else default_context())
    o = _amen_opts(opts)
    trace_buf = None
    if trace is not None:
        d = A.shape()[0].size if isinstance(A, DeviceTT) else len(A.n)
        cap = int(o.nswp) * d
        trace_buf = (AmenStep * max(cap, 1))()
        o.trace = C.cast(trace_buf, C.POINTER(AmenStep))
        o.trace_cap = cap
    owned = []

    def dev(t):
        if t is None or isinstance(t, DeviceTT):
            return t
        h = DeviceTT.upload(ctx, t)
        owned.append(h)
        return h

    dA, dy = dev(A), dev(y)
    dx0, dz0 = dev(opts.get("x0")), dev(opts.get("z0"))
    out = _vp()
    st = AmenStats()
    try:
        _check(lib().ttg_amen_solve(dA.h, dy.h, float(tol), C.byref(o),
                                    dx0.h if dx0 is not None else None,
                                    dz0.h if dz0 is not None else None, C.byref(out),
                                    C.byref(st)))
    finally:
        pass
    if stats is not None:
        stats.update(st.to_dict())
    if trace is not None:
        trace.extend(trace_buf[k].to_dict() for k in range(min(int(st.trace_len), o.trace_cap)))
    res = DeviceTT(ctx, out)
    if isinstance(y, DeviceTT):
        for h in owned:
            h.free()
        return res
    host = res.download()
    res.free()
    for h in owned:
        h.free()
    return host


_ALSTPZ_KEYS = {"x0", "nswp", "max_full_size", "local_prec", "local_iters", "local_restart",
                "kickrank", "kicktype", "ismex", "resid_damp", "symm", "verb", "precision",
                "seed"}


def alstpz_solve(A, y, tol, ctx=None, stats=None, **opts):
    """``[x] = alstpz_solve(A, y, tol, 'name', value, ...)``
    (``solve/alstpz_solve.m:1``, ALS(t+z), kicktype ``'svd'``).

    Options follow ``alstpz_solve.m:55-104`` (defaults nswp 10,
    max_full_size 50, kickrank 4, local_restart 40, local_iters 2,
    resid_damp 2); ``kicktype 'als'`` and ``symm`` are not implemented and
    raise ``TTGError``; ``ismex`` is accepted (the device local solver is
    the MEX one).  ``precision`` 'fp64' or 'mixed' for the local solves.
    ``stats`` (dict, optional) receives sweeps, per-sweep ``max_res`` and
    ``max_dx``, local solves, Krylov steps, max rank."""
    for k in opts:
        if k.lower() not in _ALSTPZ_KEYS:
            raise ValueError("Unrecognized option: %s" % k)
    opts = {k.lower(): v for k, v in opts.items()}
    if opts.get("kicktype", "svd") != "svd":
        raise TTGError(7, "kicktype %r is not implemented (only 'svd')" % opts["kicktype"])
    if opts.get("symm", False):
        raise TTGError(7, "symm is not implemented")
    lp = opts.get("local_prec", "")
    if lp not in _LOCAL_PREC:
        raise TTGError(7, "local_prec %r is unknown ('', 'cjacobi', 'ljacobi', 'rjacobi')"
                       % (lp,))
    ctx = ctx or (A.ctx if isinstance(A, DeviceTT) else default_context())
    o = AmenOpts()
    lib().ttg_alstpz_opts_default(C.byref(o))
    for k in ("nswp", "max_full_size", "local_restart", "local_iters", "kickrank"):
        if k in opts:
            setattr(o, k, int(opts[k]))
    if "resid_damp" in opts:
        o.resid_damp = float(opts["resid_damp"])
    if "verb" in opts:
        o.verb = int(opts["verb"])
    if "seed" in opts:
        o.seed = int(opts["seed"])
    o.local_prec = _LOCAL_PREC[lp]
    o.precision = _PREC[opts.get("precision", "fp64")]
    owned = []

    def dev(t):
        if t is None or isinstance(t, DeviceTT):
            return t
        h = DeviceTT.upload(ctx, t)
        owned.append(h)
        return h

    try:
        dA, dy, dx0 = dev(A), dev(y), dev(opts.get("x0"))
        out = _vp()
        st = AmenStats()
        _check(lib().ttg_alstpz_solve(dA.h, dy.h, float(tol), C.byref(o),
                                      dx0.h if dx0 is not None else None, C.byref(out),
                                      C.byref(st)))
        if stats is not None:
            stats.update(st.to_dict())
        res = DeviceTT(ctx, out)
        if isinstance(y, DeviceTT):
            return res
        host = res.download()
        res.free()
        return host
    finally:
        for h in owned:
            h.free()


def amen_solve2_batch(As, ys, tol, x0s=None, z0s=None, workers=0, ctx=None, stats=None,
                      per_system=None, grouped=False, group_stats=None, **opts):
    """Batched ``amen_solve2`` (``ttg_amen_solve_batch``): solves
    ``As[i] x = ys[i]`` for every i, concurrently on one device.

    ``grouped=True`` runs the grouped batch (``ttg_amen_solve_grouped``):
    ``workers`` is then the number of systems in flight (0: all), and
    ``group_stats`` (optional dict) receives the executor's counters.

    ``tol``: scalar or one per system; ``opts``: options shared by all
    systems; ``per_system``: optional list of option dicts merged over
    ``opts`` for each system (e.g. its own ``rmax``).  ``x0s``/``z0s``:
    optional lists (entries may be None).  Returns a list of host
    ``TensorTrain`` (``DeviceTT`` when the ys are device handles).  ``stats``:
    optional list filled with one dict per system.  Raises ``TTGError`` for
    the first failing system after all systems ran."""
    count = len(As)
    if len(ys) != count:
        raise ValueError("As and ys differ in length")
    ctx = ctx or (As[0].ctx if count and isinstance(As[0], DeviceTT) else default_context())
    base = _check_amen_opts(opts)
    for k in ("x0", "z0"):
        if k in base:
            raise ValueError("pass initial guesses as x0s / z0s")
    olist = (AmenOpts * max(count, 1))()
    for i in range(count):
        oi = dict(base)
        if per_system is not None and per_system[i]:
            oi.update(_check_amen_opts(per_system[i]))
        olist[i] = _amen_opts(oi)
    tols = np.ascontiguousarray(np.broadcast_to(np.asarray(tol, np.float64), (count,)))
    owned = []

    def dev(t):
        if t is None or isinstance(t, DeviceTT):
            return t
        h = DeviceTT.upload(ctx, t)
        owned.append(h)
        return h

    HA = (_vp * max(count, 1))()
    HY = (_vp * max(count, 1))()
    HX0 = (_vp * max(count, 1))()
    HZ0 = (_vp * max(count, 1))()
    for i in range(count):
        HA[i] = dev(As[i]).h
        HY[i] = dev(ys[i]).h
        HX0[i] = dev(x0s[i]).h if x0s is not None and x0s[i] is not None else None
        HZ0[i] = dev(z0s[i]).h if z0s is not None and z0s[i] is not None else None
    out = (_vp * max(count, 1))()
    st = (AmenStats * max(count, 1))()
    status = (C.c_int32 * max(count, 1))()
    try:
        if grouped:
            gs = GroupStats()
            code = lib().ttg_amen_solve_grouped(ctx.h, count, HA, HY, _ptrd(tols), olist,
                                                HX0 if x0s is not None else None,
                                                HZ0 if z0s is not None else None, int(workers),
                                                out, st, status, C.byref(gs))
            if group_stats is not None:
                group_stats.clear()
                group_stats.update(gs.to_dict())
        else:
            code = lib().ttg_amen_solve_batch(ctx.h, count, HA, HY, _ptrd(tols), olist,
                                              HX0 if x0s is not None else None,
                                              HZ0 if z0s is not None else None, int(workers),
                                              out, st, status)
        msg = lib().ttg_last_error().decode(errors="replace") if code else ""
        res = []
        for i in range(count):
            h = DeviceTT(ctx, out[i]) if out[i] else None
            if h is not None and not (count and isinstance(ys[0], DeviceTT)):
                t = h.download()
                h.free()
                h = t
            res.append(h)
        if stats is not None:
            stats[:] = [dict(st[i].to_dict(), status=int(status[i])) for i in range(count)]
        if code:
            raise TTGError(code, msg)
        return res
    finally:
        for h in owned:
            h.free()


def _shape3(a):
    a = np.asarray(a)
    s = list(a.shape) + [1] * (3 - a.ndim)
    return s[:3]


def bfun3(Phi1, A, Phi2, x, ctx=None, precision="fp64"):
    """Local matvec ``y = bfun3(Phi1, A, Phi2, x)`` (square: ry = rx)."""
    ctx = ctx or default_context()
    rx1, _, ra1 = _shape3(Phi1)
    A4 = np.asarray(A)
    A4 = A4.reshape(list(A4.shape) + [1] * (4 - A4.ndim), order="F")
    n = A4.shape[1]
    rx2, ra2, _ = _shape3(Phi2)
    dP1, dA, dP2 = ctx.to_device(Phi1), ctx.to_device(A4), ctx.to_device(Phi2)
    dx = ctx.to_device(np.asarray(x).ravel(order="F"))
    dy = ctx.empty(rx1 * n * rx2)
    _check(lib().ttg_local_matvec(ctx.h, rx1, n, rx2, ra1, ra2, dP1.p, dA.p, dP2.p, dx.p, dy.p,
                                  _PREC[precision]))
    return dy.get()


def compute_next_Phi(Phi_prev, x, A, y, direction, extnrm=None, want_norm=False, ctx=None):
    """``[Phi, nrm] = compute_next_Phi(Phi_prev, x, A, y, direction[, extnrm])``."""
    ctx = ctx or default_context()
    x = np.asarray(x)
    y = np.asarray(y)
    rx1, n, rx2 = _shape3(x)
    ry1, _, ry2 = _shape3(y)
    if A is not None:
        A4 = np.asarray(A)
        A4 = A4.reshape(list(A4.shape) + [1] * (4 - A4.ndim), order="F")
        ra1, ra2 = A4.shape[0], A4.shape[3]
        dA = ctx.to_device(A4)
        Ap = dA.p
    else:
        ra1 = ra2 = 1
        Ap = None
    d = 0 if direction == "lr" else 1
    cnt = rx2 * ry2 * ra2 if d == 0 else ry1 * ra1 * rx1
    dP, dx, dy = ctx.to_device(Phi_prev), ctx.to_device(x), ctx.to_device(y)
    out = ctx.empty(cnt)
    nrm = C.c_double(0.0)
    _check(lib().ttg_next_phi(ctx.h, d, rx1, n, rx2, ry1, ry2, ra1, ra2, dP.p, dx.p, Ap, dy.p,
                              out.p, C.byref(nrm) if want_norm else None))
    res = out.get()
    if extnrm is not None and not want_norm:
        res = res / extnrm
    if d == 0:
        shape = (rx2, ry2, ra2) if A is not None else (rx2, ry2)
    else:
        shape = (ry1, ra1, rx1) if A is not None else (ry1, rx1)
    res = res.reshape(shape, order="F")
    return (res, nrm.value) if want_norm else res


def solve3d_2(Phi1, A, Phi2, rhs, tol, trunc_norm, sol_prev, prec=0, nrestart=40, niters=2,
              verb=0, ctx=None, precision="fp64", info=None):
    """MEX-compatible local solve (``fmex/solve3d_2.c:121-300``); residual branch."""
    ctx = ctx or default_context()
    rx1, rx1b, ra1 = _shape3(Phi1)
    if rx1b != rx1:
        raise TTGError(1, "Phi1 is not square!")            # solve3d_2.c:150
    A4 = np.asarray(A)
    A4 = A4.reshape(list(A4.shape) + [1] * (4 - A4.ndim), order="F")
    if A4.shape[0] != ra1:
        raise TTGError(1, "ra1 in Phi1 and A are not consistent!")   # :158
    n = A4.shape[1]
    if A4.shape[2] != n:
        raise TTGError(1, "A is not square!")               # :160
    ra2 = A4.shape[3]
    rx2, ra2b, rx2b = _shape3(Phi2)
    if rx2b != rx2:
        raise TTGError(1, "Phi2 is not square!")            # :169
    if ra2b != ra2:
        raise TTGError(1, "ra2 in Phi2 and A are not consistent!")   # :170
    sz = rx1 * n * rx2
    if np.asarray(rhs).size != sz:
        raise TTGError(1, "RHS size is not consistent!")    # :173
    if np.asarray(sol_prev).size != sz:
        raise TTGError(1, "SOL_PREV size is not consistent!")  # :182
    dP1, dA, dP2 = ctx.to_device(Phi1), ctx.to_device(A4), ctx.to_device(Phi2)
    dr = ctx.to_device(np.asarray(rhs, dtype=np.float64).ravel(order="F"))
    ds = ctx.to_device(np.asarray(sol_prev, dtype=np.float64).ravel(order="F"))
    out = ctx.empty(sz)
    it = _i64(0)
    _check(lib().ttg_local_solve(ctx.h, rx1, n, rx2, ra1, ra2, dP1.p, dA.p, dP2.p, dr.p,
                                 float(tol), int(round_half(trunc_norm)), ds.p, int(prec),
                                 int(nrestart), int(niters), out.p, _PREC[precision],
                                 C.byref(it)))
    if info is not None:
        info["iters"] = it.value
    return out.get()


def dense_qr(A, ctx=None):
    """Thin QR of a host matrix on the device: ``(Q, R)`` (as ``qr(A, 0)``)."""
    ctx = ctx or default_context()
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    k = min(m, n)
    dA, dQ, dR = ctx.to_device(A), ctx.empty(m * k), ctx.empty(k * n)
    _check(lib().ttg_dense_qr(ctx.h, m, n, dA.p, dQ.p, dR.p))
    return dQ.get().reshape(m, k, order="F"), dR.get().reshape(k, n, order="F")


def dense_svd(A, ctx=None):
    """Economy SVD of a host matrix on the device: ``(U, s, VT)`` (as ``svd(A,'econ')``)."""
    ctx = ctx or default_context()
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    k = min(m, n)
    dA, dU, dS, dV = ctx.to_device(A), ctx.empty(m * k), ctx.empty(k), ctx.empty(k * n)
    _check(lib().ttg_dense_svd(ctx.h, m, n, dA.p, dU.p, dS.p, dV.p))
    return (dU.get().reshape(m, k, order="F"), dS.get(), dV.get().reshape(k, n, order="F"))


def round_half(v):
    """MATLAB's ``round`` of a scalar option (``solve3d_2.c:138-141,179``)."""
    return int(np.floor(float(v) + 0.5))


# ---------------------------------------------------------------------------
# Gradients with respect to every core (no reference counterpart; the forward
# maps are @tt_matrix/mtimes.m:38-65, @tt_tensor/dot.m:92-111 and the element
# path of @tt_tensor/subsref.m:93-123)
# ---------------------------------------------------------------------------

def _grad_call(fn, x, other, ctx, *extra, out=None):
    """Run one gradient entry.  With ``out`` (a ``DeviceArray`` of numel(x)
    doubles) the gradient stays on the device and ``(f, out)`` is returned;
    otherwise ``(f, TensorTrain)`` with the gradient downloaded."""
    ctx = ctx or (x.ctx if isinstance(x, DeviceTT) else default_context())
    owned = []

    def dev(t):
        if t is None or isinstance(t, DeviceTT):
            return t
        h = DeviceTT.upload(ctx, t)
        owned.append(h)
        return h
    dx, do = dev(x), dev(other)
    n, m, r, numel = dx.shape()
    g = out if out is not None else ctx.empty(numel)
    if g.n < numel:
        raise ValueError("out holds %d doubles, the gradient needs %d" % (g.n, numel))
    val = C.c_double(0.0)
    try:
        if do is None:
            _check(fn(dx.h, *extra, g.p, C.byref(val)))
        else:
            _check(fn(dx.h, do.h, g.p, C.byref(val)))
        if out is not None:
            return val.value, out
        return val.value, TensorTrain(n, r, g.get())
    finally:
        if out is None:
            g.free()
        for h in owned:
            h.free()


def grad_xAx(x, A, ctx=None, out=None):
    """``(f, G)`` with ``f = <x, A x>`` and ``G`` the gradient with respect to
    every core of ``x`` (a ``TensorTrain`` with x's shapes, or ``out``)."""
    return _grad_call(lib().ttg_grad_xAx, x, A, ctx, out=out)


def grad_xb(x, b, ctx=None, out=None):
    """``(f, G)`` with ``f = <x, b>``."""
    return _grad_call(lib().ttg_grad_xb, x, b, ctx, out=out)


class SampleSet:
    """Device-resident samples for ``grad_sampled``: ``idx`` [S, d] 0-based
    multi-indices (stored column-major int32) and values ``y`` [S]."""

    def __init__(self, ctx, idx, y):
        idx = np.asarray(idx)
        if idx.ndim != 2:
            raise ValueError("idx must be [S, d]")
        self.ctx = ctx
        self.S, self.d = idx.shape
        col = np.asfortranarray(idx.astype(np.int32, copy=False))
        yv = np.ascontiguousarray(np.asarray(y, dtype=np.float64).ravel())
        if yv.size != self.S:
            raise ValueError("y must have one value per sample")
        self.idx = DeviceArray(ctx, None, max(1, (self.S * self.d + 1) // 2))
        if self.S:
            _check(lib().ttg_memcpy_h2d(ctx.h, self.idx.p, col.ctypes.data_as(_vp), col.nbytes))
        self.y = DeviceArray(ctx, yv) if self.S else DeviceArray(ctx, None, 1)

    def free(self):
        self.idx.free()
        self.y.free()


def grad_sampled(x, idx, y=None, ctx=None, out=None):
    """``(f, G)`` with ``f = sum_s (X[idx[s]] - y[s])^2``.

    ``idx``: integer array ``[S, d]`` of 0-based multi-indices with ``y``
    ``[S]``, or a ``SampleSet`` already on the device (``y`` omitted)."""
    ctx = ctx or (x.ctx if isinstance(x, DeviceTT) else default_context())
    own = not isinstance(idx, SampleSet)
    ss = SampleSet(ctx, idx, y) if own else idx
    d = x.d if not isinstance(x, DeviceTT) else len(x.shape()[0])
    if ss.S and ss.d != d:
        if own:
            ss.free()
        raise ValueError("idx must be [S, d] with d = %d" % d)
    try:
        return _grad_call(lib().ttg_grad_sampled, x, None, ctx, ss.S, ss.idx.p, ss.y.p,
                          out=out)
    finally:
        if own:
            ss.free()


# ---------------------------------------------------------------------------
# SDV TT files (fmex/tt_read.c, fmex/tt_write.c)
# ---------------------------------------------------------------------------

def read_sdv(path, ctx=None, device=False):
    """``tt_tensor(filename)``: a host ``TensorTrain`` (``DeviceTT`` with
    ``device=True``) read from a SDV file."""
    ctx = ctx or default_context()
    h = _vp()
    _check(lib().ttg_tt_read_sdv(ctx.h, os.fsencode(path), C.byref(h)))
    t = DeviceTT(ctx, h)
    if device:
        return t
    host = t.download()
    t.free()
    return host


def write_sdv(path, tt, precision="double", ctx=None):
    """Write a TT tensor or matrix (host or device) as a SDV file;
    ``precision`` 'double' or 'float'."""
    ctx = ctx or (tt.ctx if isinstance(tt, DeviceTT) else default_context())
    prec = {"double": 0, "float": 1}[precision]
    dev = tt if isinstance(tt, DeviceTT) else DeviceTT.upload(ctx, tt)
    try:
        _check(lib().ttg_tt_write_sdv(dev.h, os.fsencode(path), prec))
    finally:
        if dev is not tt:
            dev.free()


def as_matrix(tt, n, m):
    """Reinterpret a TT tensor whose mode sizes are n_k m_k as a TT matrix
    (row index fastest), as ``tt_matrix(tt, n, m)``."""
    n = np.asarray(n, np.int64)
    m = np.asarray(m, np.int64)
    if not np.array_equal(np.asarray(tt.n, np.int64), n * m):
        raise ValueError("mode sizes are not n .* m")
    return TTMatrix(n, m, tt.r, tt.core)


# ---------------------------------------------------------------------------
# TT algebra on the device (@tt_matrix/mtimes.m, @tt_tensor/plus.m,
# @tt_tensor/norm.m, @tt_tensor/dot.m)
# ---------------------------------------------------------------------------

def _dev_args(ctx, *ts):
    owned, hs = [], []
    for t in ts:
        if isinstance(t, DeviceTT):
            hs.append(t)
        else:
            h = DeviceTT.upload(ctx, t)
            owned.append(h)
            hs.append(h)
    return owned, hs


def _ctx_of(ctx, *ts):
    for t in ts:
        if isinstance(t, DeviceTT):
            return ctx or t.ctx
    return ctx or default_context()


def _result(ctx, h, device):
    t = DeviceTT(ctx, h)
    if device:
        return t
    host = t.download()
    t.free()
    return host


def tt_matvec(A, x, ctx=None):
    """``A * x`` exactly (ranks multiply); a ``DeviceTT`` when ``x`` is one."""
    ctx = _ctx_of(ctx, A, x)
    owned, (dA, dx) = _dev_args(ctx, A, x)
    try:
        h = _vp()
        _check(lib().ttg_tt_matvec(dA.h, dx.h, C.byref(h)))
        return _result(ctx, h, isinstance(x, DeviceTT))
    finally:
        for t in owned:
            t.free()


def tt_axpby(a, x, b, y, ctx=None):
    """``a*x + b*y`` (ranks add); a ``DeviceTT`` when ``x`` is one."""
    ctx = _ctx_of(ctx, x, y)
    owned, (dx, dy) = _dev_args(ctx, x, y)
    try:
        h = _vp()
        _check(lib().ttg_tt_axpby(float(a), dx.h, float(b), dy.h, C.byref(h)))
        return _result(ctx, h, isinstance(x, DeviceTT))
    finally:
        for t in owned:
            t.free()


def tt_norm(x, ctx=None):
    """``norm(x)`` by the QR sweep of ``@tt_tensor/norm.m``."""
    ctx = _ctx_of(ctx, x)
    owned, (dx,) = _dev_args(ctx, x)
    try:
        v = C.c_double(0.0)
        _check(lib().ttg_tt_norm(dx.h, C.byref(v)))
        return v.value
    finally:
        for t in owned:
            t.free()


def tt_dot(x, y, ctx=None):
    """``dot(x, y)``."""
    ctx = _ctx_of(ctx, x, y)
    owned, (dx, dy) = _dev_args(ctx, x, y)
    try:
        v = C.c_double(0.0)
        _check(lib().ttg_tt_dot(dx.h, dy.h, C.byref(v)))
        return v.value
    finally:
        for t in owned:
            t.free()


def true_residual(A, x, y, ctx=None):
    """``norm(A*x - y) / norm(y)`` on the device."""
    ctx = _ctx_of(ctx, A, x, y)
    owned, (dA, dx, dy) = _dev_args(ctx, A, x, y)
    ax = r = None
    try:
        ax = tt_matvec(dA, dx, ctx)
        r = tt_axpby(1.0, ax, -1.0, dy, ctx)
        return tt_norm(r, ctx) / tt_norm(dy, ctx)
    finally:
        for t in owned + [ax, r]:
            if t is not None:
                t.free()


def amen_mv(A, x, tol, y0=None, z0=None, ctx=None, nswp=20, kickrank=4, init_qr=True, verb=0,
            seed=None):
    """``[y, z] = amen_mv(A, x, tol, 'y0', y0, 'z0', z0, ...)``
    (``core/amen_mv.m``): returns ``(y, z, sweeps)``, host TTs unless ``x``
    is a ``DeviceTT`` (``z`` is None when ``kickrank`` is 0)."""
    ctx = _ctx_of(ctx, A, x)
    o = AmenMvOpts()
    lib().ttg_amen_mv_opts_default(C.byref(o))
    o.nswp, o.kickrank, o.init_qr, o.verb = int(nswp), int(kickrank), int(bool(init_qr)), int(verb)
    if seed is not None:
        o.seed = int(seed)
    owned, hs = _dev_args(ctx, *[t for t in (A, x, y0, z0) if t is not None])
    it = iter(hs)
    dA, dx = next(it), next(it)
    dy0 = next(it) if y0 is not None else None
    dz0 = next(it) if z0 is not None else None
    yh, zh, sw = _vp(), _vp(), _i64(0)
    try:
        _check(lib().ttg_amen_mv(dA.h, dx.h, float(tol), C.byref(o),
                                 dy0.h if dy0 is not None else None,
                                 dz0.h if dz0 is not None else None,
                                 C.byref(yh), C.byref(zh), C.byref(sw)))
        dev = isinstance(x, DeviceTT)
        y = _result(ctx, yh, dev)
        z = _result(ctx, zh, dev) if zh.value else None
        return y, z, sw.value
    finally:
        for t in owned:
            t.free()


def amen_sum(X, c, tol, y0=None, z0=None, ctx=None, nswp=20, kickrank=4, init_qr=True, rmax=None,
             verb=0, seed=None):
    """``[y, z] = amen_sum(X, c, tol, 'y0', y0, 'z0', z0, ...)``
    (``core/amen_sum.m``): ``y(:, m) ~ sum_j X[j] c[j, m]``.  ``X``: list of
    TT tensors (host or ``DeviceTT``); ``c``: ``len(X)`` coefficients or a
    ``len(X) x M`` array.  Returns ``(y, z, sweeps)``: host TTs unless
    ``X[0]`` is a ``DeviceTT``; ``y`` has last rank ``M``; ``z`` is None
    when ``kickrank`` is 0."""
    coef = np.asarray(c, dtype=np.float64)
    if coef.ndim == 1:
        coef = coef[:, None]
    N, M = coef.shape
    if len(X) != N:
        raise ValueError("c must have len(X) rows")
    ctx = _ctx_of(ctx, *X)
    o = AmenSumOpts()
    lib().ttg_amen_sum_opts_default(C.byref(o))
    o.nswp, o.kickrank, o.init_qr, o.verb = int(nswp), int(kickrank), int(bool(init_qr)), int(verb)
    if rmax is not None and np.isfinite(rmax):
        o.rmax = int(rmax)
    if seed is not None:
        o.seed = int(seed)
    owned, hs = _dev_args(ctx, *(list(X) + [t for t in (y0, z0) if t is not None]))
    dX = hs[:N]
    rest = iter(hs[N:])
    dy0 = next(rest) if y0 is not None else None
    dz0 = next(rest) if z0 is not None else None
    HX = (_vp * N)(*[h.h for h in dX])
    cf = np.asfortranarray(coef).ravel(order="F").copy()
    yh, zh, sw = _vp(), _vp(), _i64(0)
    try:
        _check(lib().ttg_amen_sum(N, HX, _ptrd(cf), M, float(tol), C.byref(o),
                                  dy0.h if dy0 is not None else None,
                                  dz0.h if dz0 is not None else None,
                                  C.byref(yh), C.byref(zh), C.byref(sw)))
        dev = isinstance(X[0], DeviceTT)
        y = _result(ctx, yh, dev)
        z = _result(ctx, zh, dev) if zh.value else None
        return y, z, sw.value
    finally:
        for t in owned:
            t.free()
