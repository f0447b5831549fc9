"""TT data model and the caller-side TT algebra used by the oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Layout (``@tt_tensor/tt_tensor.m:33-41``, ``@tt_tensor/core2cell.m:9-11``):
a TT tensor is ``d``, mode sizes ``n[d]``, ranks ``r[d+1]`` and ONE flat
column-major core vector; core ``k`` occupies ``core[ps[k]:ps[k+1]]`` and is
reshaped column-major to ``[r[k], n[k], r[k+1]]``.  A TT matrix
(``@tt_matrix/tt_matrix.m:33-40``, ``@tt_matrix/core2cell.m:9-11``) stores core
``k`` as ``[r[k], n[k], m[k], r[k+1]]`` (row index faster than column index).

Here cores are held as a list of Fortran-ordered numpy arrays; ``flat()``
produces the reference's flat vector.
"""
import numpy as np


def rs(a, *shape):
    """Column-major reshape (MATLAB ``reshape``)."""
    return np.reshape(a, shape, order="F")


class TT:
    """TT tensor: list of cores ``[r_k, n_k, r_{k+1}]`` (column-major)."""

    def __init__(self, cores):
        self.cores = [np.asfortranarray(np.asarray(c, dtype=np.float64)) for c in cores]
        for c in self.cores:
            assert c.ndim == 3

    @property
    def d(self):
        return len(self.cores)

    @property
    def n(self):
        return np.array([c.shape[1] for c in self.cores], dtype=np.int64)

    @property
    def r(self):
        return np.array([self.cores[0].shape[0]] + [c.shape[2] for c in self.cores], dtype=np.int64)

    @property
    def ps(self):
        """0-based offsets; the reference's ``ps`` minus one (``tt_tensor.m:161``)."""
        n, r = self.n, self.r
        return np.concatenate([[0], np.cumsum(n * r[:-1] * r[1:])]).astype(np.int64)

    def flat(self):
        return np.concatenate([c.ravel(order="F") for c in self.cores])

    @staticmethod
    def from_flat(n, r, core):
        n = np.asarray(n, dtype=np.int64)
        r = np.asarray(r, dtype=np.int64)
        core = np.asarray(core, dtype=np.float64).ravel()
        cores, pos = [], 0
        for k in range(len(n)):
            sz = int(r[k] * n[k] * r[k + 1])
            cores.append(rs(core[pos:pos + sz], int(r[k]), int(n[k]), int(r[k + 1])))
            pos += sz
        assert pos == core.size
        return TT(cores)

    def copy(self):
        return TT([c.copy(order="F") for c in self.cores])

    def full(self):
        """Full array, column-major index order (``@tt_tensor/full.m:19-35``)."""
        res = self.cores[0].reshape(self.cores[0].shape[0] * self.cores[0].shape[1],
                                    self.cores[0].shape[2], order="F")
        for c in self.cores[1:]:
            r1 = c.shape[0]
            res = res @ rs(c, r1, -1)
            res = rs(res, -1, c.shape[2])
        return rs(res, *[int(v) for v in self.n])

    def __mul__(self, a):
        cores = [c.copy(order="F") for c in self.cores]
        cores[0] = cores[0] * a
        return TT(cores)

    __rmul__ = __mul__

    def __add__(self, other):
        return tt_plus(self, other)

    def __sub__(self, other):
        return tt_plus(self, other * (-1.0))


class TTMatrix:
    """TT matrix: list of cores ``[r_k, n_k, m_k, r_{k+1}]`` (column-major)."""

    def __init__(self, cores):
        self.cores = [np.asfortranarray(np.asarray(c, dtype=np.float64)) for c in cores]
        for c in self.cores:
            assert c.ndim == 4

    @property
    def d(self):
        return len(self.cores)

    @property
    def n(self):
        return np.array([c.shape[1] for c in self.cores], dtype=np.int64)

    @property
    def m(self):
        return np.array([c.shape[2] for c in self.cores], dtype=np.int64)

    @property
    def r(self):
        return np.array([self.cores[0].shape[0]] + [c.shape[3] for c in self.cores], dtype=np.int64)

    def flat(self):
        return np.concatenate([c.ravel(order="F") for c in self.cores])

    @staticmethod
    def from_flat(n, m, r, core):
        n = np.asarray(n, dtype=np.int64)
        m = np.asarray(m, dtype=np.int64)
        r = np.asarray(r, dtype=np.int64)
        core = np.asarray(core, dtype=np.float64).ravel()
        cores, pos = [], 0
        for k in range(len(n)):
            sz = int(r[k] * n[k] * m[k] * r[k + 1])
            cores.append(rs(core[pos:pos + sz], int(r[k]), int(n[k]), int(m[k]), int(r[k + 1])))
            pos += sz
        assert pos == core.size
        return TTMatrix(cores)

    def full(self):
        """Dense matrix (prod n) x (prod m), column-major multi-indices."""
        d = self.d
        res = np.ones((1, 1, 1))  # [rows, cols, rank]
        for c in self.cores:
            r1, n, m, r2 = c.shape
            # res[I, J, a] * c[a, i, j, b] -> [I, i, J, j, b]
            t = np.einsum("IJa,aijb->IiJjb", res, c)
            I, J = res.shape[0], res.shape[1]
            t = t.reshape(I, n, J, m, r2)
            # column-major combined index: I fastest then i
            t = np.transpose(t, (1, 0, 3, 2, 4)).reshape(n * I, m * J, r2)
            res = t
        del d
        return res[:, :, 0]


def tt_plus(a, b):
    """Rank-concatenation sum (``@tt_tensor/plus.m:40-86``)."""
    d = a.d
    cores = []
    for k in range(d):
        ca, cb = a.cores[k], b.cores[k]
        r1a, n, r2a = ca.shape
        r1b, _, r2b = cb.shape
        if d == 1:
            cores.append(ca + cb)
            continue
        if k == 0:
            c = np.zeros((r1a, n, r2a + r2b), order="F")
            c[:, :, :r2a] = ca
            c[:, :, r2a:] = cb
        elif k == d - 1:
            c = np.zeros((r1a + r1b, n, r2a), order="F")
            c[:r1a] = ca
            c[r1a:] = cb
        else:
            c = np.zeros((r1a + r1b, n, r2a + r2b), order="F")
            c[:r1a, :, :r2a] = ca
            c[r1a:, :, r2a:] = cb
        cores.append(c)
    return TT(cores)


def tt_matvec(A, x):
    """TT matrix-by-vector product, exact ranks ``ra*rx`` (``@tt_matrix/mtimes.m:38-65``).

    Output core layout ``[ra_k*rx_k, n_k, ra_{k+1}*rx_{k+1}]`` with the operator
    rank index fastest, as the reference's ``permute(pcur,[2,4,3,1,5])``
    produces it.
    """
    cores = []
    for Ak, xk in zip(A.cores, x.cores):
        ra1, n, m, ra2 = Ak.shape
        rx1, _, rx2 = xk.shape
        y = np.einsum("anmb,cmd->acnbd", Ak, xk)
        cores.append(np.asfortranarray(y.reshape(ra1 * rx1, n, ra2 * rx2, order="F")))
    return TT(cores)


def tt_norm(x):
    """Frobenius norm through a left-to-right QR sweep (``@tt_tensor/norm.m:16-42``)."""
    d = x.d
    nrm = np.zeros(d)
    core0 = x.cores[0]
    for i in range(d - 1):
        r1, n, r2 = core0.shape
        q, ru = np.linalg.qr(rs(core0, r1 * n, r2))
        nrm[i] = max(np.linalg.norm(ru), 1e-308)
        ru = ru / nrm[i]
        c1 = x.cores[i + 1]
        r2_, n1, r3 = c1.shape
        core0 = rs(ru @ rs(c1, r2_, n1 * r3), ru.shape[0], n1, r3)
    nrm[d - 1] = np.linalg.norm(core0)
    return float(np.prod(nrm))


def tt_dot(a, b):
    """Inner product by a left-to-right sweep of partial contractions (``@tt_tensor/dot.m:92-111``)."""
    p = np.ones((1, 1))
    for ca, cb in zip(a.cores, b.cores):
        # p[ra, rb] ; ca[ra, n, ra'] ; cb[rb, n, rb']
        p = np.einsum("ab,anc,bnd->cd", p, ca, cb)
    return float(p[0, 0])


def tt_ones(n, d):
    """All-ones tensor (``core/tt_ones.m:20-42``)."""
    return TT([np.ones((1, n, 1), order="F") for _ in range(d)])


def tt_randn(n, d, r, rng, scale=1.0):
    """Seeded Gaussian TT with ranks ``[1, r, ..., r, 1]`` (not orthogonalised)."""
    nn = [n] * d if np.isscalar(n) else list(n)
    rr = [1] + [r] * (d - 1) + [1] if np.isscalar(r) else list(r)
    cores = []
    for k in range(d):
        s = scale if not callable(scale) else scale(rr[k], nn[k], rr[k + 1])
        cores.append(np.asfortranarray(rng.standard_normal((rr[k], nn[k], rr[k + 1])) * s))
    return TT(cores)


def tt_rand(n, d, r, rng, direction=-1):
    """Random orthogonal TT (``core/tt_rand.m:40-62``), values from ``rng``.

    ``direction=-1``: right-to-left orthogonal, each core from
    ``qr(randn(n*r_{k+1}, r_k), 0).'`` (``tt_rand.m:52-56``).
    """
    nn = [n] * d if np.isscalar(n) else list(n)
    rr = [1] + [r] * (d - 1) + [1] if np.isscalar(r) else list(r)
    cores = [None] * d
    if direction > 0:
        for i in range(d):
            g = rng.standard_normal((rr[i] * nn[i], rr[i + 1]), ).copy(order="F")
            q, _ = np.linalg.qr(g)
            rr[i + 1] = q.shape[1]
            cores[i] = rs(q, rr[i], nn[i], rr[i + 1])
    else:
        for i in range(d - 1, -1, -1):
            g = rng.standard_normal((nn[i] * rr[i + 1], rr[i])).copy(order="F")
            q, _ = np.linalg.qr(g)
            q = q.T
            rr[i] = q.shape[0]
            cores[i] = rs(q, rr[i], nn[i], rr[i + 1])
    return TT(cores)


def true_residual(A, x, y):
    """``norm(A*x - y)/norm(y)`` with the QR-based TT norm, as the
    ``tests/tt-solve/README:15-16`` check prescribes."""
    return tt_norm(tt_plus(tt_matvec(A, x), y * (-1.0))) / tt_norm(y)
