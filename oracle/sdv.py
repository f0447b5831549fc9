"""SDV TT file format -- a plain-Python restatement for the tests.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Layout as read and written by ``fmex/tt_read.c:13-100`` and
``fmex/tt_write.c:21-80``: a 128-byte header (char txt[8], int32 ver[2],
int32 inf[4], char comment[64], int32 i[8]; inf[1] is the data type, 0
double / 1 complex double / 2 float / 3 complex float), int32 l and m
(d = m - l + 1), int32 n[d], int32 r[d+1], then the flat core vector.
Pinned by the reference's own files ``fmex/A.sdv`` and ``fmex/b.sdv``: the
fixtures keep their SHA-256, and ``write`` of the parsed contents must give
those bytes back.
"""
import hashlib
import struct

import numpy as np

HEAD = struct.Struct("<8s2i4i64s8i")


def parse(data):
    """dict(header fields, d, n, r, core) from the bytes of a SDV file."""
    txt, v0, v1, i0, i1, i2, i3, comment, *ii = HEAD.unpack_from(data, 0)
    if not txt.startswith(b"TT"):
        raise ValueError("not a SDV TT file")
    if v0 != 1:
        raise ValueError("wrong SDV version %d" % v0)
    off = HEAD.size
    l, m = struct.unpack_from("<2i", data, off)
    off += 8
    d = m - l + 1
    n = np.frombuffer(data, "<i4", d, off).astype(np.int64)
    off += 4 * d
    r = np.frombuffer(data, "<i4", d + 1, off).astype(np.int64)
    off += 4 * (d + 1)
    numel = int(sum(r[k] * n[k] * r[k + 1] for k in range(d)))
    dt = {0: "<f8", 2: "<f4"}.get(i1)
    if dt is None:
        raise ValueError("complex or unknown SDV data type %d" % i1)
    core = np.frombuffer(data, dt, numel, off).astype(np.float64)
    return dict(txt=txt, ver=(v0, v1), inf=(i0, i1, i2, i3), comment=comment, i=tuple(ii),
                lm=(l, m), d=d, n=n, r=r, core=core, dtype=i1)


def write(hd, n, r, core):
    """Bytes of a SDV file with header fields ``hd`` (as from ``parse``)."""
    out = [HEAD.pack(hd["txt"], *hd["ver"], *hd["inf"], hd["comment"], *hd["i"]),
           struct.pack("<2i", *hd["lm"]), np.asarray(n, "<i4").tobytes(),
           np.asarray(r, "<i4").tobytes(),
           np.asarray(core, "<f8" if hd["inf"][1] == 0 else "<f4").tobytes()]
    return b"".join(out)


def sha256(data):
    return hashlib.sha256(data).hexdigest()
