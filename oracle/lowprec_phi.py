"""Test infrastructure: the FP64 AMEn oracle with the interface (Phi)
contractions fed low-precision operands, to measure what precision the
Phi/core contractions of ``compute_next_Phi`` (``solve/amen_solve2.m:834-920``)
need for a 1e-8 residual.

``rounded_phi(fmt)`` is a context manager that replaces
``oracle.amen.compute_next_Phi`` by a version whose operands (the previous
interface, the cores and the operator core) are rounded to ``fmt`` before
the products, which then run in FP64: BF16 or TF32 tensor-core inputs with
an accumulation more accurate than FP32, the most favourable case for the
low-precision form.  The local solves, truncations and refinements stay
FP64, so any loss of accuracy comes from the interfaces alone: the local
systems the solver refines against are then not the projections of the
global operator, and no local FP64 refinement can recover that.
"""
import contextlib

import numpy as np

from oracle import amen as _amen


def round_to(a, fmt):
    """Round to nearest even on the FP32 bit pattern: ``'bf16'`` keeps 8
    significand bits, ``'tf32'`` 11, ``'fp32'`` all 24."""
    a = np.asarray(a, dtype=np.float64)
    f = a.astype(np.float32)
    if fmt == "fp32":
        return f.astype(np.float64)
    drop = {"bf16": 16, "tf32": 13}[fmt]
    u = f.view(np.uint32).astype(np.uint64)
    half = (1 << (drop - 1)) - 1
    u = (u + half + ((u >> drop) & 1)) & (0xFFFFFFFF ^ ((1 << drop) - 1))
    return u.astype(np.uint32).view(np.float32).astype(np.float64).reshape(a.shape)


@contextlib.contextmanager
def rounded_phi(fmt):
    orig = _amen.compute_next_Phi

    def lowp(Phi_prev, x, A, y, direction, extnrm=None, want_norm=False):
        r = lambda t: None if t is None else np.asfortranarray(round_to(t, fmt))
        return orig(r(Phi_prev), r(x), r(A), r(y), direction, extnrm=extnrm,
                    want_norm=want_norm)

    _amen.compute_next_Phi = lowp
    try:
        yield
    finally:
        _amen.compute_next_Phi = orig
