"""Mixed-precision rounding: the two contractions of the sweeps
(R * core, @tt_tensor/round.m:47, and core * (U S), :83) on the BF16 tensor
cores with FP32 accumulation, QR and SVD in FP64.  BF16 operands carry an
8-bit mantissa, so the result is accurate to about 1e-2 relative, not to
eps: the tests bound the error by eps plus that operand rounding and check
that the ranks stay those of the FP64 rounding where the cut lies well
above the BF16 noise."""
import numpy as np
import pytest

import ttgpu
from oracle.builders import round_config
from oracle.round import tt_round
from oracle.tt import TT, tt_norm, tt_randn

pytestmark = pytest.mark.gpu

BF16_ROUND_TOL = 2e-2


def _host(t):
    return ttgpu.TensorTrain(t.n, t.r, t.flat())


def _back(t):
    return TT.from_flat(t.n, t.r, t.core)


def test_round_mixed_decaying_spectrum(ctx):
    rng = np.random.default_rng(23)
    x = tt_randn(16, 8, 40, rng, scale=lambda r1, nn, r2: 1.0 / np.sqrt(r1 * nn))
    cores = [c.copy() for c in x.cores]
    for k in range(x.d - 1):
        cores[k] = cores[k] * np.exp(-0.3 * np.arange(cores[k].shape[2]))[None, None, :]
    xt = TT(cores)
    eps = 0.1
    ref, _ = tt_round(xt, eps)
    st = {}
    got = _back(ttgpu.round(_host(xt), eps, precision="mixed", ctx=ctx, stats=st))
    err = tt_norm(got - xt) / tt_norm(xt)
    assert err <= eps + BF16_ROUND_TOL
    assert max(abs(int(a) - int(b)) for a, b in zip(got.r, ref.r)) <= 2


def test_round_mixed_full_size(ctx):
    """The full-size rounding input (sum of four rank-64 TTs, d=20, n=16) at eps 1e-8:
    all ranks stay 256 and the error is the BF16 operand rounding of the 38
    contractions (1.4e-2 when the same operand rounding is emulated in FP64
    on the host)."""
    x = round_config(d=20, n=16, r=64, terms=4, seed=2)
    st = {}
    got = _back(ttgpu.round(_host(x), 1e-8, precision="mixed", ctx=ctx, stats=st))
    assert list(got.r) == [1, 16] + [256] * 17 + [16, 1]
    assert tt_norm(got - x) / tt_norm(x) <= 3e-2
