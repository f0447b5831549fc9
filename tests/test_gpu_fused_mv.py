"""The fused single-launch BF16 local matvec against the three-launch form.

Both forms run the same tcgen05 tiles in the same K order (FP32
accumulation), so the fused persistent kernel (TTG_FUSED_MV=1) must give
the same numbers bit for bit as the three separate GEMM launches (the
default), each run in a child process, with one launch per matvec instead
of three."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import ttgpu

pytestmark = pytest.mark.gpu

SHAPES = [(1, 64, 2, 1, 3), (5, 16, 7, 2, 3), (33, 17, 65, 3, 2), (61, 64, 59, 3, 3),
          (128, 64, 128, 3, 3), (132, 32, 100, 2, 2), (200, 8, 150, 3, 3)]

CHILD = r"""
import json, os, sys
import numpy as np
sys.path[:0] = [os.path.join(os.environ["ROOT"], "tt-toolbox_b200")]
import ttgpu
ctx = ttgpu.Context(int(os.environ.get("TTG_DEVICE", "0")))
out = []
launches = []
for (rx1, n, rx2, ra1, ra2) in json.loads(os.environ["SHAPES"]):
    rng = np.random.default_rng(rx1 + 7 * rx2 + n)
    Phi1 = rng.standard_normal((rx1, rx1, ra1)); A = rng.standard_normal((ra1, n, n, ra2))
    Phi2 = rng.standard_normal((rx2, ra2, rx2)); x = rng.standard_normal(rx1 * n * rx2)
    y = ttgpu.bfun3(Phi1, A, Phi2, x, ctx=ctx, precision="mixed")
    before = ctx.launch_count()
    y = ttgpu.bfun3(Phi1, A, Phi2, x, ctx=ctx, precision="mixed")
    launches.append(ctx.launch_count() - before)
    out.append(y.tolist())
print(json.dumps([out, launches]))
"""


def _run(fused):
    env = dict(os.environ)
    env["ROOT"] = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env["SHAPES"] = json.dumps(SHAPES)
    env["TTG_FUSED_MV"] = "1" if fused else "0"
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out, launches = json.loads(r.stdout.strip().splitlines()[-1])
    return [np.array(v) for v in out], launches


def test_fused_matches_three_launches_bitwise():
    """Same outputs bit for bit; ttg_local_matvec in BF16 is three operand
    conversions, the vector into the reversed FP32 layout and into BF16,
    the matvec, then the result back (zero fill + add): eight launches with
    the fused kernel, ten with the three GEMM launches."""
    (fused, lf), (split, ls) = _run(True), _run(False)
    for shape, a, b in zip(SHAPES, fused, split):
        assert np.array_equal(a, b), shape
    assert all(v == 8 for v in lf), lf
    assert all(v == 10 for v in ls), ls
