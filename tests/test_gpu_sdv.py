"""SDV TT files through the C ABI (ttg_tt_read_sdv / ttg_tt_write_sdv),
pinned on the reference's own fmex/A.sdv and fmex/b.sdv (rebuilt from the
fixtures, SHA-256 checked), and the QTT system they hold solved by AMEn on
the device against the oracle."""
import os

import numpy as np
import pytest

import ttgpu
from golden_io import load_sdv
from oracle import amen as oamen
from oracle import sdv
from oracle.tt import TT, TTMatrix, tt_norm, tt_rand, true_residual

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["A", "b"])
def test_read_reference_files(ctx, tmp_path, name):
    hd, g, data = load_sdv(name)
    path = tmp_path / (name + ".sdv")
    path.write_bytes(data)
    t = ttgpu.read_sdv(str(path), ctx=ctx)
    assert list(t.n) == list(g["n"]) and list(t.r) == list(g["r"])
    assert np.array_equal(t.core, g["core"])  # bit-exact
    # writing it back (double) gives the reference's bytes
    out = tmp_path / (name + "_w.sdv")
    ttgpu.write_sdv(str(out), t, ctx=ctx)
    assert sdv.sha256(out.read_bytes()) == str(g["sha256"])


def test_float_round_trip_and_errors(ctx, tmp_path):
    rng = np.random.default_rng(2)
    cores = [rng.standard_normal((1, 3, 2)), rng.standard_normal((2, 4, 1))]
    t = ttgpu.TensorTrain.from_cores(cores)
    p = tmp_path / "f.sdv"
    ttgpu.write_sdv(str(p), t, precision="float", ctx=ctx)
    back = ttgpu.read_sdv(str(p), ctx=ctx)
    assert np.array_equal(back.core, t.core.astype(np.float32).astype(np.float64))
    f = sdv.parse(p.read_bytes())
    assert f["dtype"] == 2 and f["lm"] == (1, 2)
    # complex data type: rejected
    data = bytearray(p.read_bytes())
    data[20:24] = (1).to_bytes(4, "little")
    (tmp_path / "c.sdv").write_bytes(bytes(data))
    with pytest.raises(ttgpu.TTGError) as e:
        ttgpu.read_sdv(str(tmp_path / "c.sdv"), ctx=ctx)
    assert e.value.code == 7
    (tmp_path / "bad.sdv").write_bytes(b"XX" + bytes(data[2:]))
    with pytest.raises(ttgpu.TTGError, match="not a SDV"):
        ttgpu.read_sdv(str(tmp_path / "bad.sdv"), ctx=ctx)
    with pytest.raises(ttgpu.TTGError, match="short"):
        (tmp_path / "short.sdv").write_bytes(bytes(data[:140]))
        ttgpu.read_sdv(str(tmp_path / "short.sdv"), ctx=ctx)
    with pytest.raises(ttgpu.TTGError, match="can not be opened"):
        ttgpu.read_sdv(str(tmp_path / "missing.sdv"), ctx=ctx)


def test_amen_on_reference_qtt_system(ctx, tmp_path):
    """A (80 QTT cores of 2x2 blocks, ranks <= 4) x = b from the reference's
    SDV files, four sweeps from the same start: the first sweep matches the
    oracle to 1e-6 and the reached residuals agree within a factor 2 (the
    system is far from converged after four sweeps, and rank choices at
    rounding-level ties may differ between two FP64 implementations)."""
    files = {}
    for name in ("A", "b"):
        _, _, data = load_sdv(name)
        (tmp_path / (name + ".sdv")).write_bytes(data)
        files[name] = ttgpu.read_sdv(str(tmp_path / (name + ".sdv")), ctx=ctx)
    d = len(files["A"].n)
    A = ttgpu.as_matrix(files["A"], [2] * d, [2] * d)
    b = files["b"]
    Ao = TTMatrix.from_flat(A.n, A.m, A.r, A.core)
    bo = TT.from_flat(b.n, b.r, b.core)
    rng = np.random.default_rng(0)
    x0 = tt_rand(2, d, 2, rng)
    z0 = tt_rand(2, d, 4, rng)
    ref, info = oamen.amen_solve2(Ao, bo, 1e-6, x0, z0, nswp=4)
    st = {}
    got = ttgpu.amen_solve2(A, b, 1e-6, ctx=ctx, stats=st, nswp=4,
                            x0=ttgpu.TensorTrain(x0.n, x0.r, x0.flat()),
                            z0=ttgpu.TensorTrain(z0.n, z0.r, z0.flat()))
    got = TT.from_flat(got.n, got.r, got.core)
    np.testing.assert_allclose(st["max_res"][:1], info["max_res"][:1], rtol=1e-6)
    assert st["sweeps"] == info["sweeps"] == 4
    rg, rr = true_residual(Ao, got, bo), true_residual(Ao, ref, bo)
    assert rr / 2 < rg < 2 * rr
