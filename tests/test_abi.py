"""The C-ABI library loads and exports every symbol the public header declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ttgpu.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ttg_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("ttg_round", "ttg_amen_solve", "ttg_local_matvec", "ttg_next_phi",
              "ttg_local_solve", "ttg_tt_upload", "ttg_tt_download"):
        assert s in syms


def test_library_exports_all_declared_symbols():
    import ttgpu
    if not os.path.exists(ttgpu.LIB_PATH):
        pytest.fail("libttgpu.so is not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(ttgpu.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_host_wrapper_argument_errors():
    """Shape validation of the MEX-compatible wrapper happens before any device call."""
    import numpy as np
    import ttgpu
    with pytest.raises(ttgpu.TTGError, match="Phi1 is not square"):
        ttgpu.solve3d_2(np.zeros((2, 3, 1)), np.zeros((1, 4, 4, 1)), np.zeros((2, 1, 2)),
                        np.zeros(16), 1e-6, 1, np.zeros(16), ctx=object())
    with pytest.raises(ValueError, match="Unrecognized option"):
        ttgpu.amen_solve2(None, None, 1e-6, bogus=1)
    t = ttgpu.TensorTrain([2, 3], [1, 2, 1], np.arange(10.0))
    assert [c.shape for c in t.cores()] == [(1, 2, 2), (2, 3, 1)]
    with pytest.raises(ValueError):
        ttgpu.TensorTrain([2, 3], [1, 2, 1], np.arange(11.0))
