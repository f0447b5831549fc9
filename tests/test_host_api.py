"""Host-side behaviour of the library and its Python binding that needs no
GPU: argument checks that fail before any device work, the C ABI's status
codes for NULL arguments, and the absence of a CPU fallback."""
import ctypes as C

import numpy as np
import pytest

import ttgpu


def _lib():
    try:
        return ttgpu.lib()
    except ImportError as e:  # the library must be built for this suite
        pytest.fail(str(e))


def test_no_cpu_fallback_without_a_device():
    """Creating a context on a machine without a CUDA device fails with a
    status code; nothing computes on the host instead."""
    lib = _lib()
    h = C.c_void_p()
    code = lib.ttg_context_create(0, C.byref(h))
    if code == 0:  # a GPU is present: nothing to check here
        lib.ttg_context_destroy(h)
        pytest.skip("a CUDA device is present")
    assert code in (1, 2)  # TTG_ERR_INVALID (no device 0) or TTG_ERR_CUDA
    assert lib.ttg_last_error().decode()
    with pytest.raises(ttgpu.TTGError):
        ttgpu.Context(0)


def test_null_arguments_return_invalid():
    lib = _lib()
    out = C.c_void_p()
    assert lib.ttg_round(None, C.c_double(1e-8), None, C.c_int64(0), C.c_int32(0),
                         C.byref(out), None) == 1
    assert b"NULL" in lib.ttg_last_error()
    assert lib.ttg_tt_download(None, None) == 1
    assert lib.ttg_context_sync(None) == 1
    assert lib.ttg_context_create(0, None) == 1
    assert lib.ttg_tt_free(None) == 0  # freeing nothing is allowed


def test_amen_option_checks():
    with pytest.raises(ValueError, match="Unrecognized option"):
        ttgpu.amen_solve2(None, None, 1e-6, NotAnOption=3)
    with pytest.raises(ttgpu.TTGError, match="kicktype"):
        ttgpu.amen_solve2(None, None, 1e-6, kicktype="svd")
    with pytest.raises(ttgpu.TTGError, match="trunc_norm"):
        ttgpu.amen_solve2(None, None, 1e-6, trunc_norm="fro")
    with pytest.raises(ttgpu.TTGError, match="local_prec"):
        ttgpu.amen_solve2(None, None, 1e-6, local_prec="ilu")
    # option names are case-insensitive, as in the reference's parser
    assert ttgpu._check_amen_opts({"NSWP": 3, "Local_Prec": "cjacobi"})["nswp"] == 3


def test_batch_argument_checks():
    with pytest.raises(ValueError, match="differ in length"):
        ttgpu.amen_solve2_batch([None, None], [None], 1e-6)


def test_tt_containers_and_reinterpretation():
    t = ttgpu.TensorTrain([6, 4], [1, 3, 1], np.arange(6 * 3 + 3 * 4, dtype=float))
    assert [c.shape for c in t.cores()] == [(1, 6, 3), (3, 4, 1)]
    M = ttgpu.as_matrix(t, [2, 2], [3, 2])
    assert list(M.n) == [2, 2] and list(M.m) == [3, 2]
    with pytest.raises(ValueError, match="n .\\* m"):
        ttgpu.as_matrix(t, [2, 2], [2, 2])
    with pytest.raises(ValueError):
        ttgpu.TTMatrix([2, 2], [3, 2], [1, 3, 1], np.zeros(5))


def test_sample_set_shape_checks():
    with pytest.raises(ValueError, match=r"\[S, d\]"):
        ttgpu.SampleSet(None, np.zeros(5, np.int32), np.zeros(5))
    with pytest.raises(ValueError, match="one value per sample"):
        ttgpu.SampleSet(None, np.zeros((5, 3), np.int32), np.zeros(4))
