"""The C ABI library: it loads on a CPU-only host and exports every symbol
that include/exageostat_b200.h declares (no compute call needs a GPU here)."""
import ctypes
import os
import re

import pytest

import exageostatcpp_b200 as egs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "exageostat_b200.h")).read()
    return sorted(set(re.findall(r"EGS_API\s+[\w\s\*]*?\b(egs_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = egs.load_library()
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(egs.SIGNATURES), "ctypes signature table out of sync with the header"


def test_status_strings():
    lib = egs.load_library()
    assert lib.egs_version() > 0
    assert lib.egs_status_string(0) == b"ok"
    assert lib.egs_status_string(egs.EGS_ERR_TIMEOUT) == b"device wait timed out"
    assert lib.egs_status_string(17) == b"matrix is not positive definite"


def test_invalid_arguments_rejected_without_device():
    lib = egs.load_library()
    h = ctypes.c_void_p()
    assert lib.egs_problem_create(ctypes.byref(h), 0, 8) == egs.EGS_ERR_INVALID
    assert lib.egs_problem_create(None, 10, 8) == egs.EGS_ERR_INVALID
    assert lib.egs_problem_destroy(None) == egs.EGS_OK


def test_no_device_is_an_error_not_a_fallback():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    lib = egs.load_library()
    h = ctypes.c_void_p()
    assert lib.egs_problem_create(ctypes.byref(h), 16, 8) == egs.EGS_ERR_NO_DEVICE
    with pytest.raises(egs.EgsError):
        egs.Problem(16, 8)


def test_failed_kernel_launch_is_reported_not_swallowed():
    # On a host without a usable CUDA driver the generator's launch itself fails.
    # The launch helper reads the runtime's error once; the entry point must return
    # that failure (EGS_ERR_CUDA with the kernel named), not EGS_OK from a second,
    # already cleared error read.  Host buffers are passed, so the call is only
    # made where no device could run the kernel.
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    import numpy as np
    lib = egs.load_library()
    buf = (ctypes.c_double * 16)()
    vp = ctypes.cast(buf, ctypes.c_void_p)
    theta = np.array([1.0, 0.1, 0.5])
    rc = lib.egs_matern_block(vp, 4, 4, 4, vp, vp, vp, vp, theta.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              0, None)
    assert rc == egs.EGS_ERR_CUDA
    assert b"matern_block_kernel" in lib.egs_last_error()
