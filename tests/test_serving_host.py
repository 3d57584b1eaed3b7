"""Host-side parts of the serving loop that need no GPU: the HBM footprint used
for admission, and server creation without a device."""
import ctypes

import pytest

import exageostatcpp_b200 as egs


def test_footprint_plain_matches_tile_storage():
    # N = 40,000, tile 960: 903 lower tiles of 960^2 doubles plus vectors and slack
    b = egs.footprint(40000, 960)
    tiles = 903 * 960 * 960 * 8
    assert tiles < b < tiles + 100 * 2**20


def test_footprint_mixed_is_smaller_at_large_n():
    n = 102400
    plain = egs.footprint(n, 1024)
    mixed = egs.footprint(n, 1024, egs.EGS_PRECISION_MIXED, 2)
    assert mixed < 0.6 * plain
    # FP32 off-band (4,753 tiles) + FP64 band (300 tiles) + FP64 workspace and inverses (201 tiles)
    ts2 = 1024 * 1024
    assert mixed > 4753 * ts2 * 4 + 300 * ts2 * 8 + 201 * ts2 * 8


def test_footprint_grows_with_n_and_rejects_bad_arguments():
    sizes = [1000, 5000, 20000, 60000]
    fps = [egs.footprint(n, 512) for n in sizes]
    assert fps == sorted(fps)
    lib = egs.load_library()
    out = ctypes.c_longlong()
    assert lib.egs_problem_footprint(0, 512, 1, 0, ctypes.byref(out)) == egs.EGS_ERR_INVALID
    assert lib.egs_problem_footprint(100, 512, 7, 0, ctypes.byref(out)) == egs.EGS_ERR_INVALID


def test_server_needs_a_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = egs.load_library()
    h = ctypes.c_void_p()
    assert lib.egs_server_create(ctypes.byref(h), 0, 1 << 30, 2) == egs.EGS_ERR_NO_DEVICE
    assert lib.egs_server_create(ctypes.byref(h), 0, 0, 2) == egs.EGS_ERR_INVALID
