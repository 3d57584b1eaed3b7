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


def test_conditioning_estimate_formula_and_measured_classification():
    # kappa = (1 + (pi beta / h)^2)^(nu + 1), h = sqrt(bounding-box area / n)
    x = [0.0, 1.0, 0.0, 1.0]
    y = [0.0, 0.0, 2.0, 2.0]
    k = egs.mixed_conditioning_estimate(x, y, [1.0, 0.1, 0.5])
    h = (2.0 / 4) ** 0.5
    assert k == pytest.approx((1 + (3.141592653589793 * 0.1 / h) ** 2) ** 1.5, rel=1e-14)
    # Outcomes of the mixed form (FP64 band of 2 tiles, FP32 off-band tiles) measured
    # on a B200 on jittered unit-square grids; the server's limit is 1e9.
    measured = [  # (n, beta, nu, mixed factorisation positive definite)
        (6000, 0.1, 1.8, True), (6000, 0.3, 1.2, True), (24000, 0.2, 1.2, True), (24000, 0.3, 0.7, True),
        (6000, 0.1, 2.5, False), (6000, 0.2, 1.8, False), (24000, 0.1, 1.8, False), (24000, 0.3, 1.2, False),
    ]
    for n, beta, nu, ok in measured:
        xs, ys = egs.generate_locations(n, 1)
        kappa = egs.mixed_conditioning_estimate(xs, ys, [1.0, beta, nu])
        assert (kappa <= 1e9) == ok, (n, beta, nu, kappa)
    with pytest.raises(egs.EgsError):
        egs.mixed_conditioning_estimate(x, y, [1.0, -0.1, 0.5])
