"""The CPU oracle against the golden vectors of the reference's own tests.

These pin the oracle before it is trusted as the GPU checker (CPU only)."""
import math

import mpmath
import numpy as np
import pytest
import scipy.special

from oracle import oracle as O


def test_glibc_rand_restatement_matches_libc():
    for seed in (0, 1, 7, 12345, 4095):
        r = O.GlibcRand(seed)
        assert [r.rand() for _ in range(2000)] == O.libc_rand_sequence(seed, 2000)


def test_morton_roundtrip_and_known_codes():
    v = np.arange(0, 65536, 37, dtype=np.uint64)
    assert np.array_equal(O.reverse_spread_bits(O.spread_bits(v)), v)
    # TestSyntheticGenerator.cpp bit tests: bit b of the input lands at bit 4b
    for b in range(16):
        assert int(O.spread_bits(np.uint64(1 << b))) == 1 << (4 * b)


def test_locations_n9_seed0(goldens):
    g = goldens["locations_n9_seed0"]
    x, y = O.generate_locations(9, O.GlibcRand(0))
    assert np.abs(x - g["x"]).max() < g["margin"]
    assert np.abs(y - g["y"]).max() < g["margin"]


@pytest.mark.parametrize("key", ["z_n9_dts5_seed0", "z_n16_dts9_seed0"])
def test_generated_observations(goldens, key):
    g = goldens[key]
    x, y, z = O.load_data(g["n"], g["seed"], g["theta"])
    assert np.abs(z - g["z"]).max() < g["margin"]


def test_fixture_is_seed0_generator_output(goldens):
    f = goldens["fixture_n16"]
    x, y, z = O.load_data(16, 0, [1.0, 0.1, 0.5])
    assert np.array_equal(x, f["x"]) and np.array_equal(y, f["y"])
    assert np.abs(z - f["z"]).max() < 1e-14


def test_modeling_loglik_golden(goldens):
    # NLopt BOBYQA with x0 = lb = 0.1 and 3 evaluations reaches theta = (1.325, 0.1, 0.1):
    # x0 + rhobeg e_1 with rhobeg = 0.25 (ub - lb).
    f = goldens["fixture_n16"]
    g = goldens["modeling_loglik_n16"]
    ll = O.mle_loglik(f["x"], f["y"], f["z"], [1.325, 0.1, 0.1])
    assert abs(ll - g["exact_dense"]) < g["margin"]


def test_prediction_mspe_golden(goldens):
    f = goldens["fixture_n16"]
    g = goldens["prediction_mspe_n16"]
    zo, xo, yo, za, xm, ym = O.shuffle_split(f["z"], f["x"], f["y"], g["z_miss_number"], O.GlibcRand(1))
    _, mspe = O.predict(xo, yo, zo, xm, ym, g["estimated_theta"], za)
    assert mspe == pytest.approx(g["mspe"], rel=1.2e-5)


@pytest.mark.parametrize("nu", [0.3, 0.4, 0.5, 0.8, 1.0, 1.5, 2.2, 2.5])
def test_matern_oracle_against_mpmath(nu):
    mpmath.mp.dps = 40
    sigma2, beta = 1.3, 0.07
    for d in (1e-4, 0.01, 0.07, 0.13, 0.3, 0.9):
        xv = d / beta
        exact = sigma2 / (mpmath.mpf(2) ** (nu - 1) * mpmath.gamma(nu)) * mpmath.mpf(xv) ** nu * mpmath.besselk(nu, xv)
        got = O.matern_block([0.0], [0.0], [d], [0.0], [sigma2, beta, nu])[0, 0]
        assert abs(got - float(exact)) <= 1e-13 * abs(float(exact)) + 1e-300


def test_oracle_cholesky_failure_is_reported():
    x = np.array([0.1, 0.2, np.nan])
    with pytest.raises(Exception):
        O.mle_loglik(x, x, np.ones(3), [1.0, 0.1, 0.5])


def test_diagonal_approximation_golden(goldens):
    # TestExaGeoStatApi.cpp:95: DIAGONAL_APPROX with band 1, same 3 BOBYQA evaluations
    f = goldens["fixture_n16"]
    g = goldens["modeling_loglik_n16"]
    vals = [O.dst_loglik(f["x"], f["y"], f["z"], th, g["dts"], 1)
            for th in ([0.1, 0.1, 0.1], [1.325, 0.1, 0.1], [0.1, 1.325, 0.1])]
    assert abs(max(vals) - g["diag_approx_band1"]) < g["margin"]


def test_wide_band_is_exact():
    x, y, z = O.load_data(200, 2, [1.0, 0.1, 0.5])
    th = [0.9, 0.12, 0.7]
    assert O.dst_loglik(x, y, z, th, 64, 4) == pytest.approx(O.mle_loglik(x, y, z, th), rel=1e-12)


def test_mloe_mmom_golden(goldens):
    # TestPrediction.cpp:129-130: Catch re-runs the test body for every SECTION, so
    # the MLOE/MMOM section sees the third PickRandomPoints split of the fresh
    # glibc state (after the MSPE and IDW sections)
    f = goldens["fixture_n16"]
    g = goldens["prediction_mloe_mmom_n16"]
    rng = O.GlibcRand(1)
    for _ in range(g["split_index"]):
        O.shuffle_split(f["z"], f["x"], f["y"], g["z_miss_number"], rng)
    zo, xo, yo, za, xm, ym = O.shuffle_split(f["z"], f["x"], f["y"], g["z_miss_number"], rng)
    mloe, mmom = O.mloe_mmom(xo, yo, xm, ym, g["truth_theta"], g["estimated_theta"])
    assert abs(mloe - g["mloe"]) < 1e-6 and abs(mmom - g["mmom"]) < 1e-6   # the reference's margin is 1e-3
    # equal thetas: no loss (TestPrediction.cpp:150-151)
    mloe0, mmom0 = O.mloe_mmom(xo, yo, xm, ym, g["truth_theta"], g["truth_theta"])
    assert abs(mloe0) < 1e-12 and abs(mmom0) < 1e-12


def test_dkv_dnu_against_mpmath():
    import mpmath as mp
    for nu in (0.4, 1.3, 2.5):
        for x in (0.01, 0.3, 2.0, 15.0):
            a = O.dkv_dnu(nu, np.array([x]))[0]
            b = float(mp.diff(lambda v: mp.besselk(v, x), nu))
            assert abs(a - b) <= 1e-14 * abs(b)


def test_fisher_golden(goldens):
    # TestPrediction.cpp:167-168.  The reference differentiates K_nu in nu by a forward
    # difference with step 1e-9 over GSL's K_nu, which leaves ~1e-7 relative rounding
    # noise in dK/dnu; with the exact derivative the inverse Fisher matrix agrees with
    # the golden values to 1.5e-5 (largest on the nu-nu entry, 10.556), so the parity
    # bound here is 2e-5 where the reference asks 1e-6 of its own noisy derivative.
    f = goldens["fixture_n16"]
    g = goldens["prediction_fisher_n16"]
    inv = O.fisher_inverse(f["x"], f["y"], g["estimated_theta"])
    got = inv.T.reshape(-1)
    assert np.abs(got - np.array(g["fisher_inverse"])).max() < 2e-5
    assert np.allclose(inv, inv.T, rtol=0, atol=1e-12)
