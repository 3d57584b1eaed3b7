"""The C++ host API (ExaGeoStat<T>, Configurations, Kernel plugin, Prediction) against
the reference's API-level goldens.  The driver tests/cpp/test_exageostat_api.cpp sets
up each case the way the reference's Catch2 test does; this file checks its output.
"""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "test_exageostat_api")


@pytest.fixture(scope="module")
def driver():
    if not os.path.exists(BIN):
        from exageostatcpp_b200 import build as b
        b.build_host_tests()
    return BIN


@pytest.fixture(scope="module")
def fixture_file(goldens, tmp_path_factory):
    f = goldens["fixture_n16"]
    p = tmp_path_factory.mktemp("fx") / "fixture.txt"
    p.write_text("\n".join(" ".join(repr(v) for v in f[k]) for k in ("x", "y", "z")) + "\n")
    return str(p)


def run(driver, *args):
    res = subprocess.run([driver, *args], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    return json.loads(res.stdout.strip().splitlines()[-1])


def test_generated_locations_cpu(driver, goldens):
    # CPU only: the location generator draws from the C library's rand()
    out = run(driver, "generated_locations")
    g = goldens["locations_n9_seed0"]
    assert np.abs(np.array(out["x"]) - g["x"]).max() < g["margin"]
    assert np.abs(np.array(out["y"]) - g["y"]).max() < g["margin"]
    assert np.abs(np.array(out["x_second"]) - g["x"]).max() > g["margin"]   # continues the sequence
    assert np.array_equal(out["x_reseeded"], out["x"])


@pytest.mark.gpu
@pytest.mark.parametrize("case,key", [("generate_n16", "z_n16_dts9_seed0"), ("generate_n9", "z_n9_dts5_seed0")])
def test_load_data_observations(driver, goldens, case, key):
    out = run(driver, case)
    g = goldens[key]
    assert np.abs(np.array(out["z"]) - g["z"]).max() < g["margin"]


@pytest.mark.gpu
def test_data_modeling_fixture(driver, goldens, fixture_file):
    out = run(driver, "modeling_fixture", fixture_file)
    g = goldens["modeling_loglik_n16"]
    assert abs(out["loglik"] - g["exact_dense"]) < g["margin"]
    assert out["iterations"] == g["max_mle_iterations"]
    assert out["theta"] == pytest.approx([1.325, 0.1, 0.1], abs=1e-12)


@pytest.mark.gpu
def test_data_modeling_fixture_diagonal_approximation(driver, goldens, fixture_file):
    # TestExaGeoStatApi.cpp:95: --computation=diag_approx on tiles of 8 (band 1)
    out = run(driver, "modeling_fixture_dst", fixture_file)
    g = goldens["modeling_loglik_n16"]
    assert abs(out["loglik"] - g["diag_approx_band1"]) < g["margin"]
    assert out["iterations"] == g["max_mle_iterations"]


@pytest.mark.gpu
def test_data_generation_and_modeling(driver, goldens):
    out = run(driver, "generate_and_model")
    g = goldens["modeling_loglik_n16"]
    assert abs(out["loglik"] - g["exact_dense"]) < g["margin"]


@pytest.mark.gpu
def test_prediction_mspe(driver, goldens, fixture_file):
    out = run(driver, "prediction_mspe", fixture_file)
    g = goldens["prediction_mspe_n16"]
    assert out["mspe"] == pytest.approx(g["mspe"], rel=1.2e-5)
    assert len(out["z_miss"]) == g["z_miss_number"]


@pytest.mark.gpu
def test_kernel_plugin_and_error_behaviour(driver, fixture_file):
    out = run(driver, "plugin_and_errors", fixture_file)
    assert out["plugin_max_rel_err"] < 1e-13
    assert "NoSuchKernel" in out["unknown_kernel"]
    assert out["non_spd"] == "Matrix is not positive definite"
    assert out["no_theta"].startswith("Can't predict without an estimated")


@pytest.mark.gpu
def test_mixed_precision_through_the_api(driver):
    # Configurations::SetPrecision(MIXED): the same three BOBYQA evaluations as in
    # FP64; the best log-likelihood within the mixed-precision tolerance (1e-6)
    out = run(driver, "mixed_modeling")
    assert abs(out["loglik_mixed"] - out["loglik_double"]) <= 1e-6 * abs(out["loglik_double"])
    assert out["theta_mixed"] == pytest.approx(out["theta_double"], abs=1e-12)


@pytest.mark.gpu
def test_prediction_mloe_mmom_and_fisher(driver, goldens, fixture_file):
    # TestPrediction.cpp:129-130 (reference margin 1e-3) and :167-168 (the
    # reference's 1e-6 applies to its own forward-difference dK/dnu; the exact
    # derivative agrees to 1.5e-5)
    out = run(driver, "prediction_aux", fixture_file)
    g = goldens["prediction_mloe_mmom_n16"]
    assert abs(out["mloe"] - g["mloe"]) < 1e-6 and abs(out["mmom"] - g["mmom"]) < 1e-6
    fg = goldens["prediction_fisher_n16"]
    assert max(abs(a - b) for a, b in zip(out["fisher"], fg["fisher_inverse"])) < 2e-5


@pytest.mark.gpu
def test_csv_loader_round_trip(driver, tmp_path):
    # CSVLoader.cpp:37-289: 15 significant digits written, read back through
    # ExaGeoStatLoadData(--datapath); a 4-value line is rejected for 2-D data
    out = run(driver, "csv_roundtrip", str(tmp_path))
    assert out["n"] == 16
    assert out["max_diff"] < 1e-14
    assert abs(out["loglik_csv"] - out["loglik_generated"]) <= 1e-12 * abs(out["loglik_generated"])
    assert "dimensions" in out["bad"]
    assert any(p.name == "SYN_16_1" for p in (tmp_path / "synthetic_ds").iterdir())


@pytest.mark.gpu
def test_seam_tile_operations_match_the_evaluation_and_the_oracle(driver):
    # LinearAlgebraMethods' tile operations (InitiateDescriptors, CreateSequence,
    # LapackCopyTile, PotrfTile, TrsmTile, SequenceWait, PosvTile, Desc2Lap,
    # Lap2Desc) strung together as ChameleonImplementation.cpp:113-265 does.
    from oracle import oracle as O
    import scipy.linalg
    out = run(driver, "seam_tile_operations")
    x, y, z = (np.array(out[k]) for k in ("x", "y", "z"))
    theta = [1.0, 0.1, 0.5]
    ref, rlogdet, rdot = O.mle_loglik(x, y, z, theta, return_parts=True)
    assert out["loglik_tiles"] == pytest.approx(ref, rel=1e-10, abs=0)
    assert out["loglik_tiles"] == pytest.approx(out["loglik_eval"], rel=1e-12, abs=0)
    assert out["dot"] == pytest.approx(rdot, rel=1e-10)
    w = scipy.linalg.cho_solve(scipy.linalg.cho_factor(O.covariance(x, y, theta), lower=True), z)
    assert np.abs(np.array(out["w"]) - w).max() <= 1e-9 * np.abs(w).max()
    assert out["roundtrip"] == 0.0
    assert "lower" in out["bad_uplo"] and "left" in out["bad_trans"] and "unexpected" in out["bad_desc"]
