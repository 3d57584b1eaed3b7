"""Command-line parser of the C++ host API's Configurations, on the CPU.

Compiles tests/cpp/test_configurations.cpp with host/src/Configurations.cpp
(g++, no GPU library) and runs it: the reference's spellings of
--computation (exact / dense / diag_approx), --precision (double / mixed),
--band, --datapath and snake_case kernel names, this build's --mixedband, and
the errors the reference raises for invalid values (Validator.cpp:108-136),
with tile low-rank, single precision and 3-D locations refused as not on the
B200 path.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CASES = ["mixed_run", "diag_approx", "dense_double", "mix_spelling", "precision_invalid",
         "precision_single_not_run", "computation_invalid", "computation_tlr_not_run", "unknown_argument",
         "dimension_3d_not_run", "distance_invalid", "idw_not_run", "process_grid_not_run", "prediction_flags"]


def test_configurations_parser(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "test_configurations"
    cmd = [cxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "exageostatcpp_b200", "host", "include"),
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "exageostatcpp_b200", "host", "src", "Configurations.cpp"),
           os.path.join(HERE, "cpp", "test_configurations.cpp"), "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    lines = dict(line.split(": ", 1) for line in run.stdout.strip().splitlines())
    for case in CASES:
        assert case in lines, run.stdout + run.stderr
        assert lines[case].startswith("ok"), f"{case}: {lines[case]}"
    assert run.returncode == 0
