"""CSV data loader and writer of the C++ host API, on the CPU.

Compiles tests/cpp/test_csv_loader.cpp against the host headers with g++ and
runs it in a scratch directory: the 15-significant-digit round trip, the
SYN_<n>_<i> file numbering next to log_<n>_<i> files, blank lines, and the
rejection of lines with four or two values, of an empty path and of a missing
file (CSVLoader.cpp:37-289 in the reference).  No GPU call is made.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CASES = ["write_name", "round_trip", "write_index", "blank_lines", "reject_four_values", "reject_two_values",
         "reject_empty_path", "reject_missing_file"]


@pytest.fixture(scope="module")
def csv_driver(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("csv_build") / "test_csv_loader"
    cmd = [cxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "exageostatcpp_b200", "host", "include"),
           "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "cpp", "test_csv_loader.cpp"), "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return str(out)


def test_csv_loader_cases(csv_driver, tmp_path):
    res = subprocess.run([csv_driver, str(tmp_path)], capture_output=True, text=True, timeout=60)
    lines = dict(line.split(": ", 1) for line in res.stdout.strip().splitlines())
    for case in CASES:
        assert case in lines, res.stdout + res.stderr
        assert lines[case].startswith("ok"), f"{case}: {lines[case]}"
    assert res.returncode == 0
