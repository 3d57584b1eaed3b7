"""The end-to-end example program of the C++ API (host/examples/end_to_end.cpp), on the CPU.

Without a GPU the program must stop with the library's error rather than
compute anything on the host (there is no CPU path), and a flag value the
reference rejects must be reported before any device work.  On a machine with
a visible CUDA device these checks do not apply and the test is skipped.
"""
import os
import subprocess

import pytest


def _example():
    from exageostatcpp_b200 import build as b
    if not os.path.exists(b.EXAMPLE_BIN):
        b.build_example()
    return b.EXAMPLE_BIN


def _gpu_visible():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_visible(), reason="a CUDA device is visible: the example would run")
def test_example_fails_loudly_without_a_gpu():
    exe = _example()
    args = ["--N=1600", "--dts=320", "--kernel=univariate_matern_stationary", "--itheta=1:0.1:0.5",
            "--lb=0.1:0.01:0.01", "--ub=5:5:5", "--tolerance=4", "--max_mle_iterations=20", "--zmiss=10",
            "--mspe=true", "--precision=mixed"]
    res = subprocess.run([exe, *args], capture_output=True, text=True, timeout=120)
    assert res.returncode == 1
    assert "no CUDA device" in res.stderr
    assert res.stdout == ""


@pytest.mark.skipif(_gpu_visible(), reason="a CUDA device is visible: the example would run")
def test_example_reports_invalid_flags_first():
    res = subprocess.run([_example(), "--precision=quad"], capture_output=True, text=True, timeout=60)
    assert res.returncode == 1
    assert "Invalid value for Computation. Please use Single, Double or Mixed." in res.stderr
