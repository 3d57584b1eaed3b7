"""Timed CPU baseline: the reference's log-likelihood evaluation restated on the host.

TEST INFRASTRUCTURE ONLY (the checker / CPU baseline, never the product).
Covariance generation runs in oracle/matern_cpu.c (OpenMP over all host
threads, the restatement of UnivariateMaternStationary.cpp:39-67); the Cholesky
factorisation, triangular solve and dot product use LAPACK/BLAS from scipy's
bundled OpenBLAS (multi-threaded), in place of Chameleon's tile algorithms
(ChameleonImplementation.cpp:113-265).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import time

import numpy as np
import scipy.linalg.lapack as lapack

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libegs_oracle.so")
PI = 3.141592653589793

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.egs_oracle_matern_lower.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _lib.egs_oracle_max_threads.restype = ctypes.c_int
    return _lib


def threads() -> int:
    return load().egs_oracle_max_threads()


def matern_lower(x, y, theta, a=None) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    n = len(x)
    if a is None:
        a = np.zeros((n, n), dtype=np.float64, order="F")
    load().egs_oracle_matern_lower(a.ctypes.data, n, n, x.ctypes.data, y.ctypes.data, th.ctypes.data, 0)
    return a


def timed_eval(x, y, z, theta, a=None):
    """One log-likelihood evaluation on the host; returns (loglik, seconds per stage)."""
    n = len(z)
    t0 = time.perf_counter()
    a = matern_lower(x, y, theta, a)
    t1 = time.perf_counter()
    c, info = lapack.dpotrf(a, lower=1, clean=0, overwrite_a=1)
    if info != 0:
        raise np.linalg.LinAlgError("Matrix is not positive definite")
    t2 = time.perf_counter()
    d = np.diag(c)
    logdet = 2.0 * float(np.sum(np.log(d[d > 0])))
    w, info = lapack.dtrtrs(c, np.asarray(z, dtype=np.float64), lower=1)
    dot = float(w @ w)
    t3 = time.perf_counter()
    loglik = -0.5 * dot - 0.5 * logdet - (n / 2.0) * math.log(2.0 * PI)
    return loglik, {"generate": t1 - t0, "potrf": t2 - t1, "solve": t3 - t2}


def scaled_evals_per_s(stage_s: dict, n_sample: int, n_target: int) -> float:
    """Scale a sample evaluation to n_target: generation and solve ~ n^2, potrf ~ n^3."""
    r = n_target / n_sample
    t = (stage_s["generate"] + stage_s["solve"]) * r * r + stage_s["potrf"] * r ** 3
    return 1.0 / t
