"""Timed CPU baseline: the reference's log-likelihood evaluation restated on the host.

TEST INFRASTRUCTURE ONLY (the checker / CPU baseline, never the product).
Covariance generation runs in oracle/matern_cpu.c (POSIX threads over all host
threads, the restatement of UnivariateMaternStationary.cpp:39-67); the Cholesky
factorisation and triangular solves are blocked (tile) algorithms on the
multi-threaded OpenBLAS bundled with numpy, in place of Chameleon's tile
algorithms (ChameleonImplementation.cpp:113-265).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import time

import numpy as np

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
        _lib.egs_oracle_matern_block.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _lib.egs_oracle_max_threads.restype = ctypes.c_int
    return _lib


# --------------------------------------------------------------------------
# Blocked FP64 Cholesky and triangular solves on numpy's bundled OpenBLAS
# (64-bit integer interface), called through ctypes on sub-blocks of one
# column-major matrix, in place.  This restates Chameleon's tile algorithm
# behind CHAMELEON_dpotrf_Tile (ChameleonDense.cpp:25-37): per block column,
# potrf of the diagonal block, trsm of the blocks below it, syrk/gemm of the
# trailing block columns.  Every call sees operands of at most n x nb elements:
# OpenBLAS's multi-threaded syrk (inside its dpotrf) faults on whole-matrix
# operands from n of about 36,000, and the whole-matrix calls are what the
# reference's tile algorithm never makes either.
# --------------------------------------------------------------------------
_blas = None
_I64 = ctypes.c_int64


def _blas64():
    global _blas
    if _blas is None:
        import glob
        libdir = os.path.join(os.path.dirname(np.__file__), os.pardir, "numpy.libs")
        cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas64_*.so")))
        if not cands:
            raise RuntimeError("numpy's bundled 64-bit-integer OpenBLAS not found")
        _blas = ctypes.CDLL(cands[0])
    return _blas


def _i(v):
    return ctypes.byref(_I64(int(v)))


def _d(v):
    return ctypes.byref(ctypes.c_double(float(v)))


def _ch(c):
    return ctypes.c_char_p(c)


_ONE = ctypes.c_size_t(1)


def potrf_blocked(a: np.ndarray, nb: int = 2048) -> int:
    """Lower Cholesky factor of the F-ordered square a in place (its strict upper
    part is not read); returns 0 or the LAPACK info of the failing pivot."""
    lib = _blas64()
    n = a.shape[0]
    assert a.flags["F_CONTIGUOUS"] and a.dtype == np.float64 and a.shape == (n, n)
    base, lda = a.ctypes.data, n

    def p(i, j):
        return ctypes.c_void_p(base + 8 * (i + j * lda))

    info = _I64(0)
    for k0 in range(0, n, nb):
        kb = min(nb, n - k0)
        lib.scipy_dpotrf_64_(_ch(b"L"), _i(kb), p(k0, k0), _i(lda), ctypes.byref(info), _ONE)
        if info.value != 0:
            return k0 + info.value
        m = n - k0 - kb
        if m == 0:
            break
        lib.scipy_dtrsm_64_(_ch(b"R"), _ch(b"L"), _ch(b"T"), _ch(b"N"), _i(m), _i(kb), _d(1.0), p(k0, k0),
                            _i(lda), p(k0 + kb, k0), _i(lda), _ONE, _ONE, _ONE, _ONE)
        for j0 in range(k0 + kb, n, nb):
            jb = min(nb, n - j0)
            lib.scipy_dsyrk_64_(_ch(b"L"), _ch(b"N"), _i(jb), _i(kb), _d(-1.0), p(j0, k0), _i(lda), _d(1.0),
                                p(j0, j0), _i(lda), _ONE, _ONE)
            r = n - j0 - jb
            if r:
                lib.scipy_dgemm_64_(_ch(b"N"), _ch(b"T"), _i(r), _i(jb), _i(kb), _d(-1.0), p(j0 + jb, k0),
                                    _i(lda), p(j0, k0), _i(lda), _d(1.0), p(j0 + jb, j0), _i(lda), _ONE, _ONE)
    return 0


def trsv_blocked(c: np.ndarray, z, transpose: bool = False, nb: int = 2048) -> np.ndarray:
    """L^-1 z (or L^-T z) for the lower factor c from potrf_blocked, by blocks."""
    lib = _blas64()
    n = c.shape[0]
    base, lda = c.ctypes.data, n
    v = np.array(z, dtype=np.float64, copy=True)
    vb = v.ctypes.data

    def p(i, j):
        return ctypes.c_void_p(base + 8 * (i + j * lda))

    def q(i):
        return ctypes.c_void_p(vb + 8 * i)

    starts = list(range(0, n, nb))
    for k0 in (reversed(starts) if transpose else starts):
        kb = min(nb, n - k0)
        m = n - k0 - kb
        if transpose and m:
            lib.scipy_dgemv_64_(_ch(b"T"), _i(m), _i(kb), _d(-1.0), p(k0 + kb, k0), _i(lda), q(k0 + kb), _i(1),
                                _d(1.0), q(k0), _i(1), _ONE)
        lib.scipy_dtrsv_64_(_ch(b"L"), _ch(b"T" if transpose else b"N"), _ch(b"N"), _i(kb), p(k0, k0), _i(lda),
                            q(k0), _i(1), _ONE, _ONE, _ONE)
        if not transpose and m:
            lib.scipy_dgemv_64_(_ch(b"N"), _i(m), _i(kb), _d(-1.0), p(k0 + kb, k0), _i(lda), q(k0), _i(1),
                                _d(1.0), q(k0 + kb), _i(1), _ONE)
    return v


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


def matern_block(x1, y1, x2, y2, theta) -> np.ndarray:
    """C(i, j) between row locations (x1, y1) and column locations (x2, y2) (C12 of the kriging)."""
    x1, y1, x2, y2 = (np.ascontiguousarray(v, dtype=np.float64) for v in (x1, y1, x2, y2))
    th = np.ascontiguousarray(theta, dtype=np.float64)
    a = np.empty((len(x1), len(x2)), dtype=np.float64, order="F")
    load().egs_oracle_matern_block(a.ctypes.data, len(x1), len(x1), len(x2), x1.ctypes.data, y1.ctypes.data,
                                   x2.ctypes.data, y2.ctypes.data, th.ctypes.data, 0)
    return a


def eval_and_predict(x_obs, y_obs, z_obs, x_miss, y_miss, theta, z_actual=None):
    """Log-likelihood of the observed set and kriging of the targets from ONE factorisation.

    The kriging's C22 (LinearAlgebraMethods.cpp:527-544) is the covariance
    matrix of the evaluation at the same theta (ChameleonImplementation.cpp:113-265),
    so one generation and one dpotrf serve both: logdet and dot as in
    timed_eval, w = C22^-1 z by the two triangular solves of dposv,
    z_miss = C12 w (:552) and mspe = mean((z_actual - z_miss)^2) (:567-577),
    -1 without the truth (:579-581).
    Returns (loglik, logdet, dot, z_miss, mspe, seconds per stage)."""
    n = len(z_obs)
    t0 = time.perf_counter()
    a = matern_lower(x_obs, y_obs, theta)
    t1 = time.perf_counter()
    if potrf_blocked(a) != 0:
        raise np.linalg.LinAlgError("Matrix is not positive definite")
    t2 = time.perf_counter()
    d = np.diag(a)
    logdet = 2.0 * float(np.sum(np.log(d[d > 0])))
    v = trsv_blocked(a, z_obs)
    dot = float(v @ v)
    w = trsv_blocked(a, v, transpose=True)
    t3 = time.perf_counter()
    del a
    c12 = matern_block(x_miss, y_miss, x_obs, y_obs, theta)
    z_miss = c12 @ w
    t4 = time.perf_counter()
    loglik = -0.5 * dot - 0.5 * logdet - (n / 2.0) * math.log(2.0 * PI)
    mspe = -1.0 if z_actual is None else float(np.sum((np.asarray(z_actual) - z_miss) ** 2)) / len(z_miss)
    return loglik, logdet, dot, z_miss, mspe, {"generate": t1 - t0, "potrf": t2 - t1, "solve": t3 - t2,
                                               "predict": t4 - t3}


def timed_eval(x, y, z, theta, a=None):
    """One log-likelihood evaluation on the host; returns (loglik, seconds per stage)."""
    n = len(z)
    t0 = time.perf_counter()
    a = matern_lower(x, y, theta, a)
    t1 = time.perf_counter()
    if potrf_blocked(a) != 0:
        raise np.linalg.LinAlgError("Matrix is not positive definite")
    t2 = time.perf_counter()
    d = np.diag(a)
    logdet = 2.0 * float(np.sum(np.log(d[d > 0])))
    w = trsv_blocked(a, z)
    dot = float(w @ w)
    t3 = time.perf_counter()
    loglik = -0.5 * dot - 0.5 * logdet - (n / 2.0) * math.log(2.0 * PI)
    return loglik, {"generate": t1 - t0, "potrf": t2 - t1, "solve": t3 - t2}


def timed_eval_parts(x, y, z, theta):
    """(loglik, logdet, dot) of one host evaluation (the pieces of timed_eval)."""
    n = len(z)
    a = matern_lower(x, y, theta)
    if potrf_blocked(a) != 0:
        raise np.linalg.LinAlgError("Matrix is not positive definite")
    d = np.diag(a)
    logdet = 2.0 * float(np.sum(np.log(d[d > 0])))
    w = trsv_blocked(a, z)
    dot = float(w @ w)
    return -0.5 * dot - 0.5 * logdet - (n / 2.0) * math.log(2.0 * PI), logdet, dot


def scaled_evals_per_s(stage_s: dict, n_sample: int, n_target: int) -> float:
    """Scale a sample evaluation to n_target: generation and solve ~ n^2, potrf ~ n^3."""
    r = n_target / n_sample
    t = (stage_s["generate"] + stage_s["solve"]) * r * r + stage_s["potrf"] * r ** 3
    return 1.0 / t
