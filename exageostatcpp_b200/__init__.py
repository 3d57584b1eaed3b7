"""B200 (sm_100a) ExaGeoStat maximum-likelihood path.

Python view of the C ABI declared in ``include/exageostat_b200.h``.  The compute
lives in ``libexageostat_b200.so`` (built in-tree by ``exageostatcpp_b200.build``);
this module only marshals numpy arrays through ctypes.  There is no CPU
fallback: if the shared library is missing, importing the bindings raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libexageostat_b200.so")

EGS_OK = 0
EGS_ERR_INVALID = -1
EGS_ERR_CUDA = -2
EGS_ERR_NO_DEVICE = -3
EGS_ERR_OOM = -4
EGS_ERR_TIMEOUT = -5
EGS_ERR_STATE = -6
EGS_PRECISION_DOUBLE = 1
EGS_PRECISION_MIXED = 2
EGS_BAND_OZAKI_INT8 = 0
EGS_BAND_FP64_DMMA = 1
EGS_REQ_LOGLIK = 1
EGS_REQ_FIT = 2
EGS_REQ_PREDICT = 3
EGS_FP64_REASON_NONE = 0
EGS_FP64_REASON_PREDICTED = 1
EGS_FP64_REASON_AFTER_FAILURE = 2

STAGES = ("generate", "panel", "update", "solve", "reduce", "update_low")
NUM_STAGES = len(STAGES)

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_LL = ctypes.POINTER(ctypes.c_longlong)
_P = ctypes.c_void_p

# name -> (restype, argtypes); every symbol of include/exageostat_b200.h.
SIGNATURES = {
    "egs_version": (ctypes.c_int, []),
    "egs_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "egs_last_error": (ctypes.c_char_p, []),
    "egs_hardware_init": (ctypes.c_int, [ctypes.c_int]),
    "egs_problem_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, ctypes.c_int]),
    "egs_problem_destroy": (ctypes.c_int, [_P]),
    "egs_problem_info": (ctypes.c_int, [_P, _I, _I, _I, _LL]),
    "egs_problem_set_stream": (ctypes.c_int, [_P, _P]),
    "egs_problem_set_band": (ctypes.c_int, [_P, ctypes.c_int]),
    "egs_problem_set_graphs": (ctypes.c_int, [_P, ctypes.c_int]),
    "egs_problem_set_precision": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
    "egs_problem_set_locations": (ctypes.c_int, [_P, _D, _D]),
    "egs_problem_set_locations_device": (ctypes.c_int, [_P, _P, _P]),
    "egs_problem_set_observations": (ctypes.c_int, [_P, _D]),
    "egs_problem_set_observations_device": (ctypes.c_int, [_P, _P]),
    "egs_covariance_generate": (ctypes.c_int, [_P, _D]),
    "egs_potrf": (ctypes.c_int, [_P]),
    "egs_restore_observations": (ctypes.c_int, [_P]),
    "egs_trsv": (ctypes.c_int, [_P]),
    "egs_loglik_parts": (ctypes.c_int, [_P, _D, _D, _D]),
    "egs_get_tile": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _D]),
    "egs_get_observations": (ctypes.c_int, [_P, _D]),
    "egs_mle_eval": (ctypes.c_int, [_P, _D, _D, _D, _D]),
    "egs_generate_locations": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D]),
    "egs_dlarnv_normal": (ctypes.c_int, [_I, ctypes.c_int, _D]),
    "egs_save_observations": (ctypes.c_int, [_P]),
    "egs_trsv_transpose": (ctypes.c_int, [_P]),
    "egs_set_tile": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _D]),
    "egs_sequence_create": (ctypes.c_int, [ctypes.POINTER(_P)]),
    "egs_sequence_wait": (ctypes.c_int, [_P]),
    "egs_sequence_destroy": (ctypes.c_int, [_P]),
    "egs_batch_set_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, _I, _D, _D, _D, ctypes.c_int, _I, _I]),
    "egs_batch_set_destroy": (ctypes.c_int, [_P]),
    "egs_batch_set_eval": (ctypes.c_int, [_P, _D, _D, _I]),
    "egs_batch_set_info": (ctypes.c_int, [_P, _I, _I, _I, ctypes.POINTER(ctypes.c_longlong)]),
    "egs_batch_set_autotune": (ctypes.c_int, [ctypes.c_int, _I, _D, _D, _D, _D, _I, ctypes.c_int, ctypes.c_int, _I,
                                              _I, _I, _D]),
    "egs_shuffle_split": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D, _D, _D]),
    "egs_generate_observations": (ctypes.c_int, [_P, _D, ctypes.c_int, _D]),
    "egs_mle_noalloc_workspace": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _LL]),
    "egs_mle_eval_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _P, _P, _P, _D, _P, ctypes.c_longlong, _D,
                                            _P]),
    "egs_problem_set_profiling": (ctypes.c_int, [_P, ctypes.c_int]),
    "egs_problem_stage_stats": (ctypes.c_int, [_P, _D, _D, _LL]),
    "egs_matern_block": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _D,
                                        ctypes.c_int, _P]),
    "egs_mle_loglik_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D]),
    "egs_predict_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D,
                                        _D, _D]),
    "egs_batch_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, _I, ctypes.c_int, _D, _D, _D]),
    "egs_batch_destroy": (ctypes.c_int, [_P]),
    "egs_batch_info": (ctypes.c_int, [_P, _I, _I, _LL, _LL]),
    "egs_batch_eval": (ctypes.c_int, [_P, _D, _D, _I]),
    "egs_batch_autotune": (ctypes.c_int, [ctypes.c_int, _I, _D, _D, _D, _D, _I, ctypes.c_int, _I, _D]),
    "egs_split_update": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _D]),
    "egs_problem_create_ex": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int]),
    "egs_problem_footprint": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _LL]),
    "egs_problem_predict": (ctypes.c_int, [_P, _D, ctypes.c_int, _D, _D, _D]),
    "egs_ozaki_band_update": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _D]),
    "egs_problem_set_band_method": (ctypes.c_int, [_P, ctypes.c_int]),
    "egs_problem_set_lookahead": (ctypes.c_int, [_P, ctypes.c_int]),
    "egs_mloe_mmom_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D, _D]),
    "egs_fisher_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D]),
}


class Request(ctypes.Structure):
    """egs_request of the serving API."""
    _fields_ = [("kind", ctypes.c_int), ("n", ctypes.c_int), ("dts", ctypes.c_int), ("precision", ctypes.c_int),
                ("band_tiles", ctypes.c_int), ("x", _D), ("y", _D), ("z", _D), ("theta", ctypes.c_double * 3),
                ("lb", ctypes.c_double * 3), ("ub", ctypes.c_double * 3), ("ftol_abs", ctypes.c_double),
                ("max_evals", ctypes.c_int), ("n_miss", ctypes.c_int), ("x_miss", _D), ("y_miss", _D)]


class Result(ctypes.Structure):
    """egs_result of the serving API."""
    _fields_ = [("status", ctypes.c_int), ("kind", ctypes.c_int), ("loglik", ctypes.c_double),
                ("theta", ctypes.c_double * 3), ("evals", ctypes.c_int), ("queue_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double), ("footprint", ctypes.c_longlong), ("precision_used", ctypes.c_int),
                ("fp64_reason", ctypes.c_int)]


SIGNATURES.update({
    "egs_server_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, ctypes.c_longlong, ctypes.c_int]),
    "egs_server_submit": (ctypes.c_int, [_P, ctypes.POINTER(Request), _LL]),
    "egs_server_wait": (ctypes.c_int, [_P, ctypes.c_longlong, ctypes.POINTER(Result), _D]),
    "egs_server_stats": (ctypes.c_int, [_P, _I, _I, _LL, _I, _LL, _LL, _LL]),
    "egs_server_destroy": (ctypes.c_int, [_P]),
    "egs_mixed_conditioning_estimate": (ctypes.c_int, [ctypes.c_int, _D, _D, _D, _D]),
})

OBJECTIVE = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_int, _D, ctypes.c_void_p)
SIGNATURES["egs_bobyqa_maximize"] = (ctypes.c_int, [ctypes.c_int, _D, _D, _D, ctypes.c_double, ctypes.c_double,
                                                    ctypes.c_int, OBJECTIVE, ctypes.c_void_p, _D, _I])

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the sm_100a library and declare every C ABI signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m exageostatcpp_b200.build`; "
                           "this package has no CPU fallback")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class EgsError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = load_library()
        msg = lib.egs_status_string(status).decode()
        detail = lib.egs_last_error().decode()
        super().__init__(f"{where}: {msg} ({status}) {detail}")
        self.status = status


class NotPositiveDefinite(EgsError):
    pass


def _check(status: int, where: str) -> None:
    if status == EGS_OK:
        return
    if status > 0:
        raise NotPositiveDefinite(status, where)
    raise EgsError(status, where)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Problem:
    """Device-resident problem of n locations (``egs_problem``)."""

    def __init__(self, n: int, dts: int, precision: int = 0, band_tiles: int = 0):
        """precision 0: FP64, switchable later with set_precision; EGS_PRECISION_*: created in that precision."""
        self._lib = load_library()
        self._h = _P()
        if precision:
            _check(self._lib.egs_problem_create_ex(ctypes.byref(self._h), int(n), int(dts), int(precision),
                                                   int(band_tiles)), "egs_problem_create_ex")
        else:
            _check(self._lib.egs_problem_create(ctypes.byref(self._h), int(n), int(dts)), "egs_problem_create")
        self.n = int(n)
        self.dts = int(dts)
        nn, ts, nt, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        self._lib.egs_problem_info(self._h, ctypes.byref(nn), ctypes.byref(ts), ctypes.byref(nt), ctypes.byref(nb))
        self.ts, self.nt, self.device_bytes = ts.value, nt.value, nb.value

    def close(self) -> None:
        if self._h:
            self._lib.egs_problem_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_graphs(self, enable: bool) -> None:
        """Replay evaluations as one CUDA graph (default on)."""
        _check(self._lib.egs_problem_set_graphs(self._h, 1 if enable else 0), "set_graphs")

    def set_band(self, band: int) -> None:
        """0: exact dense Cholesky; >= 1: diagonal super-tile approximation with this band."""
        _check(self._lib.egs_problem_set_band(self._h, int(band)), "set_band")

    def set_locations(self, x, y) -> None:
        x, y = _f64(x), _f64(y)
        assert x.size == self.n and y.size == self.n
        _check(self._lib.egs_problem_set_locations(self._h, _dptr(x), _dptr(y)), "set_locations")

    def set_observations(self, z) -> None:
        z = _f64(z)
        assert z.size == self.n
        _check(self._lib.egs_problem_set_observations(self._h, _dptr(z)), "set_observations")

    def generate(self, theta) -> None:
        th = _f64(theta)
        _check(self._lib.egs_covariance_generate(self._h, _dptr(th)), "covariance_generate")

    def potrf(self) -> None:
        _check(self._lib.egs_potrf(self._h), "potrf")

    def restore_observations(self) -> None:
        _check(self._lib.egs_restore_observations(self._h), "restore_observations")

    def trsv(self) -> None:
        _check(self._lib.egs_trsv(self._h), "trsv")

    def loglik_parts(self):
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(self._lib.egs_loglik_parts(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "loglik_parts")
        return a.value, b.value, c.value

    def tile(self, i: int, j: int) -> np.ndarray:
        out = np.empty((self.ts, self.ts), dtype=np.float64, order="F")
        _check(self._lib.egs_get_tile(self._h, i, j, out.ctypes.data_as(_D)), "get_tile")
        return out

    def lower_matrix(self) -> np.ndarray:
        """Assemble the stored lower tiles into an n x n lower-triangular array (tests)."""
        npad = self.nt * self.ts
        full = np.zeros((npad, npad))
        for j in range(self.nt):
            for i in range(j, self.nt):
                full[i * self.ts:(i + 1) * self.ts, j * self.ts:(j + 1) * self.ts] = self.tile(i, j)
        return np.tril(full)[: self.n, : self.n]

    def observations(self) -> np.ndarray:
        out = np.empty(self.n)
        _check(self._lib.egs_get_observations(self._h, _dptr(out)), "get_observations")
        return out

    def generate_observations(self, theta, seed: int) -> np.ndarray:
        """Z = L e at theta (the reference's synthetic observations); returns Z."""
        th = _f64(theta)
        z = np.empty(self.n)
        _check(self._lib.egs_generate_observations(self._h, _dptr(th), int(seed), _dptr(z)),
               "generate_observations")
        return z

    def set_profiling(self, enable: bool) -> None:
        _check(self._lib.egs_problem_set_profiling(self._h, 1 if enable else 0), "set_profiling")

    def stage_stats(self):
        """(ms[5], flops[5], launches[5]) per stage: generate, panel, update, solve, reduce."""
        ms = np.zeros(NUM_STAGES)
        fl = np.zeros(NUM_STAGES)
        ln = (ctypes.c_longlong * NUM_STAGES)()
        _check(self._lib.egs_problem_stage_stats(self._h, _dptr(ms), _dptr(fl), ln), "stage_stats")
        return ms, fl, np.array(list(ln), dtype=np.int64)

    def set_precision(self, precision: int, band_tiles: int = 0) -> None:
        """EGS_PRECISION_DOUBLE or EGS_PRECISION_MIXED (FP64 band of band_tiles tile rows)."""
        _check(self._lib.egs_problem_set_precision(self._h, int(precision), int(band_tiles)), "set_precision")
        nn, ts, nt, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        self._lib.egs_problem_info(self._h, ctypes.byref(nn), ctypes.byref(ts), ctypes.byref(nt), ctypes.byref(nb))
        self.ts, self.nt, self.bytes = ts.value, nt.value, nb.value

    def set_band_method(self, method: int) -> None:
        """EGS_BAND_OZAKI_INT8 (default) or EGS_BAND_FP64_DMMA for the FP64 band of a mixed problem."""
        _check(self._lib.egs_problem_set_band_method(self._h, int(method)), "set_band_method")

    def set_lookahead(self, sms: int) -> None:
        """SMs given to the look-ahead panel of a mixed problem (0: none); results do not change."""
        _check(self._lib.egs_problem_set_lookahead(self._h, int(sms)), "set_lookahead")

    def predict(self, theta, x_miss, y_miss) -> np.ndarray:
        """Kriging at the targets with the resident observations (either precision)."""
        th = _f64(theta)
        xm, ym = _f64(x_miss), _f64(y_miss)
        out = np.zeros(len(xm))
        _check(self._lib.egs_problem_predict(self._h, _dptr(th), len(xm), _dptr(xm), _dptr(ym), _dptr(out)),
               "predict")
        return out

    def set_stream(self, cuda_stream_handle) -> None:
        _check(self._lib.egs_problem_set_stream(self._h, _P(cuda_stream_handle)), "set_stream")

    def mle_eval(self, theta):
        th = _f64(theta)
        ll, ld, dt = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(self._lib.egs_mle_eval(self._h, _dptr(th), ctypes.byref(ll), ctypes.byref(ld), ctypes.byref(dt)),
               "mle_eval")
        return ll.value, ld.value, dt.value


def mle_loglik_host(x, y, z, theta, dts: int) -> float:
    lib = load_library()
    x, y, z, th = _f64(x), _f64(y), _f64(z), _f64(theta)
    out = ctypes.c_double()
    _check(lib.egs_mle_loglik_host(len(z), int(dts), _dptr(x), _dptr(y), _dptr(z), _dptr(th), ctypes.byref(out)),
           "mle_loglik_host")
    return out.value


def predict_host(x_obs, y_obs, z_obs, x_miss, y_miss, theta, dts: int, z_actual=None):
    lib = load_library()
    x_obs, y_obs, z_obs = _f64(x_obs), _f64(y_obs), _f64(z_obs)
    x_miss, y_miss, th = _f64(x_miss), _f64(y_miss), _f64(theta)
    nm = len(x_miss)
    zm = np.empty(nm)
    mspe = ctypes.c_double()
    za = _dptr(_f64(z_actual)) if z_actual is not None else None
    keep = _f64(z_actual) if z_actual is not None else None  # noqa: F841 (keeps the buffer alive)
    if keep is not None:
        za = _dptr(keep)
    _check(lib.egs_predict_host(len(z_obs), nm, int(dts), _dptr(x_obs), _dptr(y_obs), _dptr(z_obs), _dptr(x_miss),
                                _dptr(y_miss), za, _dptr(th), _dptr(zm), ctypes.byref(mspe)), "predict_host")
    return zm, mspe.value


def generate_locations(n: int, seed: int, reseed: bool = True):
    """The reference's synthetic locations (libc srand/rand, Morton sorted)."""
    lib = load_library()
    x, y = np.empty(n), np.empty(n)
    _check(lib.egs_generate_locations(int(n), int(seed), 1 if reseed else 0, _dptr(x), _dptr(y)),
           "generate_locations")
    return x, y


def shuffle_split(z, x, y, n_miss: int):
    """The reference's random hold-out split (PickRandomPoints): a Fisher-Yates
    shuffle on the C library's rand() state as it stands, the first n_miss held
    out.  Returns (z_obs, x_obs, y_obs, z_miss, x_miss, y_miss)."""
    lib = load_library()
    z, x, y = _f64(z), _f64(x), _f64(y)
    n = len(z)
    no = max(n - int(n_miss), 0)
    out = [np.empty(no) for _ in range(3)] + [np.empty(max(int(n_miss), 0)) for _ in range(3)]
    _check(lib.egs_shuffle_split(n, int(n_miss), _dptr(z), _dptr(x), _dptr(y), *(_dptr(a) for a in out)),
           "shuffle_split")
    return tuple(out)


def dlarnv_normal(seed: int, n: int) -> np.ndarray:
    """LAPACK DLARNV(3, {seed, seed, seed, 1}, n) restated in the library."""
    lib = load_library()
    iseed = (ctypes.c_int * 4)(seed, seed, seed, 1)
    out = np.empty(n)
    _check(lib.egs_dlarnv_normal(iseed, int(n), _dptr(out)), "dlarnv_normal")
    return out


def bobyqa_maximize(f, x0, lb, ub, ftol_abs: float, maxeval: int, rhobeg: float = 0.0):
    """Maximise f(theta) over the box with the library's BOBYQA; returns (theta, fbest, nevals)."""
    lib = load_library()
    x = _f64(x0).copy()
    lo, hi = _f64(lb), _f64(ub)
    err = []

    def cb(n, xp, ctx):
        try:
            return float(f(np.ctypeslib.as_array(xp, shape=(n,)).copy()))
        except Exception as exc:  # keep the exception for the caller; stop improving
            err.append(exc)
            return float("-inf")

    fn = OBJECTIVE(cb)
    fb = ctypes.c_double()
    ne = ctypes.c_int()
    _check(lib.egs_bobyqa_maximize(len(x), _dptr(x), _dptr(lo), _dptr(hi), float(rhobeg), float(ftol_abs),
                                   int(maxeval), fn, None, ctypes.byref(fb), ctypes.byref(ne)), "bobyqa_maximize")
    if err:
        raise err[0]
    return x, fb.value, ne.value


class Batch:
    """Many independent problems evaluated together (``egs_batch``).

    ``sizes[i]`` points of problem i; ``x``, ``y``, ``z`` are the problems'
    arrays concatenated in order.  ``eval(theta)`` takes a (B, 3) array and
    returns (loglik[B], status[B]); status[i] > 0 marks a problem whose
    covariance was not positive definite (its loglik is not meaningful)."""

    def __init__(self, sizes, x, y, z, dts: int):
        self._lib = load_library()
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int32)
        x, y, z = _f64(x), _f64(y), _f64(z)
        if not (len(x) == len(y) == len(z) == int(self.sizes.sum())):
            raise ValueError("x, y, z must hold sum(sizes) points")
        self.B = len(self.sizes)
        self._h = _P()
        _check(self._lib.egs_batch_create(ctypes.byref(self._h), self.B, self.sizes.ctypes.data_as(_I), int(dts),
                                          _dptr(x), _dptr(y), _dptr(z)), "egs_batch_create")

    def info(self):
        ts, ntm, nb, nl = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
        _check(self._lib.egs_batch_info(self._h, ctypes.byref(ts), ctypes.byref(ntm), ctypes.byref(nb),
                                        ctypes.byref(nl)), "egs_batch_info")
        return {"ts": ts.value, "nt_max": ntm.value, "bytes": nb.value, "launches_per_eval": nl.value}

    def eval(self, theta):
        th = _f64(np.broadcast_to(np.asarray(theta, dtype=np.float64), (self.B, 3)))
        ll = np.empty(self.B)
        st = np.zeros(self.B, dtype=np.int32)
        rc = self._lib.egs_batch_eval(self._h, _dptr(th), _dptr(ll), st.ctypes.data_as(_I))
        if rc not in (EGS_OK, EGS_ERR_STATE):
            _check(rc, "egs_batch_eval")
        return ll, st

    def close(self) -> None:
        if self._h:
            self._lib.egs_batch_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_autotune(sizes, x, y, z, theta, candidates=(128, 192, 256, 320)):
    """Fastest common tile size for a batch (one timed replay per candidate)."""
    lib = load_library()
    sizes = np.ascontiguousarray(sizes, dtype=np.int32)
    B = len(sizes)
    th = _f64(np.broadcast_to(np.asarray(theta, dtype=np.float64), (B, 3)))
    cand = np.ascontiguousarray(candidates, dtype=np.int32)
    best, ms = ctypes.c_int(), ctypes.c_double()
    _check(lib.egs_batch_autotune(B, sizes.ctypes.data_as(_I), _dptr(_f64(x)), _dptr(_f64(y)), _dptr(_f64(z)),
                                  _dptr(th), cand.ctypes.data_as(_I), len(cand), ctypes.byref(best),
                                  ctypes.byref(ms)), "egs_batch_autotune")
    return best.value, ms.value


class BatchSet:
    """A batch cut into size classes (``egs_batch_set``), each with its own tile
    size; the classes of one evaluation overlap on the device.  ``upper_n[c]`` is
    the largest N of class c; arguments as for :class:`Batch`."""

    def __init__(self, sizes, x, y, z, upper_n, dts):
        self._lib = load_library()
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int32)
        x, y, z = _f64(x), _f64(y), _f64(z)
        if not (len(x) == len(y) == len(z) == int(self.sizes.sum())):
            raise ValueError("x, y, z must hold sum(sizes) points")
        self.B = len(self.sizes)
        up = np.ascontiguousarray(upper_n, dtype=np.int32)
        ts = np.ascontiguousarray(dts, dtype=np.int32)
        self._h = _P()
        _check(self._lib.egs_batch_set_create(ctypes.byref(self._h), self.B, self.sizes.ctypes.data_as(_I), _dptr(x),
                                              _dptr(y), _dptr(z), len(up), up.ctypes.data_as(_I),
                                              ts.ctypes.data_as(_I)), "egs_batch_set_create")

    def info(self):
        nc = ctypes.c_int()
        up = np.zeros(16, dtype=np.int32)
        ts = np.zeros(16, dtype=np.int32)
        nb = ctypes.c_longlong()
        _check(self._lib.egs_batch_set_info(self._h, ctypes.byref(nc), up.ctypes.data_as(_I), ts.ctypes.data_as(_I),
                                            ctypes.byref(nb)), "egs_batch_set_info")
        return {"classes": nc.value, "upper_n": up[:nc.value].tolist(), "ts": ts[:nc.value].tolist(),
                "bytes": nb.value}

    def eval(self, theta):
        th = _f64(np.broadcast_to(np.asarray(theta, dtype=np.float64), (self.B, 3)))
        ll = np.empty(self.B)
        st = np.zeros(self.B, dtype=np.int32)
        rc = self._lib.egs_batch_set_eval(self._h, _dptr(th), _dptr(ll), st.ctypes.data_as(_I))
        if rc not in (EGS_OK, EGS_ERR_STATE):
            _check(rc, "egs_batch_set_eval")
        return ll, st

    def close(self) -> None:
        if self._h:
            self._lib.egs_batch_set_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_set_autotune(sizes, x, y, z, theta, candidates=(128, 192, 256, 320), max_classes=3):
    """Schedule of a batch: (upper_n list, tile list, ms per evaluation) of the fastest class split."""
    lib = load_library()
    sizes = np.ascontiguousarray(sizes, dtype=np.int32)
    B = len(sizes)
    th = _f64(np.broadcast_to(np.asarray(theta, dtype=np.float64), (B, 3)))
    cand = np.ascontiguousarray(candidates, dtype=np.int32)
    nc = ctypes.c_int()
    up = np.zeros(16, dtype=np.int32)
    ts = np.zeros(16, dtype=np.int32)
    ms = ctypes.c_double()
    _check(lib.egs_batch_set_autotune(B, sizes.ctypes.data_as(_I), _dptr(_f64(x)), _dptr(_f64(y)), _dptr(_f64(z)),
                                      _dptr(th), cand.ctypes.data_as(_I), len(cand), int(max_classes),
                                      ctypes.byref(nc), up.ctypes.data_as(_I), ts.ctypes.data_as(_I),
                                      ctypes.byref(ms)), "egs_batch_set_autotune")
    return up[:nc.value].tolist(), ts[:nc.value].tolist(), ms.value


def split_update(ts: int, nt: int, band: int, k: int, panel_ptr: int, offband_ptr: int) -> float:
    """egs_split_update on device pointers; returns the kernel's device milliseconds."""
    lib = load_library()
    ms = ctypes.c_double()
    _check(lib.egs_split_update(int(ts), int(nt), int(band), int(k), _P(panel_ptr), _P(offband_ptr),
                                ctypes.byref(ms)), "egs_split_update")
    return ms.value


def ozaki_band_update(ts: int, nt: int, band: int, k: int, w_ptr: int, band_ptr: int) -> float:
    """One Ozaki-scheme band update on device buffers (test entry); returns the kernel time in ms."""
    ms = ctypes.c_double()
    _check(load_library().egs_ozaki_band_update(int(ts), int(nt), int(band), int(k), _P(w_ptr), _P(band_ptr),
                                                ctypes.byref(ms)), "egs_ozaki_band_update")
    return ms.value


def mloe_mmom_host(x_obs, y_obs, x_miss, y_miss, theta_true, theta_est, dts: int):
    """(MLOE, MMOM) of kriging with theta_est when theta_true holds (egs_mloe_mmom_host)."""
    xo, yo, xm, ym = _f64(x_obs), _f64(y_obs), _f64(x_miss), _f64(y_miss)
    tt, te = _f64(theta_true), _f64(theta_est)
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(load_library().egs_mloe_mmom_host(len(xo), len(xm), int(dts), _dptr(xo), _dptr(yo), _dptr(xm), _dptr(ym),
                                             _dptr(tt), _dptr(te), ctypes.byref(a), ctypes.byref(b)),
           "egs_mloe_mmom_host")
    return a.value, b.value


def fisher_host(x, y, theta, dts: int) -> np.ndarray:
    """Inverse Fisher information (3 x 3) of (sigma^2, beta, nu) at theta (egs_fisher_host)."""
    xx, yy, th = _f64(x), _f64(y), _f64(theta)
    out = np.zeros(9)
    _check(load_library().egs_fisher_host(len(xx), int(dts), _dptr(xx), _dptr(yy), _dptr(th), _dptr(out)),
           "egs_fisher_host")
    return out.reshape(3, 3).T


def mixed_conditioning_estimate(x, y, theta) -> float:
    """The serving loop's condition estimate of the Matern covariance (host arithmetic)."""
    lib = load_library()
    x, y, th = _f64(x), _f64(y), _f64(theta)
    k = ctypes.c_double()
    _check(lib.egs_mixed_conditioning_estimate(len(x), _dptr(x), _dptr(y), _dptr(th), ctypes.byref(k)),
           "mixed_conditioning_estimate")
    return k.value


def footprint(n: int, dts: int, precision: int = EGS_PRECISION_DOUBLE, band_tiles: int = 0) -> int:
    """Device bytes of a problem of this shape (no device needed)."""
    b = ctypes.c_longlong()
    _check(load_library().egs_problem_footprint(int(n), int(dts), int(precision), int(band_tiles), ctypes.byref(b)),
           "footprint")
    return b.value


class Server:
    """The serving loop: queued requests admitted by HBM footprint, run concurrently."""

    def __init__(self, hbm_budget: int, max_active: int, device: int = 0):
        self._lib = load_library()
        h = _P()
        _check(self._lib.egs_server_create(ctypes.byref(h), int(device), int(hbm_budget), int(max_active)),
               "egs_server_create")
        self._h = h
        self._keep = {}

    def submit(self, kind, x, y, z, dts, theta=(1.0, 0.1, 0.5), precision=EGS_PRECISION_DOUBLE, band_tiles=0,
               lb=(0.01, 0.01, 0.01), ub=(5.0, 5.0, 5.0), ftol_abs=1e-9, max_evals=100, x_miss=None, y_miss=None):
        x, y, z = _f64(x), _f64(y), _f64(z)
        r = Request(kind=int(kind), n=len(z), dts=int(dts), precision=int(precision), band_tiles=int(band_tiles),
                    x=_dptr(x), y=_dptr(y), z=_dptr(z), ftol_abs=float(ftol_abs), max_evals=int(max_evals))
        r.theta[:] = list(theta)
        r.lb[:] = list(lb)
        r.ub[:] = list(ub)
        n_miss = 0
        if x_miss is not None:
            xm, ym = _f64(x_miss), _f64(y_miss)
            r.n_miss, r.x_miss, r.y_miss = len(xm), _dptr(xm), _dptr(ym)
            n_miss = len(xm)
        t = ctypes.c_longlong()
        _check(self._lib.egs_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)), "egs_server_submit")
        self._keep[t.value] = n_miss
        return t.value

    def wait(self, ticket: int):
        """(Result, predictions or None); raises nothing: the status is in the result."""
        n_miss = self._keep.pop(ticket)
        res = Result()
        out = np.zeros(max(n_miss, 1))
        _check(self._lib.egs_server_wait(self._h, int(ticket), ctypes.byref(res), _dptr(out)), "egs_server_wait")
        return res, (out[:n_miss] if n_miss else None)

    def stats(self) -> dict:
        q, a, pa = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        r, pr, c, e = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        _check(self._lib.egs_server_stats(self._h, ctypes.byref(q), ctypes.byref(a), ctypes.byref(r),
                                          ctypes.byref(pa), ctypes.byref(pr), ctypes.byref(c), ctypes.byref(e)),
               "egs_server_stats")
        return {"queued": q.value, "active": a.value, "reserved": r.value, "peak_active": pa.value,
                "peak_reserved": pr.value, "completed": c.value, "evals": e.value}

    def close(self) -> None:
        if self._h:
            self._lib.egs_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
