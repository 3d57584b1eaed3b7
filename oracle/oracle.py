"""CPU restatement of ExaGeoStatCPP's Gaussian maximum-likelihood path.

TEST INFRASTRUCTURE ONLY -- this module is the checker, never the product.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import it.  The product package does not import it and has no CPU
fallback.

Every function cites the reference file:line whose behaviour it restates
(paths are relative to the ExaGeoStatCPP source tree).  Third-party arithmetic
at the boundary is handled as follows:

* glibc ``rand()`` (TYPE_3 additive-feedback generator) is restated in
  :class:`GlibcRand` and cross-checked against the C library through ctypes.
* LAPACK ``dlarnv`` (idist=3, Box-Muller over ``dlaruv``) is *called* from the
  OpenBLAS build bundled with scipy (exported symbol ``scipy_dlarnv_``).
* GSL 2.7.1 ``gsl_sf_bessel_Knu`` (absent from the reference tree) is replaced
  by ``scipy.special.kv`` (AMOS); ``mpmath.besselk`` is the high-precision
  referee in the tests.
* Chameleon ``dpotrf``/``dtrsm``/``dposv``/``dgemm`` are replaced by LAPACK via
  scipy; their results are mathematically unique.

Parity is pinned by the golden vectors of the reference's own tests (see
``tests/golden/reference_goldens.json``).
"""
from __future__ import annotations

import ctypes
import glob
import math
import os

import numpy as np
import scipy.linalg
import scipy.special

PI = 3.141592653589793  # inst/include/common/Definitions.hpp:45


# --------------------------------------------------------------------------
# glibc rand(): srand/rand, TYPE_3 (degree 31, separation 3) additive feedback
# Used by LocationGenerator.cpp:84-89 and PredictionHelpers.cpp:146.
# --------------------------------------------------------------------------
class GlibcRand:
    """Restatement of glibc's default ``random()`` state machine.

    Seeding fills r[0..30] with a Lehmer (Park-Miller, multiplier 16807)
    sequence, copies r[0..2] into r[31..33], then runs the lagged recurrence
    r[i] = r[i-31] + r[i-3] (mod 2**32); outputs start at i = 344 and are
    ``r[i] >> 1``.  ``srand(0)`` behaves like ``srand(1)``.
    """

    RAND_MAX = 2147483647

    def __init__(self, seed: int = 1):
        self.srand(seed)

    def srand(self, seed: int) -> None:
        seed &= 0xFFFFFFFF
        if seed == 0:
            seed = 1
        r = [0] * 34
        r[0] = seed
        for i in range(1, 31):
            # Schrage's factorisation keeps the product in 32-bit signed range.
            hi, lo = divmod(r[i - 1] if r[i - 1] < 2**31 else r[i - 1] - 2**32, 127773)
            word = 16807 * lo - 2836 * hi
            if word < 0:
                word += 2147483647
            r[i] = word & 0xFFFFFFFF
        for i in range(31, 34):
            r[i] = r[i - 31]
        self._r = r
        # discard the first 310 outputs
        for _ in range(310):
            self._step()

    def _step(self) -> int:
        r = self._r
        v = (r[-31] + r[-3]) & 0xFFFFFFFF
        r.append(v)
        if len(r) > 64:
            del r[:-34]
        return v

    def rand(self) -> int:
        return self._step() >> 1


def libc_rand_sequence(seed: int, count: int) -> list[int]:
    """The C library's own srand/rand, used only to cross-check GlibcRand."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(ctypes.c_uint(seed))
    return [libc.rand() for _ in range(count)]


# --------------------------------------------------------------------------
# Morton ordering: src/helpers/ByteHandler.cpp:19-47
# --------------------------------------------------------------------------
def spread_bits(v):
    """Interleave the low 16 bits of v with three zero bits (ByteHandler.cpp:19-32)."""
    v = np.asarray(v, dtype=np.uint64) & np.uint64(0xFFFF)
    v = (v ^ (v << np.uint64(24))) & np.uint64(0x000000FF000000FF)
    v = (v ^ (v << np.uint64(12))) & np.uint64(0x000F000F000F000F)
    v = (v ^ (v << np.uint64(6))) & np.uint64(0x0303030303030303)
    v = (v ^ (v << np.uint64(3))) & np.uint64(0x1111111111111111)
    return v


def reverse_spread_bits(v):
    """Inverse of :func:`spread_bits` (ByteHandler.cpp:34-47)."""
    v = np.asarray(v, dtype=np.uint64) & np.uint64(0x1111111111111111)
    v = (v ^ (v >> np.uint64(3))) & np.uint64(0x0303030303030303)
    v = (v ^ (v >> np.uint64(6))) & np.uint64(0x000F000F000F000F)
    v = (v ^ (v >> np.uint64(12))) & np.uint64(0x000000FF000000FF)
    v = (v ^ (v >> np.uint64(24))) & np.uint64(0x000000000000FFFF)
    return v


# --------------------------------------------------------------------------
# Synthetic locations: src/data-generators/LocationGenerator.cpp:25-123
# --------------------------------------------------------------------------
def generate_locations(n: int, rng: GlibcRand) -> tuple[np.ndarray, np.ndarray]:
    """Jittered grid in [0,1]^2, Morton sorted, coordinates 16-bit quantised.

    rootN = ceil(sqrt(n)); point (i, j) (i outer) is
    ((i+1) - 0.5 + U(-0.4, 0.4)) / rootN, with U = rand()/(1+RAND_MAX)*0.8-0.4
    (LocationGenerator.cpp:33-71, 84-89).  SortLocations (:91-123) quantises to
    uint16 with +0.5 rounding, sorts the Morton codes and REPLACES the
    coordinates by the quantised values / 65535.
    """
    root_n = int(math.ceil(math.sqrt(n)))
    xs = np.empty(n)
    ys = np.empty(n)
    idx = 0
    inv = 1.0 / (1.0 + GlibcRand.RAND_MAX)
    for i in range(root_n):
        if idx >= n:
            break
        for j in range(root_n):
            if idx >= n:
                break
            ux = rng.rand() * inv * 0.8 + (-0.4)
            xs[idx] = ((i + 1) - 0.5 + ux) / root_n
            uy = rng.rand() * inv * 0.8 + (-0.4)
            ys[idx] = ((j + 1) - 0.5 + uy) / root_n
            idx += 1
    qx = (xs * 65535.0 + 0.5).astype(np.uint64) & np.uint64(0xFFFF)
    qy = (ys * 65535.0 + 0.5).astype(np.uint64) & np.uint64(0xFFFF)
    code = (spread_bits(qy) << np.uint64(1)) + spread_bits(qx)
    code.sort()
    x = reverse_spread_bits(code).astype(np.float64) / 65535.0
    y = reverse_spread_bits(code >> np.uint64(1)).astype(np.float64) / 65535.0
    return x, y


# --------------------------------------------------------------------------
# LAPACK dlarnv(3, iseed, n): LinearAlgebraMethods.cpp:347-364
# --------------------------------------------------------------------------
_openblas = None


def _load_openblas():
    global _openblas
    if _openblas is None:
        libdir = os.path.join(os.path.dirname(scipy.__file__), os.pardir, "scipy.libs")
        cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
        if not cands:
            raise RuntimeError("scipy's bundled OpenBLAS not found")
        _openblas = ctypes.CDLL(cands[0])
    return _openblas


def dlarnv_normal(seed: int, n: int) -> np.ndarray:
    """N(0,1) samples from LAPACK dlarnv with ISEED = {seed, seed, seed, 1}."""
    lib = _load_openblas()
    idist = ctypes.c_int(3)
    iseed = (ctypes.c_int * 4)(seed, seed, seed, 1)
    out = np.empty(n, dtype=np.float64)
    nn = ctypes.c_int(n)
    lib.scipy_dlarnv_(ctypes.byref(idist), iseed, ctypes.byref(nn),
                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


# --------------------------------------------------------------------------
# Matern covariance: src/kernels/concrete/UnivariateMaternStationary.cpp:39-67
# --------------------------------------------------------------------------
def matern_block(x1, y1, x2, y2, theta) -> np.ndarray:
    """C[i, j] = sigma2 / (2^(nu-1) Gamma(nu)) * (d/beta)^nu * K_nu(d/beta), = sigma2 at d == 0.

    theta = (sigma2, beta, nu) (UnivariateMaternStationary.cpp:47-49, 61-62);
    d is the Euclidean distance (DistanceCalculationHelpers.cpp:38-57, metric 0).
    """
    sigma2, beta, nu = float(theta[0]), float(theta[1]), float(theta[2])
    x1 = np.asarray(x1, dtype=np.float64)[:, None]
    y1 = np.asarray(y1, dtype=np.float64)[:, None]
    x2 = np.asarray(x2, dtype=np.float64)[None, :]
    y2 = np.asarray(y2, dtype=np.float64)[None, :]
    dx = x2 - x1
    dy = y2 - y1
    dist = np.sqrt(dx * dx + dy * dy) / beta
    con = sigma2 * (1.0 / (math.pow(2.0, nu - 1.0) * math.gamma(nu)))
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        val = con * np.power(dist, nu) * scipy.special.kv(nu, dist)
    return np.where(dist == 0.0, sigma2, val)


def covariance(x, y, theta) -> np.ndarray:
    return matern_block(x, y, x, y, theta)


# --------------------------------------------------------------------------
# Synthetic observations: LinearAlgebraMethods.cpp:333-449  (Z = L e)
# --------------------------------------------------------------------------
def generate_observations(x, y, theta, seed: int) -> np.ndarray:
    n = len(x)
    e = dlarnv_normal(seed, n)
    c = covariance(x, y, theta)
    L = cholesky_lower(c)
    return L @ e


def load_data(n: int, seed: int, theta) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """ExaGeoStat::ExaGeoStatLoadData for synthetic data (src/api/ExaGeoStat.cpp:72-88):
    srand(seed), locations, then Z at the initial theta."""
    rng = GlibcRand(seed)
    x, y = generate_locations(n, rng)
    z = generate_observations(x, y, theta, seed)
    return x, y, z


# --------------------------------------------------------------------------
# One log-likelihood evaluation:
# ChameleonImplementation.cpp:113-265, dmdet-codelet.cpp:73-80, ddotp-codelet.cpp:63-72
# --------------------------------------------------------------------------
def cholesky_lower(c: np.ndarray) -> np.ndarray:
    """LAPACK dpotrf; a NaN or non-positive pivot raises like ChameleonDense.cpp:29-32."""
    L = scipy.linalg.cholesky(c, lower=True, check_finite=False)
    if not np.all(np.isfinite(np.diag(L))) or not np.all(np.diag(L) > 0):
        raise np.linalg.LinAlgError("Matrix is not positive definite")
    return L


def mle_loglik(x, y, z, theta, return_parts: bool = False):
    n = len(z)
    c = covariance(x, y, theta)
    L = cholesky_lower(c)
    d = np.diag(L)
    logdet = 2.0 * float(np.sum(np.log(d[d > 0])))
    w = scipy.linalg.solve_triangular(L, np.asarray(z, dtype=np.float64), lower=True,
                                      check_finite=False)
    dot = float(w @ w)
    loglik = -0.5 * dot - 0.5 * logdet - (n / 2.0) * math.log(2.0 * PI)
    if return_parts:
        return loglik, logdet, dot
    return loglik


def dst_loglik(x, y, z, theta, ts: int, band: int, return_parts: bool = False):
    """Log-likelihood with the diagonal super-tile (band) factorisation.

    Follows ChameleonDST<T>::ExaGeoStatParallelPotrfDiagonal
    (src/linear-algebra-solvers/concrete/chameleon/dst/ChameleonDST.cpp:90-150) for
    the lower case: at step k, potrf of tile (k,k); trsm of tiles (m,k) for
    k < m < k+band; syrk of (n,n) and gemm of (m,n) for k < n < k+band,
    n < m < n+band, reading tile (m,k) whether solved or not.  The rest of the
    evaluation (log-det over diagonal tiles, Z := L^-1 Z over the whole lower
    triangle, dot) is ChameleonImplementation.cpp:180-265 unchanged.
    """
    n = len(z)
    A = np.tril(covariance(x, y, theta)).copy()
    nt = -(-n // ts)
    blk = lambda i: slice(i * ts, min(n, (i + 1) * ts))  # noqa: E731
    for k in range(nt):
        try:
            A[blk(k), blk(k)] = cholesky_lower(A[blk(k), blk(k)])
        except (np.linalg.LinAlgError, ValueError) as exc:
            raise np.linalg.LinAlgError("Matrix is not positive definite") from exc
        for m in range(k + 1, min(nt, k + band)):
            A[blk(m), blk(k)] = scipy.linalg.solve_triangular(A[blk(k), blk(k)], A[blk(m), blk(k)].T,
                                                              lower=True).T
        for c in range(k + 1, min(nt, k + band)):
            A[blk(c), blk(c)] -= np.tril(A[blk(c), blk(k)] @ A[blk(c), blk(k)].T)
            for m in range(c + 1, min(nt, c + band)):
                A[blk(m), blk(c)] -= A[blk(m), blk(k)] @ A[blk(c), blk(k)].T
    L = np.tril(A)
    d = np.diag(L)
    logdet = 2.0 * float(np.sum(np.log(d[d > 0])))
    w = scipy.linalg.solve_triangular(L, np.asarray(z, dtype=np.float64), lower=True, check_finite=False)
    dot = float(w @ w)
    loglik = -0.5 * dot - 0.5 * logdet - (n / 2.0) * math.log(2.0 * PI)
    return (loglik, logdet, dot) if return_parts else loglik


# --------------------------------------------------------------------------
# Random hold-out split: PredictionHelpers.cpp:23-168 (Shuffle :140-168)
# --------------------------------------------------------------------------
def shuffle_split(z, x, y, n_miss: int, rng: GlibcRand):
    """Fisher-Yates with j = i + rand() / (RAND_MAX/(n-i) + 1); first n_miss are held out.

    SortInplace (PredictionHelpers.cpp:249-326) leaves the order unchanged.
    Returns (z_obs, x_obs, y_obs, z_actual, x_miss, y_miss)."""
    z = np.array(z, dtype=np.float64)
    x = np.array(x, dtype=np.float64)
    y = np.array(y, dtype=np.float64)
    n = len(z)
    if n > 1:
        for i in range(n - 1):
            j = i + rng.rand() // (GlibcRand.RAND_MAX // (n - i) + 1)
            z[i], z[j] = z[j], z[i]
            x[i], x[j] = x[j], x[i]
            y[i], y[j] = y[j], y[i]
    return (z[n_miss:], x[n_miss:], y[n_miss:], z[:n_miss], x[:n_miss], y[:n_miss])


# --------------------------------------------------------------------------
# Kriging: LinearAlgebraMethods.cpp:451-605
# --------------------------------------------------------------------------
def predict(x_obs, y_obs, z_obs, x_miss, y_miss, theta, z_actual=None):
    """C22 (obs x obs) Cholesky solve, Zmiss = C12 * (C22^-1 Zobs), MSPE = mean((Zactual - Zmiss)^2).

    Returns (z_miss, mspe) where mspe is -1 without z_actual (:579-581)."""
    c22 = covariance(x_obs, y_obs, theta)
    c12 = matern_block(x_miss, y_miss, x_obs, y_obs, theta)
    cf = scipy.linalg.cho_factor(c22, lower=True, check_finite=False)
    w = scipy.linalg.cho_solve(cf, np.asarray(z_obs, dtype=np.float64), check_finite=False)
    z_miss = c12 @ w
    if z_actual is None:
        return z_miss, -1.0
    err = float(np.sum((np.asarray(z_actual) - z_miss) ** 2))
    return z_miss, err / len(z_miss)


def flops_potrf(n: float) -> float:
    """Chameleon's flops_dpotrf for real arithmetic: n^3/3 + n^2/2 + n/6."""
    return n ** 3 / 3.0 + n ** 2 / 2.0 + n / 6.0


# --------------------------------------------------------------------------
# MLOE / MMOM: LinearAlgebraMethods.cpp:802-1131, dmloe-mmom-codelet.cpp:73-102
# --------------------------------------------------------------------------
def mloe_mmom(x_obs, y_obs, x_miss, y_miss, theta_true, theta_est):
    """Mean loss of efficiency and mean misspecification of the mean square error
    of kriging with theta_est when theta_true holds, over the target points.

    Per target p, with k_t, k_a the covariances between the observed points
    and target p under theta_true / theta_est and K_t, K_a the observed
    covariance matrices (univariate: alpha = sigma^2):
        w_a   = K_a^-1 k_a
        e2    = sigma2_t - 2 k_t.w_a + w_a' K_t w_a    (MSE of the misspecified predictor)
        e3    = sigma2_t - k_t' K_t^-1 k_t               (MSE of the right predictor)
        e4    = sigma2_a - k_a' K_a^-1 k_a               (MSE the misspecified model claims)
        loe_p = e2 / e3 - 1,  mom_p = e4 / e2 - 1  (both -1 when e3 == 0)
    and MLOE, MMOM are the means over the targets."""
    kt_all = matern_block(x_obs, y_obs, x_miss, y_miss, theta_true)
    ka_all = matern_block(x_obs, y_obs, x_miss, y_miss, theta_est)
    Kt = covariance(x_obs, y_obs, theta_true)
    Ka = covariance(x_obs, y_obs, theta_est)
    ct = scipy.linalg.cho_factor(Kt, lower=True, check_finite=False)
    ca = scipy.linalg.cho_factor(Ka, lower=True, check_finite=False)
    s2t, s2a = float(theta_true[0]), float(theta_est[0])
    loe = mom = 0.0
    m = kt_all.shape[1]
    for p in range(m):
        kt, ka = kt_all[:, p], ka_all[:, p]
        wa = scipy.linalg.cho_solve(ca, ka, check_finite=False)
        e2 = s2t - 2.0 * kt @ wa + wa @ (Kt @ wa)
        e3 = s2t - kt @ scipy.linalg.cho_solve(ct, kt, check_finite=False)
        e4 = s2a - ka @ wa
        if e3 == 0.0:
            loe -= 1.0
            mom -= 1.0
        else:
            loe += e2 / e3 - 1.0
            mom += e4 / e2 - 1.0
    return loe / m, mom / m


# --------------------------------------------------------------------------
# Fisher information: LinearAlgebraMethods.cpp:1133-1306 with the derivative
# kernels UnivariateMaternDdsigmaSquare / Dbeta / Dnu
# (src/kernels/concrete/UnivariateMaternD*.cpp) and BasselFunction.cpp:23-33.
# --------------------------------------------------------------------------
def dkv_dnu(nu: float, x: np.ndarray) -> np.ndarray:
    """d K_nu(x) / d nu from K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt:
    d/dnu = int_0^inf t sinh(nu t) exp(-x cosh t) dt.  The integrand is smooth and
    decays double-exponentially, so the trapezoid rule on a fine grid converges
    to full double precision (checked against mpmath.diff(besselk) in the tests).
    The reference takes a forward difference with step 1e-9
    (BasselFunction.cpp:23-33), which carries ~1e-7 relative rounding noise."""
    xs = np.asarray(x, dtype=np.float64)
    flat = xs.reshape(-1)
    out = np.empty_like(flat)
    h = 1.0 / 256.0
    for i, xv in enumerate(flat):
        # stop where exp(-x cosh t) < 1e-300 relative to the peak
        tmax = np.arccosh(max(1.0, 700.0 / max(xv, 1e-300) + 1.0)) + 1.0
        t = np.arange(0.0, tmax + h, h)
        f = t * np.sinh(nu * t) * np.exp(-xv * (np.cosh(t) - 1.0))
        out[i] = np.exp(-xv) * h * (f.sum() - 0.5 * f[-1])  # f(0) = 0
    return out.reshape(xs.shape)


def matern_derivatives(x, y, theta):
    """dC/dsigma2, dC/dbeta, dC/dnu on all pairs (full matrices), as the reference's kernels:
    at distance 0 they are 1, 0, 0."""
    from scipy.special import kv, gamma, digamma
    sigma2, beta, nu = float(theta[0]), float(theta[1]), float(theta[2])
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    d = np.sqrt((x[None, :] - x[:, None]) ** 2 + (y[None, :] - y[:, None]) ** 2)
    e = d / beta
    zero = e == 0
    es = np.where(zero, 1.0, e)
    con = 1.0 / (2.0 ** (nu - 1.0) * gamma(nu))
    k0 = kv(nu, es)
    k1 = kv(nu + 1.0, es)
    dsig = np.where(zero, 1.0, con * es ** nu * k0)
    beta_expr = -nu / beta * es ** nu * k0 - es ** nu * (nu / es * k0 - k1) * es / beta
    dbeta = np.where(zero, 0.0, sigma2 * con * beta_expr)
    dk = dkv_dnu(nu, es)
    nu_expr = (-2.0 * np.log(2.0) * 2.0 ** (-nu) / gamma(nu) * es ** nu * k0
               + 2.0 ** (1.0 - nu) * (-digamma(nu) / gamma(nu) * es ** nu * k0
                                       + (es ** nu * np.log(es) * k0 + es ** nu * dk) / gamma(nu)))
    dnu = np.where(zero, 0.0, sigma2 * nu_expr)
    return dsig, dbeta, dnu


def fisher_inverse(x, y, theta) -> np.ndarray:
    """Inverse of the Fisher information A_jk = 1/2 tr(C^-1 C_j C^-1 C_k) (3 x 3, column-major list)."""
    c = covariance(x, y, theta)
    cf = scipy.linalg.cho_factor(c, lower=True, check_finite=False)
    ders = matern_derivatives(x, y, theta)
    sol = [scipy.linalg.cho_solve(cf, dj, check_finite=False) for dj in ders]
    a = np.empty((3, 3))
    for j in range(3):
        for k in range(3):
            a[j, k] = 0.5 * np.sum(sol[j] * sol[k].T)
    return np.linalg.inv(a)
