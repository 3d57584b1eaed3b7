"""The serving loop (egs_server_*) and the resident-problem kriging it uses.

Results of a request must be the same alone and in a mix of concurrent
requests: every kernel reduces in a fixed order and each request owns its
problem and stream, so the comparison is exact (tolerance 0) for the
log-likelihood, the fitted theta and the predictions.  Against the FP64
oracle the tolerances are those of the paths themselves: 1e-10 (FP64
log-likelihood), 1e-8 relative (FP64 kriging), 1e-6 (mixed precision).
"""
import numpy as np
import pytest

import exageostatcpp_b200 as egs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

D, M = egs.EGS_PRECISION_DOUBLE, egs.EGS_PRECISION_MIXED


def data(n, seed, theta=(1.0, 0.1, 0.5)):
    return O.load_data(n, seed, theta)


def targets(m, seed):
    rng = np.random.default_rng(seed)
    return rng.random(m), rng.random(m)


@pytest.mark.parametrize("precision,tol", [(D, 1e-8), (M, 1e-5)])
def test_problem_predict_matches_oracle(precision, tol):
    n, theta = 1800, (1.0, 0.08, 0.7)
    x, y, z = data(n, 21, theta)
    xm, ym = targets(60, 4)
    p = egs.Problem(n, 256, precision, 2 if precision == M else 0)
    p.set_locations(x, y)
    p.set_observations(z)
    got = p.predict(theta, xm, ym)
    ref, _ = O.predict(x, y, z, xm, ym, theta)
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    # the problem stays usable: an evaluation after the prediction is unchanged
    ll = p.mle_eval(theta)[0]
    rl = O.mle_loglik(x, y, z, theta)
    assert abs(ll - rl) <= (1e-10 if precision == D else 1e-6) * abs(rl)
    p.close()


def test_create_ex_mixed_equals_set_precision():
    n, theta = 1500, (1.0, 0.1, 0.5)
    x, y, z = data(n, 5, theta)
    a = egs.Problem(n, 256, M, 1)
    b = egs.Problem(n, 256)
    b.set_precision(M, 1)
    for p in (a, b):
        p.set_locations(x, y)
        p.set_observations(z)
    assert a.mle_eval(theta)[0] == b.mle_eval(theta)[0]


@pytest.mark.parametrize("precision,band", [(D, 0), (M, 2)])
def test_footprint_bounds_device_bytes(precision, band):
    for n, dts in [(700, 128), (3000, 256), (5000, 512)]:
        p = egs.Problem(n, dts, precision, band) if precision == M else egs.Problem(n, dts)
        assert p.device_bytes <= egs.footprint(n, dts, precision, band), (n, dts)
        p.close()


def request_mix():
    """Loglik, fit and predict requests of different N, plain and mixed."""
    reqs = []
    specs = [(egs.EGS_REQ_LOGLIK, 2600, D), (egs.EGS_REQ_FIT, 900, D), (egs.EGS_REQ_PREDICT, 2000, D),
             (egs.EGS_REQ_LOGLIK, 3000, M), (egs.EGS_REQ_FIT, 1200, M), (egs.EGS_REQ_PREDICT, 2300, M),
             (egs.EGS_REQ_LOGLIK, 700, D), (egs.EGS_REQ_FIT, 1600, D)]
    for i, (kind, n, prec) in enumerate(specs):
        theta = (1.0 + 0.1 * i, 0.05 + 0.01 * i, 0.5 + 0.1 * i)
        x, y, z = data(n, 30 + i, theta)
        r = dict(kind=kind, x=x, y=y, z=z, dts=256, theta=theta, precision=prec, band_tiles=2 if prec == M else 0,
                 max_evals=15, ftol_abs=1e-9)
        if kind == egs.EGS_REQ_PREDICT:
            r["x_miss"], r["y_miss"] = targets(50, i)
        reqs.append(r)
    return reqs


def run_all(server, reqs, together):
    out = []
    if together:
        tickets = [server.submit(**r) for r in reqs]
        out = [server.wait(t) for t in tickets]
    else:
        for r in reqs:
            out.append(server.wait(server.submit(**r)))
    return out


def test_results_same_alone_and_in_the_mix():
    reqs = request_mix()
    with egs.Server(hbm_budget=64 << 30, max_active=1) as s:
        alone = run_all(s, reqs, together=False)
    with egs.Server(hbm_budget=64 << 30, max_active=4) as s:
        mixed = run_all(s, reqs, together=True)
        st = s.stats()
    assert st["completed"] == len(reqs) and st["peak_active"] > 1
    for (ra, pa), (rm, pm), r in zip(alone, mixed, reqs):
        assert ra.status == 0 and rm.status == 0, (ra.status, rm.status)
        assert ra.loglik == rm.loglik
        assert list(ra.theta) == list(rm.theta)
        assert ra.evals == rm.evals
        if r["kind"] == egs.EGS_REQ_PREDICT:
            assert np.array_equal(pa, pm)


def test_request_results_match_the_direct_calls():
    reqs = request_mix()
    with egs.Server(hbm_budget=64 << 30, max_active=3) as s:
        res = run_all(s, reqs, together=True)
    for (r, pred), q in zip(res, reqs):
        if q["kind"] == egs.EGS_REQ_LOGLIK:
            ref = O.mle_loglik(q["x"], q["y"], q["z"], q["theta"])
            assert abs(r.loglik - ref) <= (1e-10 if q["precision"] == D else 1e-6) * abs(ref)
        elif q["kind"] == egs.EGS_REQ_PREDICT:
            ref, _ = O.predict(q["x"], q["y"], q["z"], q["x_miss"], q["y_miss"], q["theta"])
            tol = 1e-8 if q["precision"] == D else 1e-5
            assert np.max(np.abs(pred - ref)) <= tol * np.max(np.abs(ref))
        else:
            # the same BOBYQA run driven directly on a resident problem
            p = egs.Problem(len(q["z"]), q["dts"], q["precision"], q["band_tiles"]) if q["precision"] == M \
                else egs.Problem(len(q["z"]), q["dts"])
            p.set_locations(q["x"], q["y"])
            p.set_observations(q["z"])
            def objective(t):
                # the server rejects a non-positive-definite point with -1e300 and goes on
                try:
                    return p.mle_eval(t)[0]
                except egs.NotPositiveDefinite:
                    return -1e300

            th, best, nev = egs.bobyqa_maximize(objective, [0.01] * 3, [0.01] * 3, [5.0] * 3, q["ftol_abs"],
                                                q["max_evals"])
            p.close()
            assert r.evals == nev and r.loglik == best
            assert np.allclose(list(r.theta), th, rtol=0, atol=0)


def test_admission_keeps_reserved_bytes_within_the_budget():
    reqs = [r for r in request_mix() if r["kind"] != egs.EGS_REQ_FIT]
    biggest = max(egs.footprint(len(r["z"]), r["dts"], r["precision"], r["band_tiles"]) +
                  (len(r["z"]) * 50 + 200) * 8 for r in reqs)
    budget = int(1.2 * biggest)
    with egs.Server(hbm_budget=budget, max_active=4) as s:
        res = run_all(s, reqs, together=True)
        st = s.stats()
    assert all(r.status == 0 for r, _ in res)
    assert st["peak_reserved"] <= budget
    assert st["reserved"] == 0 and st["active"] == 0 and st["queued"] == 0


def test_oversized_request_is_refused():
    x, y, z = data(2000, 3)
    with egs.Server(hbm_budget=1 << 20, max_active=2) as s:
        with pytest.raises(egs.EgsError) as ei:
            s.submit(egs.EGS_REQ_LOGLIK, x, y, z, 256)
        assert ei.value.status == egs.EGS_ERR_OOM


def test_mixed_request_that_loses_definiteness_is_answered_in_fp64():
    # Very smooth, long-range kernels on a dense grid: kappa(Sigma) ~ 1e10 and more,
    # beyond FP32 off-band storage; the server answers such mixed requests with the
    # FP64 path (precision_used) instead of failing them.
    x, y = egs.generate_locations(1600, 0)
    z = egs.dlarnv_normal(0, 1600)
    fell_back = 0
    with egs.Server(hbm_budget=16 << 30, max_active=2) as s:
        for theta in [(1.2, 0.2, 2.5), (1.0, 0.3, 2.5), (1.0, 0.5, 2.0)]:
            tp = s.submit(egs.EGS_REQ_LOGLIK, x, y, z, 256, theta=theta)
            tm = s.submit(egs.EGS_REQ_LOGLIK, x, y, z, 256, theta=theta, precision=M, band_tiles=1)
            (rp, _), (rm, _) = s.wait(tp), s.wait(tm)
            if rp.status != 0:
                continue
            assert rm.status == 0
            if rm.precision_used == D:
                fell_back += 1
                assert rm.loglik == rp.loglik
                assert rm.fp64_reason in (egs.EGS_FP64_REASON_PREDICTED, egs.EGS_FP64_REASON_AFTER_FAILURE)
            else:
                assert rm.fp64_reason == egs.EGS_FP64_REASON_NONE
                assert abs(rm.loglik - rp.loglik) <= 1e-4 * abs(rp.loglik)
    assert fell_back >= 1


def test_ill_conditioned_mixed_request_goes_to_fp64_up_front():
    # theta = (1, 0.3, 2.5) on 24,000 points: estimated kappa ~ 1e15, far above the
    # FP32 off-band storage's reach (it fails there on a B200); the request is
    # answered by the FP64 path without a mixed attempt, with the plain result.
    # theta = (1, 0.05, 0.5) on the same points stays in mixed precision.
    x, y = egs.generate_locations(24000, 2)
    z = egs.dlarnv_normal(2, 24000)
    with egs.Server(hbm_budget=60 << 30, max_active=2) as s:
        tm = s.submit(egs.EGS_REQ_LOGLIK, x, y, z, 1024, theta=(1.0, 0.3, 2.5), precision=M, band_tiles=2)
        tp = s.submit(egs.EGS_REQ_LOGLIK, x, y, z, 1024, theta=(1.0, 0.3, 2.5))
        (rm, _), (rp, _) = s.wait(tm), s.wait(tp)
        tk = s.submit(egs.EGS_REQ_LOGLIK, x, y, z, 1024, theta=(1.0, 0.05, 0.5), precision=M, band_tiles=2)
        rk, _ = s.wait(tk)
    assert rp.status == 0 and rm.status == 0
    assert rm.precision_used == D and rm.fp64_reason == egs.EGS_FP64_REASON_PREDICTED
    assert rm.loglik == rp.loglik and rm.evals == 1
    assert rk.status == 0 and rk.precision_used == M and rk.fp64_reason == egs.EGS_FP64_REASON_NONE
