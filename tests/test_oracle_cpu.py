"""The C restatement of the Matern generator that serves as the large-N oracle and
the timed CPU baseline (oracle/matern_cpu.c), against the numpy/scipy oracle.

At N = 40,000 and above the scipy oracle cannot hold its full-matrix
temporaries, so the large parity cases use oracle/cpu_baseline.py; this pins
that path to oracle/oracle.py (itself pinned to the reference's goldens)."""
import numpy as np
import pytest

from oracle import cpu_baseline as C
from oracle import oracle as O


@pytest.mark.parametrize("nu", [0.5, 0.8, 1.5, 0.3, 2.2, 3.7])
def test_c_generator_matches_scipy_oracle(nu):
    x, y = O.generate_locations(500, O.GlibcRand(2))
    theta = [1.3, 0.07, nu]
    ref = O.covariance(x, y, theta)
    low = C.matern_lower(x, y, theta)
    li = np.tril_indices(500)
    err = np.abs(low[li] - ref[li])
    assert np.all(err <= 1e-13 * np.abs(ref[li]) + 1e-16 * theta[0]), err.max()
    xm, ym = O.generate_locations(37, O.GlibcRand(9))
    blk = C.matern_block(xm, ym, x, y, theta)
    rb = O.matern_block(xm, ym, x, y, theta)
    assert np.all(np.abs(blk - rb) <= 1e-13 * np.abs(rb) + 1e-16 * theta[0])


def test_eval_and_predict_matches_the_scipy_oracle():
    theta = [1.0, 0.05, 0.8]
    x, y, z = O.load_data(1200, 3, theta)
    zo, xo, yo, za, xm, ym = O.shuffle_split(z, x, y, 50, O.GlibcRand(4))
    ll, logdet, dot, zm, mspe, _ = C.eval_and_predict(xo, yo, zo, xm, ym, theta, za)
    rll, rlogdet, rdot = O.mle_loglik(xo, yo, zo, theta, return_parts=True)
    assert ll == pytest.approx(rll, rel=1e-12)
    assert dot == pytest.approx(rdot, rel=1e-11)
    rzm, rmspe = O.predict(xo, yo, zo, xm, ym, theta, za)
    assert np.abs(zm - rzm).max() <= 1e-11 * np.abs(rzm).max()
    assert mspe == pytest.approx(rmspe, rel=1e-10)
