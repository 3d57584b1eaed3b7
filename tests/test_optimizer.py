"""The BOBYQA maximiser of the MLE driver (egs_bobyqa_maximize), on the CPU."""
import numpy as np
import pytest

import exageostatcpp_b200 as egs
from oracle import oracle as O


def test_first_evaluations_reproduce_the_reference_golden(goldens):
    # NLopt LN_BOBYQA from x0 = lb with 3 evaluations: x0, x0 + rho e1, x0 + rho e2,
    # rho = 0.25 (ub - lb); the best is the reference's -24.026000 (TestExaGeoStatApi.cpp:93).
    f = goldens["fixture_n16"]
    g = goldens["modeling_loglik_n16"]
    seen = []

    def obj(th):
        seen.append(th.copy())
        return O.mle_loglik(f["x"], f["y"], f["z"], th)

    th, fb, ne = egs.bobyqa_maximize(obj, g["lb"], g["lb"], g["ub"], 10.0 ** -g["tolerance_exponent"],
                                     g["max_mle_iterations"])
    assert ne == 3
    assert np.allclose(seen, [[0.1, 0.1, 0.1], [1.325, 0.1, 0.1], [0.1, 1.325, 0.1]], atol=1e-15)
    assert abs(fb - g["exact_dense"]) < g["margin"]
    assert th == pytest.approx([1.325, 0.1, 0.1])


def test_bounded_quadratic_is_solved_exactly():
    def quad(x):
        return -((x[0] - 0.3) ** 2 + 2 * (x[1] + 0.7) ** 2 + 3 * (x[2] - 1.9) ** 2 + 0.5 * x[0] * x[1])

    th, fb, ne = egs.bobyqa_maximize(quad, [0, 0, 0], [-1, -1, -1], [1, 1, 1], 1e-14, 500)
    x1 = -2.95 / 3.875
    assert th == pytest.approx([0.3 - 0.25 * x1, x1, 1.0], abs=1e-7)
    assert ne < 500


def test_rosenbrock_converges():
    def rb(x):
        return -((1 - x[0]) ** 2 + 100 * (x[1] - x[0] ** 2) ** 2 + (x[2] - 0.5) ** 2)

    th, fb, ne = egs.bobyqa_maximize(rb, [-1, 2, 0], [-2, -2, -2], [2, 2, 2], 1e-14, 3000)
    assert th == pytest.approx([1.0, 1.0, 0.5], abs=1e-4)


def test_bounds_and_maxeval_are_respected():
    pts = []

    def f(x):
        pts.append(x.copy())
        return float(np.sum(x))  # increasing: the optimum is the upper corner

    lb, ub = np.array([0.01, 0.02, 0.03]), np.array([5.0, 4.0, 3.0])
    th, fb, ne = egs.bobyqa_maximize(f, lb, lb, ub, 1e-12, 60)
    pts = np.array(pts)
    assert ne <= 60 and len(pts) == ne
    assert np.all(pts >= lb - 1e-15) and np.all(pts <= ub + 1e-15)
    assert th == pytest.approx(ub, abs=1e-9)


def test_objective_exception_propagates():
    def bad(x):
        raise RuntimeError("boom")

    with pytest.raises(RuntimeError, match="boom"):
        egs.bobyqa_maximize(bad, [1, 1, 1], [0, 0, 0], [2, 2, 2], 1e-9, 10)
