"""Batched evaluation of many independent problems (egs_batch_*) against the
single-problem path and the CPU oracle.

Tolerances:
  * same tile size as a single-problem call: relative error <= 1e-13 (the same
    kernels run on the same tiles; only launch grouping differs)
  * against the oracle: relative error <= 1e-10 (plain FP64 MLE contract)
"""
import numpy as np
import pytest

import exageostatcpp_b200 as egs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SAME_TS_RTOL = 1e-13
LOGLIK_RTOL = 1e-10


def make_problems(sizes, seed, theta=(1.0, 0.1, 0.5)):
    xs, ys, zs = [], [], []
    for i, n in enumerate(sizes):
        x, y, z = O.load_data(int(n), seed + i, theta)
        xs.append(x)
        ys.append(y)
        zs.append(z)
    return xs, ys, zs


def concat(*parts):
    return [np.concatenate(p) for p in parts]


def thetas_for(B, seed):
    rng = np.random.default_rng(seed)
    return np.column_stack([rng.uniform(0.5, 2.0, B), rng.uniform(0.03, 0.2, B), rng.uniform(0.3, 1.5, B)])


@pytest.mark.parametrize("sizes,dts", [
    ([700, 300, 64, 1, 129, 450], 128),
    ([1000, 1000, 1000], 192),
    ([90, 640, 2, 333], 64),
])
def test_batch_matches_single_problem_path(sizes, dts):
    xs, ys, zs = make_problems(sizes, 11)
    th = thetas_for(len(sizes), 5)
    b = egs.Batch(sizes, *concat(xs, ys, zs), dts=dts)
    ll, st = b.eval(th)
    assert np.all(st == 0)
    for i, n in enumerate(sizes):
        p = egs.Problem(n, dts)
        p.set_locations(xs[i], ys[i])
        p.set_observations(zs[i])
        ref = p.mle_eval(th[i])[0]
        p.close()
        assert abs(ll[i] - ref) <= SAME_TS_RTOL * abs(ref), (i, n, ll[i], ref)
    b.close()


def test_batch_matches_oracle():
    sizes = [400, 257, 31, 512]
    xs, ys, zs = make_problems(sizes, 21)
    th = thetas_for(len(sizes), 9)
    b = egs.Batch(sizes, *concat(xs, ys, zs), dts=128)
    ll, st = b.eval(th)
    assert np.all(st == 0)
    for i in range(len(sizes)):
        ref = O.mle_loglik(xs[i], ys[i], zs[i], th[i])
        assert abs(ll[i] - ref) <= LOGLIK_RTOL * abs(ref), (i, ll[i], ref)


def test_batch_graph_replay_repeats_and_follows_theta():
    sizes = [600, 200, 350]
    xs, ys, zs = make_problems(sizes, 31)
    b = egs.Batch(sizes, *concat(xs, ys, zs), dts=128)
    th1, th2 = thetas_for(3, 1), thetas_for(3, 2)
    a1, _ = b.eval(th1)   # direct launches
    a2, _ = b.eval(th2)   # captured graph
    a3, _ = b.eval(th1)   # replay
    a4, _ = b.eval(th2)
    assert np.array_equal(a1, a3)
    assert np.array_equal(a2, a4)
    assert b.info()["launches_per_eval"] > 0
    fresh = egs.Batch(sizes, *concat(xs, ys, zs), dts=128)
    f2, _ = fresh.eval(th2)
    assert np.array_equal(f2, a2)


def test_batch_failure_is_per_problem():
    """A problem whose covariance has a NaN pivot (a NaN location) reports it;
    the other problems' results are the same as when evaluated without it."""
    sizes = [300, 150, 200]
    xs, ys, zs = make_problems(sizes, 41)
    xs[1] = xs[1].copy()
    xs[1][77] = np.nan
    th = np.array([[1.0, 0.1, 0.5]] * 3)
    b = egs.Batch(sizes, *concat(xs, ys, zs), dts=128)
    ll, st = b.eval(th)
    assert st[0] == 0 and st[2] == 0
    assert st[1] > 0
    keep = [0, 2]
    b2 = egs.Batch([sizes[i] for i in keep], *concat([xs[i] for i in keep], [ys[i] for i in keep],
                                                     [zs[i] for i in keep]), dts=128)
    ll2, st2 = b2.eval(th[keep])
    assert np.all(st2 == 0)
    assert np.array_equal(ll[keep], ll2)


def test_batch_rejects_bad_input():
    x = np.zeros(10)
    with pytest.raises(egs.EgsError):
        egs.Batch([5, 0, 5], x, x, x, dts=64)
    with pytest.raises(ValueError):
        egs.Batch([5, 6], x, x, x, dts=64)
    xs, ys, zs = make_problems([50, 60], 3)
    b = egs.Batch([50, 60], *concat(xs, ys, zs), dts=64)
    with pytest.raises(egs.EgsError):
        b.eval([[1.0, 0.1, 0.5], [1.0, -0.1, 0.5]])


def test_batch_autotune_returns_a_candidate():
    sizes = [500, 300, 800]
    xs, ys, zs = make_problems(sizes, 51)
    ts, ms = egs.batch_autotune(sizes, *concat(xs, ys, zs), theta=[1.0, 0.1, 0.5], candidates=(64, 128, 192))
    assert ts in (64, 128, 192)
    assert ms > 0


def test_batch_of_64_uneven_problems_matches_the_single_problem_path():
    # The batched configuration's shape at test size: 64 problems, N log-uniform
    # in [256, 1024], theta drawn per problem as in that configuration (beta up to
    # 0.3, nu up to 2.5; a draw whose covariance is not numerically positive
    # definite must be reported the same way by both paths).
    rng = np.random.default_rng(7)
    B = 64
    sizes = np.rint(np.exp(rng.uniform(np.log(256), np.log(1024), B))).astype(int)
    th = np.column_stack([rng.uniform(0.5, 2.0, B), rng.uniform(0.02, 0.3, B), rng.uniform(0.3, 2.5, B)])
    xs, ys, zs = [], [], []
    for i, n in enumerate(sizes):
        x, y = egs.generate_locations(int(n), i)
        xs.append(x)
        ys.append(y)
        zs.append(egs.dlarnv_normal(i, int(n)))
    b = egs.Batch(sizes, *concat(xs, ys, zs), dts=192)
    ll, st = b.eval(th)
    ll2, st2 = b.eval(th)  # graph replay
    assert np.array_equal(ll, ll2) and np.array_equal(st, st2)
    b.close()
    compared = 0
    for i, n in enumerate(sizes):
        p = egs.Problem(int(n), 192)
        p.set_locations(xs[i], ys[i])
        p.set_observations(zs[i])
        try:
            ref = p.mle_eval(th[i])[0]
        except egs.NotPositiveDefinite:
            assert st[i] > 0, i
            continue
        finally:
            p.close()
        assert st[i] == 0, i
        assert abs(ll[i] - ref) <= SAME_TS_RTOL * abs(ref), (i, n, ll[i], ref)
        compared += 1
    assert compared >= B // 2


def test_size_classes_match_the_single_problem_path_and_autotune():
    # Two size classes with their own tiles, launched together: each problem's
    # result equals its single-problem evaluation at the class's tile size.
    rng = np.random.default_rng(3)
    B = 40
    sizes = np.rint(np.exp(rng.uniform(np.log(200), np.log(1500), B))).astype(int)
    th = np.column_stack([rng.uniform(0.5, 2.0, B), rng.uniform(0.02, 0.12, B), rng.uniform(0.3, 1.2, B)])
    xs, ys, zs = [], [], []
    for i, n in enumerate(sizes):
        x, y = egs.generate_locations(int(n), 100 + i)
        xs.append(x)
        ys.append(y)
        zs.append(egs.dlarnv_normal(100 + i, int(n)))
    upper = [600, int(sizes.max())]
    tiles = [128, 256]
    s = egs.BatchSet(sizes, *concat(xs, ys, zs), upper_n=upper, dts=tiles)
    info = s.info()
    assert info["classes"] == 2 and info["ts"] == tiles
    ll, st = s.eval(th)
    ll2, st2 = s.eval(th)  # captured graphs
    ll3, _ = s.eval(th)    # replays
    assert np.array_equal(ll, ll2) and np.array_equal(ll, ll3) and np.all(st == 0)
    s.close()
    for i, n in enumerate(sizes):
        ts = tiles[0] if n <= upper[0] else tiles[1]
        p = egs.Problem(int(n), ts)
        p.set_locations(xs[i], ys[i])
        p.set_observations(zs[i])
        ref = p.mle_eval(th[i])[0]
        p.close()
        assert abs(ll[i] - ref) <= SAME_TS_RTOL * abs(ref), (i, n, ll[i], ref)
    up, ts, ms = egs.batch_set_autotune(sizes, *concat(xs, ys, zs), theta=th, candidates=(128, 256), max_classes=2)
    assert 1 <= len(up) <= 2 and up[-1] == int(sizes.max()) and all(t in (128, 256) for t in ts) and ms > 0
