"""The random hold-out split of the prediction module (egs_shuffle_split), on the CPU.

PredictionHelpers<T>::Shuffle (src/prediction/PredictionHelpers.cpp:140-168)
draws from the C library's rand() without reseeding, so in the reference's
generate -> predict flow the split continues the rand() stream that
LocationGenerator consumed.  The library call must take exactly those draws:
it is checked bit for bit against the oracle's restatement of glibc rand()."""
import ctypes

import numpy as np
import pytest

import exageostatcpp_b200 as egs
from oracle import oracle as O


def test_split_continues_the_location_generators_rand_stream():
    n, n_miss, seed = 2117, 100, 5
    x, y = egs.generate_locations(n, seed)          # srand(seed), 2 n draws
    z = np.arange(n, dtype=np.float64) * 0.5 - 3.0
    got = egs.shuffle_split(z, x, y, n_miss)
    rng = O.GlibcRand(seed)
    xr, yr = O.generate_locations(n, rng)
    assert np.array_equal(x, xr) and np.array_equal(y, yr)
    ref = O.shuffle_split(z, xr, yr, n_miss, rng)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    # every value appears once: the first n_miss held out, the rest observed
    assert np.array_equal(np.sort(np.concatenate([got[0], got[3]])), np.sort(z))


def test_split_from_a_fresh_rand_state_matches_the_oracle():
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(ctypes.c_uint(7))
    x, y = O.generate_locations(40, O.GlibcRand(1))
    z = np.linspace(-1.0, 1.0, 40)
    got = egs.shuffle_split(z, x, y, 4)
    ref = O.shuffle_split(z, x, y, 4, O.GlibcRand(7))
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_split_rejects_bad_sizes():
    with pytest.raises(egs.EgsError):
        egs.shuffle_split([1.0, 2.0], [0.1, 0.2], [0.3, 0.4], 3)
    zo, xo, yo, zm, xm, ym = egs.shuffle_split([1.0, 2.0], [0.1, 0.2], [0.3, 0.4], 0)
    assert len(zm) == 0 and sorted(zo) == [1.0, 2.0]
