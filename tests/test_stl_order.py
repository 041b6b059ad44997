"""The device restatement of libstdc++'s std::sort and std::minmax_element orders (used for score
lists holding NaN) against libstdc++ itself (called by the oracle)."""

import numpy as np

from cusingler_b200 import abi
from oracle import oracle as O


def test_sort_and_minmax_match_libstdcxx():
    rng = np.random.default_rng(0)
    for trial in range(4000):
        n = int(rng.integers(1, 400))
        v = rng.standard_normal(n).astype(np.float32)
        if rng.random() < 0.5:
            v = np.round(v * 2) / 2
        v[rng.random(n) < rng.choice([0.0, 0.01, 0.1, 0.5, 1.0])] = np.nan
        a = abi.stl_sort(v)
        b = O.std_sort(v)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), trial
        assert abi.stl_minmax(v) == O.minmax(v), trial


def test_minmax_last_max_first_min():
    assert abi.stl_minmax([0.5, 0.9, 0.2, 0.9]) == (2, 3)
    assert abi.stl_minmax([0.2, 0.2, 0.2]) == (0, 2)
    nan = float("nan")
    assert abi.stl_minmax([nan] * 5) == O.minmax([nan] * 5)
