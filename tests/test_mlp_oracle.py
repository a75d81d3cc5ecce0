"""The learned-source MLP's CPU oracle, pinned by finite differences of its exact-arithmetic form."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as mo  # noqa: E402


def small_problem(seed=3, nbins=8, hidden=6, rows=5):
    rng = np.random.default_rng(seed)
    n = hidden * nbins + hidden * 4 + hidden + 2 * (hidden * hidden + hidden) + nbins * hidden + nbins
    p = rng.normal(0.0, 0.4, n)
    X = rng.normal(0.0, 1.0, (rows, nbins))
    E = rng.normal(0.0, 1.0, (rows, 4))
    T = rng.normal(0.0, 1.0, (rows, nbins))
    return p, X, E, T


def test_oracle_gradient_matches_finite_differences():
    nb, hd = 8, 6
    p, X, E, T = small_problem(nbins=nb, hidden=hd)
    loss, g, _ = mo.forward_backward(p, X, E, T, nb, hd, rounding=False)
    rng = np.random.default_rng(7)
    for i in rng.choice(p.size, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.forward_backward(pp, X, E, T, nb, hd, rounding=False)[0]
              - mo.forward_backward(pm, X, E, T, nb, hd, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5, 3.0e38], dtype=np.float32)
    got = mo.bf16(x)
    want = np.array([1.0, 1.0, 1.0 + 2 ** -7, 1.0, -2.5], dtype=np.float32)
    assert np.array_equal(got[:5], want)
    assert abs(float(got[5]) - 3.0e38) / 3.0e38 <= 2.0 ** -8             # within half a BF16 ulp
