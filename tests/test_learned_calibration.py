"""The learned scorer's shrink factor: the least-absolute-error scale of the
predicted correction on a validation split, clipped to [0, 1]."""
import numpy as np

from remobench_b200.learned import mae_shrink


def test_mae_shrink_is_the_least_absolute_error_factor():
    rng = np.random.default_rng(3)
    y = rng.normal(size=20000)
    t = 0.37 * y + rng.laplace(scale=0.05, size=20000)
    a = mae_shrink(y, t)
    grid = np.linspace(0.0, 1.0, 2001)
    best = grid[np.argmin([np.abs(t - g * y).sum() for g in grid])]
    assert abs(a - best) <= 1e-3
    assert np.abs(t - a * y).sum() <= np.abs(t).sum()  # never worse than no correction


def test_mae_shrink_edges():
    assert mae_shrink(np.zeros(5), np.ones(5)) == 0.0
    y = np.linspace(-1, 1, 101)
    assert mae_shrink(y, -y) == 0.0          # anti-correlated: trust none of it
    assert mae_shrink(y, 3.0 * y) == 1.0     # never more than the network says
