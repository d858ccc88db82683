"""Lloyd's quantization on top of the GPU solve (tests/test_quantization.py of the reference; its `Polygon` square is
the unit `Box` here)."""
import numpy as np
import pytest

import sdot
from sdot import quantization

pytestmark = pytest.mark.gpu


def test_lloyd_on_a_square_reaches_the_regular_grid():
    """tests/test_quantization.py:3-15: 4 diracs of equal mass go to the centres of the quadrants; W2^2 decreases"""
    grid = np.array([[0.25, 0.25], [0.75, 0.25], [0.25, 0.75], [0.75, 0.75]])
    x0 = grid + np.random.default_rng(0).uniform(-0.1, 0.1, grid.shape)
    costs = []
    x = quantization(sdot.Box(nb_dims=2), x0, tol=1e-6, callback=lambda it, pos, plan: costs.append(float(plan.cost)))
    assert isinstance(x, np.ndarray) and x.shape == (4, 2)
    assert np.abs(x - grid).max() < 1e-4
    assert all(b <= a + 1e-12 for a, b in zip(costs, costs[1:]))


def test_the_callback_receives_the_positions_of_each_solve():
    """tests/test_quantization.py:18-27"""
    x0 = np.random.default_rng(1).uniform(0, 1, (50, 2))
    seen = []
    quantization(sdot.Box(nb_dims=2), x0, callback=lambda it, pos, plan: seen.append((it, np.asarray(pos))))
    assert [it for it, _ in seen] == list(range(len(seen)))
    assert np.array_equal(seen[0][1], x0)
    assert len(seen) > 1 and not np.allclose(seen[-1][1], x0)


def test_max_iter_reached_warns():
    """tests/test_quantization.py:30-37"""
    x0 = np.random.default_rng(2).uniform(0, 1, (50, 2))
    with pytest.warns(UserWarning, match="iterations without reaching"):
        quantization(sdot.Box(nb_dims=2), x0, max_iter=2)


def test_a_number_of_diracs_starts_them_in_the_support():
    """tests/test_quantization.py:40-49 (on an image target: the support is its frame)"""
    from sdot.quantization import uniform_in_support
    img = sdot.Image(1 + np.arange(12.0).reshape(4, 3), frame=[0.5, 0.25])
    x0 = uniform_in_support(img, 500, seed=3)
    assert x0.shape == (500, 2) and (x0 >= 0).all() and (x0[:, 0] <= 2).all() and (x0[:, 1] <= 0.75).all()
    seen = []
    x = quantization(img, 500, seed=3, callback=lambda it, pos, plan: seen.append(np.asarray(pos)))
    assert np.array_equal(seen[0], x0) and x.shape == (500, 2)


def test_lloyd_on_a_density_spreads_blue_noise():
    """a 3D gaussian bump: every Lloyd step lowers W2^2 (x <- b(x) is a gradient step on it) and the points stay in the box"""
    g = sdot.SumOfGaussians(np.array([[0.5, 0.5, 0.5]]), np.array([0.2]), support_box=(np.zeros(3), np.ones(3)))
    costs = []
    x = quantization(g, 2000, seed=5, tol=5e-2, callback=lambda it, pos, plan: costs.append(float(plan.cost)))
    assert x.shape == (2000, 3) and (x >= 0).all() and (x <= 1).all()
    assert all(b <= a * (1 + 1e-9) for a, b in zip(costs, costs[1:])) and len(costs) > 2
