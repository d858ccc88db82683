"""The memory model of a solve (sdot_solve_bytes, which restates the reference's CardMemory.card_solve_bytes,
src/sdot/CardMemory.py:1-150) against the device pool's real peak, and the refusal of a solve that does not fit
(CardMemory.check_card_memory, src/sdot/CardMemory.py:158-190): a MemoryError that says what the solve needs, raised
before anything is built."""
import numpy as np
import pytest

import sdot
from sdot import Iterative, Tuning, _lib
from sdot.PowerDiagram import _domain_box
from sdot.SdotPlanNd import solver_options

pytestmark = pytest.mark.gpu


def _problem(d, n, gauss, seed=0):
    rng = np.random.default_rng([seed, d, n])
    pos = rng.uniform(size=(n, d))
    if gauss:
        t = sdot.SumOfGaussians(rng.uniform(0.3, 0.7, size=(2, d)), np.array([0.1, 0.15]), np.array([0.5, 0.5]),
                                support_box=(np.zeros(d), np.ones(d)))
    else:
        t = sdot.Box(nb_dims=d)
    t = t.normalized_version(nb_dims=d)
    lo, hi = _domain_box(t.bounding_half_spaces(), d)
    return (pos, None, None, lo, hi, t._sdot_density())


def _options():
    return solver_options(Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-8)), 0)


@pytest.mark.parametrize("d,n,gauss", [(2, 20000, False), (2, 200000, False), (3, 20000, False), (2, 20000, True)])
def test_the_memory_model_bounds_the_pool_peak(d, n, gauss):
    """a solve alone in a fresh context takes at most what the model says, and not less than a third of it"""
    ctx = _lib.new_context()
    try:
        _lib.solve_batch([_problem(d, 500, gauss, 1)], [_options()], ctx=ctx)      # the context's own buffers, once
        base = _lib.context_memory(ctx, reset_peak=True)
        pb = _problem(d, n, gauss)
        r = _lib.solve_batch([pb], [_options()], ctx=ctx)[0]
        assert not isinstance(r, Exception), r
        assert r["stats"][0] == 1, r["stats"][0]
        peak = _lib.context_memory(ctx)["peak"] - base["in_use"]
        model = _lib.solve_bytes(d, n, pb[5])
        print(f"\n{d}D n={n} {'gaussians' if gauss else 'uniform'}: pool peak {peak / n:.0f} B per seed, model {model / n:.0f}")
        assert peak <= model, (peak, model)
        assert model <= 3 * peak, (peak, model)
    finally:
        _lib.destroy_context(ctx)


def test_a_solve_past_the_pool_limit_is_a_memory_error():
    """a context whose pool may hand out half of what a solve of 1e5 seeds needs refuses that solve with a MemoryError
    naming its need, then solves a small problem as usual"""
    d, n = 2, 100_000
    pb = _problem(d, n, False)
    model = _lib.solve_bytes(d, n, pb[5])
    probe = _lib.new_context()
    fixed = _lib.context_memory(probe)["in_use"]
    _lib.destroy_context(probe)
    ctx = _lib.new_context(pool_limit=fixed + model // 2)
    try:
        r = _lib.solve_batch([pb], [_options()], ctx=ctx)[0]
        assert isinstance(r, MemoryError), r
        assert "needs about" in str(r), str(r)
        assert _lib.context_memory(ctx)["in_use"] <= fixed + model // 2
        r = _lib.solve_batch([_problem(d, 2000, False)], [_options()], ctx=ctx)[0]
        assert not isinstance(r, Exception), r
        assert r["stats"][0] == 1
    finally:
        _lib.destroy_context(ctx)
