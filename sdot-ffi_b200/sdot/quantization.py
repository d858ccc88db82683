"""`quantization`: optimal quantization of a density by Lloyd's algorithm in its transport form (quantization.py:1-30).

    pos = sdot.quantization(target, pos0)
    pos = sdot.quantization(target, 1000)          # 1000 diracs drawn uniformly in the support of `target`

The diracs keep their masses and move: each iteration solves the transport from the diracs to `target` and sends each
dirac to the barycentre of its cell. `x <- b(x)` is a gradient step of size 1 / (2 m_i) on W2^2, which therefore decreases.

Stopping: `rms_i |b_i - x_i| <= tol * sqrt(W2^2)` (scale free: sqrt(W2^2) is the typical distance from a point of the
target to its dirac). The problem is kept from one iteration to the next, so each solve starts from the previous weights
and takes a few Newton steps. The transports need not be precise: their tolerance is `1e-4 / n` unless `ot_tol` says
otherwise, and a solve that stagnates above it is used all the same, with a warning.
"""
import numbers
import warnings

import numpy as np

from .OtProblem import Iterative, OtNotConverged, OtProblem
from .distributions import SumOfDiracs


def quantization(target, positions, masses=None, *, tol=2e-2, max_iter=200, callback=None, verbose=False, ot_tol=None,
                 seed=None, **settings):
    """the positions of diracs that quantize `target`, by Lloyd iterations from `positions` ([n, d], or a number of diracs
    drawn uniformly in the support of `target` with `numpy.random.default_rng(seed)`), as an [n, d] array
    (quantization.py:41-110). `masses`: [n], kept (equal by default). `callback(iteration, positions, plan)` is called after
    each solve with the positions that plan was solved for (iteration 0: the start). `settings` are `Iterative`'s, but
    its `tol` is named `ot_tol` here."""
    if isinstance(positions, numbers.Integral):
        positions = uniform_in_support(target, int(positions), seed)
    x = np.array(positions, dtype=np.float64)
    pb = OtProblem(SumOfDiracs(x, masses), target)
    n = pb.nb_diracs
    it_settings = Iterative(tol=1e-4 / n if ot_tol is None else ot_tol, **settings)
    stagnations = []
    ratio = np.inf
    for iteration in range(max_iter + 1):
        try:
            plan = pb.solve(it_settings, verbose)
        except OtNotConverged as e:
            if e.solution.stats["status"] != "stagnation":
                raise
            plan = e.solution
            stagnations.append(plan.stats["residual"])
        if callback is not None:
            callback(iteration, x.copy(), plan)
        b = np.asarray(plan.barycenters, dtype=np.float64)
        ratio = (float(((b - x) ** 2).sum()) / n / float(plan.cost)) ** 0.5
        if ratio <= tol or iteration == max_iter:
            break
        x = b.copy()
        pb.source = SumOfDiracs(x, masses)
    if stagnations:
        warnings.warn(f"sdot.quantization: {len(stagnations)} of {iteration + 1} transports stagnated above their tolerance "
                      f"(worst residual {max(stagnations):.3g}, for a dirac mass of {1 / n:.3g}) -- their solutions were used "
                      "all the same", stacklevel=2)
    if ratio > tol:
        warnings.warn(f"sdot.quantization: {max_iter} iterations without reaching tol = {tol} (the last move is {ratio:.3g} "
                      "times the cell size)", stacklevel=2)
    return np.asarray(plan.barycenters, dtype=np.float64)


def uniform_in_support(target, n, seed=None):
    """`n` points drawn uniformly in the support of `target` (its `bounding_half_spaces`), by rejection in the bounding box
    of that polytope (quantization.py:113-130)"""
    support = target.bounding_half_spaces()
    if support is None:
        raise ValueError("sdot.quantization: the target declares no support (`bounding_half_spaces` is None), the starting "
                         "positions have to be given")
    dirs, offs = (np.asarray(a, dtype=np.float64) for a in support)
    offs = offs.reshape(-1)
    lo, hi = _bounding_box(dirs, offs)
    rng = np.random.default_rng(seed)
    res = np.zeros((0, len(lo)))
    while len(res) < n:
        x = rng.uniform(lo, hi, (2 * (n - len(res)) + 16, len(lo)))
        res = np.concatenate([res, x[np.all(x @ dirs.T <= offs, axis=1)]])
    return res[:n]


def _bounding_box(dirs, offs):
    """the extent of `{x : dirs x <= offs}` along each axis (one small LP per side)"""
    from scipy.optimize import linprog
    d = dirs.shape[1]
    lo, hi = np.zeros(d), np.zeros(d)
    for a in range(d):
        c = np.zeros(d)
        c[a] = 1.0
        for sign, out in ((1.0, lo), (-1.0, hi)):
            r = linprog(sign * c, A_ub=dirs, b_ub=offs, bounds=[(None, None)] * d, method="highs")
            if not r.success:
                raise ValueError("sdot.quantization: the support of the target is empty or unbounded")
            out[a] = r.x[a]
    return lo, hi
