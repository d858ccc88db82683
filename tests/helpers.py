"""Comparison helpers shared by the parity tests."""
import numpy as np


def neighbour_sets(nb, nid, meas, rel_floor=1e-9, scale=None):
    """per cell, the set of neighbours whose facet measure is above `rel_floor` of the cell's largest facet
    (facets below are degenerate: their presence depends on rounding, not on the diagram)"""
    out = []
    for i in range(len(nb)):
        k = int(nb[i])
        ids, m = nid[i, :k], meas[i, :k]
        top = m.max() if k else 0.0
        out.append(frozenset(int(j) for j, v in zip(ids, m) if v > rel_floor * top))
    return out


def degenerate_pairs(nb, nid, meas, lo=1e-9, hi=1e-6):
    """pairs (i, j) whose facet sits in the ambiguous band [lo, hi] relative to the cell's largest facet"""
    res = set()
    for i in range(len(nb)):
        k = int(nb[i])
        if not k:
            continue
        top = meas[i, :k].max()
        for j, v in zip(nid[i, :k], meas[i, :k]):
            if lo * top <= v <= hi * top:
                res.add((min(i, int(j)), max(i, int(j))))
    return res


def compare_neighbours(a, b, skip_pairs=()):
    """number of cells whose non-degenerate neighbour sets differ, ignoring pairs in `skip_pairs`"""
    bad = 0
    for i, (sa, sb) in enumerate(zip(a, b)):
        d = {j for j in sa ^ sb if (min(i, j), max(i, j)) not in skip_pairs}
        bad += bool(d)
    return bad


def monte_carlo_masses(pos, lo, hi, weights=None, nb_samples=200000, seed=0):
    """measures by sampling the definition `argmin |x - p|^2 - w` (the reference's independent check,
    tests/test_PowerDiagram.py:15-32)"""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    res = np.zeros(len(pos))
    done = 0
    while done < nb_samples:
        m = min(20000, nb_samples - done)
        pts = rng.uniform(lo, hi, size=(m, lo.size))
        d2 = ((pts[:, None, :] - pos[None, :, :]) ** 2).sum(axis=2)
        if weights is not None:
            d2 = d2 - np.asarray(weights, float)[None, :]
        res += np.bincount(d2.argmin(axis=1), minlength=len(pos))
        done += m
    return res / nb_samples * float(np.prod(hi - lo))
