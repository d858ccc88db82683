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


def degenerate_clouds(d, seed):
    """`{ name: (positions, groups) }`: a uniform cloud in [0.05, 0.95]^d (400 seeds in 2D, 600 in 3D) with some seeds moved
    onto others (tests/test_SdotPlanNd.py:1377-1404); `groups` lists `(members, exact)`, `exact` when the members share
    one position"""
    rng = np.random.default_rng(seed)
    n = 400 if d == 2 else 600
    base = rng.uniform(0.05, 0.95, size=(n, d))
    diag = np.ones(d) / np.sqrt(d)
    axis = np.eye(d)[0]

    def cloud(*moves):
        pos, groups = base.copy(), []
        for members, shifts in moves:
            for m, sh in zip(members[1:], shifts):
                pos[m] = pos[members[0]] + sh
            groups.append((list(members), all(not np.any(sh) for sh in shifts)))
        return pos, groups

    return {
        "exact pair": cloud(([5, 7], [0 * diag])),
        "exact triple": cloud(([3, 11, 29], [0 * diag, 0 * diag])),
        "pair at 1e-9": cloud(([5, 7], [1e-9 * diag])),
        "pair at 1e-12": cloud(([8, 2], [1e-12 * diag])),
        "triple at 1e-10": cloud(([4, 9, 13], [1e-10 * diag, 2e-10 * axis])),
        "pair and duplicate": cloud(([1, 6], [3e-10 * diag]), ([12, 15, 30], [0 * diag, 2e-10 * axis])),
    }
