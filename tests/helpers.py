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


def gaussian_facet_case(d, perm=None, flip=None):
    """the reference's closed-form facet of a sum of gaussians (tests/test_SumOfGaussians.py:20-43): two seeds at
    x = 1/4 and 3/4 of the unit cube share the facet x = 1/2, on which each gaussian is a product of erf factors.
    `d` 2 drops the last axis. `perm` / `flip` map the configuration by a symmetry of the cube (the facet then lies
    across another axis, the seeds and centres move with it), so the same answer checks the frame of the face
    integral. Returns `(positions, centres, sigmas, masses, c_01)`, the masses normalised to 1 and
    `c_01 = int_facet rho / (2 |p_1 - p_0|)`."""
    from math import erf, exp, pi, sqrt
    c = np.array([[0.43, 0.58, 0.47], [0.52, 0.31, 0.66], [0.2, 0.7, 0.5]])[:, :d]
    s = np.array([0.17, 0.05, 0.3])
    m = np.array([0.5, 1.0, 0.7])
    m = m / m.sum()
    pos = np.array([[0.25, 0.5, 0.5], [0.75, 0.5, 0.5]])[:, :d]
    seg = lambda a, sg: 0.5 * (erf((1 - a) / (sg * sqrt(2))) - erf(-a / (sg * sqrt(2))))
    facet = sum(m[k] * exp(-(0.5 - c[k, 0]) ** 2 / (2 * s[k] ** 2)) / (s[k] * sqrt(2 * pi)) * np.prod([seg(c[k, a], s[k]) for a in range(1, d)])
                for k in range(3))
    perm = list(range(d)) if perm is None else list(perm)
    pos, c = pos[:, perm].copy(), c[:, perm].copy()
    for a in range(d):
        if flip is not None and flip[a]:
            pos[:, a], c[:, a] = 1 - pos[:, a], 1 - c[:, a]
    return pos, c, s, m, facet / (2 * 0.5)


def coefficient(nb, nid, nc, i, j):
    """c_ij as row i holds it (0 if j is not a neighbour of i)"""
    row = [int(x) for x in nid[i, : nb[i]]]
    return float(nc[i, row.index(j)]) if j in row else 0.0
