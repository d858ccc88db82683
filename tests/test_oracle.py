"""Pins the CPU oracle (oracle/sdot_oracle.c) before anything is compared with it: the reference's own
known-answer tests (tests/golden/known_answers.json), and independent checks that share no code with it --
brute force versus the grid search, Monte-Carlo sampling of `argmin |x - p|^2 - w`, the lifted convex hull,
finite differences for the Laplacian.  CPU only."""
import numpy as np
import pytest
from scipy.spatial import ConvexHull

import oracle as O
from helpers import monte_carlo_masses, neighbour_sets


def _cells(case, brute):
    pos = np.array(case["positions"], float)
    w = None if case["weights"] is None else np.array(case["weights"], float)
    return O.cells(pos, w, box=(np.array(case["lo"], float), np.array(case["hi"], float)), brute=brute)


@pytest.mark.parametrize("brute", [False, True])
def test_known_answers(known_answers, brute):
    for case in known_answers:
        r = _cells(case, brute)
        assert r["status"] == 0, case["name"]
        m = r["mass"]
        tol = case["atol"]
        if case.get("masses") is not None:
            assert np.abs(m - np.array(case["masses"])).max() < tol, (case["name"], m)
        for k, v in case.get("mass_at", {}).items():
            assert abs(m[int(k)] - v) < tol, (case["name"], m)
        if "total" in case:
            assert abs(m.sum() - case["total"]) < tol * max(1, case["total"]), (case["name"], m.sum())
        if case.get("positive"):
            assert (m > 0).all()


@pytest.mark.parametrize("d,n", [(2, 3000), (3, 600)])
def test_grid_search_is_the_brute_force(d, n):
    rng = np.random.default_rng(40 + d)
    pos = rng.uniform(size=(n, d))
    w = rng.uniform(0, 2e-3 if d == 2 else 5e-3, size=n)
    a, b = O.cells(pos, w), O.cells(pos, w, brute=True)
    assert a["status"] == 0 and b["status"] == 0
    assert np.abs(a["mass"] - b["mass"]).max() < 1e-14
    sa = neighbour_sets(a["nb"], a["nid"], a["nm"])
    sb = neighbour_sets(b["nb"], b["nid"], b["nm"])
    assert sa == sb
    assert abs(a["mass"].sum() - 1) < 1e-12


@pytest.mark.parametrize("brute", [False, True])
@pytest.mark.parametrize("shape", [(40, 30), (3, 3, 3), (12, 10, 8), (20, 20, 20)])
def test_grids_give_the_exact_boxes(shape, brute):
    """tests/test_CardCells.py:166-187, 900-941: seeds on a grid -- every vertex shared by 4 (2D) or 8 (3D) cells, cuts
    through vertices already on them -- have the grid's boxes as cells, 1e-10 relative"""
    d = len(shape)
    g = np.stack(np.meshgrid(*[(np.arange(k) + 0.5) / k for k in shape], indexing="ij"), axis=-1).reshape(-1, d)
    if brute and len(g) > 1000:
        pytest.skip("the brute-force search is quadratic")
    r = O.cells(g, brute=brute)
    assert r["status"] == 0
    assert np.abs(r["mass"] * len(g) - 1).max() < 1e-10


@pytest.mark.parametrize("d", [2, 3])
def test_a_seed_outside_and_lighter_duplicates(d):
    """tests/test_CardCells.py:180-187, 934-941: a seed outside the domain, and 19 seeds repeated with a weight 1e-4
    lower: the repeats' cells are empty and every other cell is the one of the cloud without them"""
    rng = np.random.default_rng(3 if d == 2 else 33)
    pos = rng.uniform(0.1, 0.9, size=(500, d))
    pos[0] = [1.5] + [0.5] * (d - 1)
    both = np.concatenate([pos, pos[1:20]])
    w = np.zeros(len(both))
    w[500:] = -1e-4
    a, b = O.cells(both, w), O.cells(pos)
    assert a["status"] == 0 and b["status"] == 0
    assert (a["mass"][500:] == 0).all()
    assert np.abs(a["mass"][:500] - b["mass"]).max() < 1e-15 and abs(a["mass"].sum() - 1) < 1e-12


@pytest.mark.parametrize("d", [2, 3])
def test_monte_carlo_partition(d):
    rng = np.random.default_rng(100 + d)
    pos = rng.uniform(0.1, 0.9, size=(8, d))
    w = rng.uniform(-0.02, 0.02, size=8)
    m = O.cells(pos, w)["mass"]
    mc = monte_carlo_masses(pos, np.zeros(d), np.ones(d), weights=w, nb_samples=200000)
    assert np.abs(m - mc).max() < 5e-3


def test_lifted_hull_gives_the_neighbours():
    """interior cells: their neighbours are the edges of the regular triangulation, the lower hull of (p, |p|^2 - w)"""
    rng = np.random.default_rng(3)
    n = 400
    pos = rng.uniform(size=(n, 2))
    w = rng.uniform(0, 1e-3, size=n)
    r = O.cells(pos, w)
    lifted = np.c_[pos, (pos ** 2).sum(axis=1) - w]
    hull = ConvexHull(lifted)
    edges = {i: set() for i in range(n)}
    for simplex, eq in zip(hull.simplices, hull.equations):
        if eq[2] < 0:                                   # lower facets
            for a in range(3):
                for b in range(3):
                    if a != b:
                        edges[simplex[a]].add(int(simplex[b]))
    got = neighbour_sets(r["nb"], r["nid"], r["nm"], rel_floor=0)
    checked = 0
    for i in range(n):
        if r["nb"][i] == len(got[i]) and 0.15 < pos[i, 0] < 0.85 and 0.15 < pos[i, 1] < 0.85:
            assert got[i] == edges[i], i
            checked += 1
    assert checked > 100


def test_a_constant_image_is_the_volume_up_to_its_mass():
    """tests/test_PowerDiagram.py:1527-1551: a constant image integrates to volume / total"""
    rng = np.random.default_rng(902)
    shape = (3, 4)
    pos = rng.uniform(0.2, np.array(shape) - 0.2, size=(12, 2))
    box = (np.zeros(2), np.array(shape, float))
    plain = O.cells(pos, box=box)["mass"]
    img = O.cells(pos, box=box, density=("image", [0, 0], [1, 1], np.full(shape, 1.0 / 12)))["mass"]
    assert np.abs(img - plain / 12).max() < 1e-12
    assert abs(img.sum() - 1) < 1e-12


def test_an_image_integrates_what_a_sampling_says():
    rng = np.random.default_rng(904)
    shape = (4, 3)
    values = rng.uniform(0, 1, size=shape)
    values[0, 0] = 0
    values /= values.sum()
    pos = rng.uniform(0.1, np.array(shape) - 0.1, size=(10, 2))
    got = O.cells(pos, box=(np.zeros(2), np.array(shape, float)), density=("image", [0, 0], [1, 1], values))["mass"]
    pts = rng.uniform(np.zeros(2), np.array(shape, float), size=(400000, 2))
    owner = ((pts[:, None, :] - pos[None]) ** 2).sum(axis=2).argmin(axis=1)
    dens = values[pts[:, 0].astype(int), pts[:, 1].astype(int)]
    ref = np.bincount(owner, weights=dens, minlength=10) / len(pts) * 12
    assert abs(got.sum() - 1) < 1e-12
    assert np.abs(got - ref).max() < 0.02


def test_gaussians_integrate_what_a_sampling_says():
    rng = np.random.default_rng(905)
    c = rng.uniform(0.3, 0.7, size=(3, 2))
    s = rng.uniform(0.08, 0.15, size=3)
    m = np.array([0.5, 0.3, 0.2])
    pos = rng.uniform(0.1, 0.9, size=(12, 2))
    got = O.cells(pos, density=("gauss", c, s, m))
    # the gaussian masses inside the unit box, by sampling the mixture and counting owners
    k = rng.choice(3, size=600000, p=m)
    pts = c[k] + s[k, None] * rng.standard_normal((600000, 2))
    inside = ((pts >= 0) & (pts <= 1)).all(axis=1)
    owner = ((pts[inside][:, None, :] - pos[None]) ** 2).sum(axis=2).argmin(axis=1)
    ref = np.bincount(owner, minlength=12) / len(pts)
    assert np.abs(got["mass"] - ref).max() < 3e-3
    # the exact closed-form facet fluxes are consistent with the masses: d m_i / d w_j = - c_ij
    w = np.zeros(12)
    i, j = 0, int(got["nid"][0, 0])
    h = 1e-7
    wp = w.copy(); wp[j] += h
    wm = w.copy(); wm[j] -= h
    fd = (O.cells(pos, wp, density=("gauss", c, s, m))["mass"][i] - O.cells(pos, wm, density=("gauss", c, s, m))["mass"][i]) / (2 * h)
    assert abs(fd + got["nc"][0, 0]) < 1e-6 * max(1, abs(fd))


def test_3d_gaussians_integrate_what_a_sampling_says():
    """the oracle's tetrahedral quadrature of 3D gaussians: total = the mixture's mass in the cube (erf products),
    cells = what a sampling of the mixture gives, and the face integrals are the Jacobian: d m_i / d w_j = - c_ij"""
    from scipy.special import erf
    rng = np.random.default_rng(906)
    c = rng.uniform(0.3, 0.7, size=(2, 3))
    s = np.array([0.1, 0.13])
    m = np.array([0.6, 0.4])
    pos = rng.uniform(0.1, 0.9, size=(40, 3))
    got = O.cells(pos, density=("gauss", c, s, m))
    assert got["status"] == 0
    inside = sum(m[k] * np.prod([0.5 * (erf((1 - c[k, a]) / (s[k] * np.sqrt(2))) - erf(-c[k, a] / (s[k] * np.sqrt(2)))) for a in range(3)])
                 for k in range(2))
    assert abs(got["mass"].sum() - inside) < 1e-12
    k = rng.choice(2, size=600000, p=m)
    pts = c[k] + s[k, None] * rng.standard_normal((600000, 3))
    keep = ((pts >= 0) & (pts <= 1)).all(axis=1)
    owner = ((pts[keep][:, None, :] - pos[None]) ** 2).sum(axis=2).argmin(axis=1)
    ref = np.bincount(owner, minlength=40) / len(pts)
    assert np.abs(got["mass"] - ref).max() < 3e-3
    big = np.nonzero(got["mass"] > 0.02)[0]
    bref = np.array([pts[keep][owner == i].mean(axis=0) for i in big])
    assert np.abs(got["bary"][big] - bref).max() < 5e-3
    w = np.zeros(40)
    i, j = 0, int(got["nid"][0, 0])
    h = 1e-6
    wp = w.copy(); wp[j] += h
    wm = w.copy(); wm[j] -= h
    fd = (O.cells(pos, wp, density=("gauss", c, s, m))["mass"][i] - O.cells(pos, wm, density=("gauss", c, s, m))["mass"][i]) / (2 * h)
    assert abs(fd + got["nc"][0, 0]) < 1e-5 * max(1e-3, abs(fd))


@pytest.mark.parametrize("d", [2, 3])
def test_a_gaussian_facet_is_the_closed_form(d):
    """tests/test_SumOfGaussians.py:20-43: the facet x = 1/2 of two seeds under three gaussians (narrow, mid, wide) is a
    product of erf factors; 1e-12 relative, from both sides, under every symmetry of the cube (the reference rotates
    its domain; the box of this path is axis-aligned, so the rotations are the cube's own)"""
    import itertools
    from helpers import coefficient, gaussian_facet_case
    for perm in itertools.permutations(range(d)):
        for flip in itertools.product([0, 1], repeat=d):
            pos, c, s, m, ref = gaussian_facet_case(d, perm, flip)
            r = O.cells(pos, density=("gauss", c, s, m), want=("facets",))
            assert r["status"] == 0
            for i, j in ((0, 1), (1, 0)):
                got = coefficient(r["nb"], r["nid"], r["nc"], i, j)
                assert abs(got - ref) < 1e-12 * ref, (perm, flip, i, got, ref)


def test_3d_gaussian_facets_agree_from_both_sides():
    """tests/test_SumOfGaussians.py:46-61: 30 seeds, oblique facets cut by their neighbours, each integrated from both
    of its cells; the Laplacian is symmetric to 1e-12 of its largest entry"""
    rng = np.random.default_rng(33)
    n = 30
    pos = rng.uniform(0.1, 0.9, size=(n, 3))
    w0 = rng.uniform(-0.01, 0.01, n)
    c = rng.uniform(0.3, 0.7, size=(3, 3))
    m = np.array([0.5, 1.0, 0.7])
    r = O.cells(pos, w0, density=("gauss", c, np.array([0.04, 0.2, 0.35]), m / m.sum()), want=("facets",))
    assert r["status"] == 0
    H = np.zeros((n, n))
    for i in range(n):
        for q in range(r["nb"][i]):
            H[i, r["nid"][i, q]] -= r["nc"][i, q]
            H[i, i] += r["nc"][i, q]
    assert (H - np.diag(np.diag(H)) < 0).sum() > 2 * n
    assert np.abs(H - H.T).max() < 1e-12 * np.abs(H).max()


@pytest.mark.parametrize("d", [2, 3])
def test_the_laplacian_is_the_jacobian_of_the_measures(d):
    """tests/test_SdotPlanNd.py:184-243: d m_i / d w_j = - c_ij, d m_i / d w_i = sum_j c_ij"""
    rng = np.random.default_rng(70 + d)
    n = 30 if d == 2 else 20
    pos = rng.uniform(size=(n, d))
    w = rng.uniform(0, 1e-3, size=n)
    r = O.cells(pos, w)
    h = 1e-7
    for i in range(0, n, 7):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        col = (O.cells(pos, wp)["mass"] - O.cells(pos, wm)["mass"]) / (2 * h)
        expect = np.zeros(n)
        for k in range(r["nb"][i]):
            expect[r["nid"][i, k]] -= r["nc"][i, k]
        expect[i] = r["nc"][i, : r["nb"][i]].sum()
        assert np.abs(col - expect).max() < 1e-5 * np.abs(expect).max(), i


def test_moments_match_a_sampling():
    rng = np.random.default_rng(11)
    pos = rng.uniform(0.1, 0.9, size=(6, 2))
    r = O.cells(pos)
    pts = rng.uniform(size=(400000, 2))
    owner = ((pts[:, None, :] - pos[None]) ** 2).sum(axis=2).argmin(axis=1)
    for i in range(6):
        sel = pts[owner == i]
        assert np.abs(sel.mean(axis=0) - r["bary"][i]).max() < 5e-3
        assert abs(((sel - pos[i]) ** 2).sum(axis=1).sum() / len(pts) - r["cost"][i]) < 2e-4


@pytest.mark.parametrize("d", [2, 3])
def test_moments_are_the_closed_forms(d):
    """tests/test_SdotPlanNd.py:460-498: one seed owns the unit square (cube): mass 1, barycentre the centre,
    `int |x|^2 = d / 3`; one lit pixel of an image puts the barycentre at that pixel's centre (the orientation of the
    grid: `values[i, j]` at `origin + (i, j) * step`); 15 seeds share those moments"""
    def second(r, pos):
        first = r["mass"][:, None] * r["bary"]
        return r["cost"] + 2 * (pos * first).sum(axis=1) - (pos * pos).sum(axis=1) * r["mass"]
    one = np.array([[0.3, 0.6, 0.2][:d]])
    r = O.cells(one)
    assert abs(r["mass"][0] - 1) < 1e-12 and np.abs(r["bary"][0] - 0.5).max() < 1e-12
    assert abs(second(r, one)[0] - d / 3) < 1e-12
    pos = np.random.default_rng(11).uniform(0.1, 0.9, size=(15, d))
    r = O.cells(pos)
    assert np.abs((r["mass"][:, None] * r["bary"]).sum(axis=0) - 0.5).max() < 1e-12
    assert abs(second(r, pos).sum() - d / 3) < 1e-12
    if d == 2:
        values = np.zeros((4, 3))
        values[3, 1] = 1 / (0.5 * 0.25)     # normalised, as `Image.normalized_version` makes it
        r = O.cells(one, box=(np.zeros(2), np.array([2.0, 0.75])), density=("image", [0, 0], [0.5, 0.25], values))
        assert abs(r["mass"][0] - 1) < 1e-12
        assert np.abs(r["bary"][0] - [3.5 * 0.5, 1.5 * 0.25]).max() < 1e-12


def test_many_gaussians_stay_exact():
    """tests/test_SdotPlanNd.py:1884-1902: 400 gaussians of width 0.01 along an arc, 100 seeds drawn in the unit square
    (most outside the support box: the similarity start), `continuation = "always"`: converged to 1e-11 through more
    than 5 widths, and a diagram at the fitted weights on the exact density gives the target masses to 1e-9"""
    rng = np.random.default_rng(5)
    G = 400
    t = rng.uniform(0.2 * np.pi, 0.8 * np.pi, G)
    r = 0.35 + 0.02 * rng.standard_normal(G)
    c = np.c_[0.5 + r * np.cos(t), 0.2 + r * np.sin(t)]
    s = np.full(G, 0.01)
    lo, hi = (c - 6 * s[:, None]).min(axis=0), (c + 6 * s[:, None]).max(axis=0)
    dens = ("gauss", c, s, np.full(G, 1 / G))
    pos = rng.uniform(0, 1, (100, 2))
    sol = O.solve(pos, box=(lo, hi), density=dens, tol_abs=1e-11, maxit=200, continuation=2)
    assert sol["stats"]["status"] == 1 and sol["stats"]["nb_continuation_steps"] > 5, sol["stats"]
    m = O.cells(pos, sol["weights"], box=(lo, hi), density=dens)["mass"]
    assert np.abs(m - sol["stats"]["domain_mass"] / 100).max() < 1e-9


def test_newton_reaches_the_target_masses():
    """tests/test_SdotPlanNd.py:39-62: the fitted masses are the targets"""
    rng = np.random.default_rng(1)
    n = 2000
    pos = rng.uniform(size=(n, 2))
    s = O.solve(pos, tol_abs=0.0, tol_rel=1e-8)
    assert s["stats"]["status"] == 1
    assert np.abs(s["masses"] - 1 / n).max() * n <= 1e-8
    assert s["weights"][0] == 0
    # an independent diagram at the fitted weights agrees
    m = O.cells(pos, s["weights"], brute=True)["mass"]
    assert np.abs(m - 1 / n).max() * n < 1e-8


def _gaussian_target(c, s, m):
    """the oracle's density and domain of a sum of gaussians: the masses normalised, the box `c +- 6 sigma`
    (distributions/SumOfGaussians.py, the declared support)"""
    lo, hi = (c - 6 * s[:, None]).min(axis=0), (c + 6 * s[:, None]).max(axis=0)
    return ("gauss", c, s, m / m.sum()), (lo, hi)


def test_a_nonzero_start_is_kept_and_converges():
    """tests/test_SdotPlanNd.py:137-158: 18 seeds, two overlapping gaussians (the soft case, the reference's
    `_overlapping_target(2, 2, seed=3)`), small random start weights that empty no cell: kept, and converged"""
    rng = np.random.default_rng(2)
    pos = rng.uniform(0.1, 0.9, size=(18, 2))
    g = np.random.default_rng(3)
    c = 0.5 + g.uniform(-0.12, 0.12, size=(2, 2))
    dens, box = _gaussian_target(c, g.uniform(0.18, 0.24, 2), g.uniform(0.6, 1.4, 2))
    w0 = rng.uniform(-0.003, 0.003, 18)
    s = O.solve(pos, box=box, density=dens, w0=w0, tol_abs=1e-12, maxit=50)
    assert s["stats"]["status"] == 1 and s["stats"]["start"] == 0
    assert np.abs(s["masses"] - s["stats"]["domain_mass"] / 18).max() < 1e-10


@pytest.mark.parametrize("continuation", [0, 1])
def test_no_cell_dies_on_scattered_targets(continuation):
    """tests/test_SdotPlanNd.py:160-182: 40 seeds, four narrow separate gaussians (the hard case, the reference's
    `_scattered_target(2, 4, seed=6)`): no cell is empty at any step of the history, and the fit reaches the targets"""
    rng = np.random.default_rng(5)
    pos = rng.uniform(0.1, 0.9, size=(40, 2))
    g = np.random.default_rng(6)
    c = g.uniform(0.3, 0.7, size=(4, 2))
    dens, box = _gaussian_target(c, np.full(4, 0.13), g.uniform(0.7, 1.3, 4))
    s = O.solve(pos, box=box, density=dens, tol_abs=1e-12, maxit=200, continuation=continuation)
    assert s["stats"]["status"] == 1
    assert (s["history"][:, 3] > 0).all()
    assert np.abs(s["masses"] - s["stats"]["domain_mass"] / 40).max() < 1e-10


def test_newton_converges_quadratically_on_an_image():
    """tests/test_SdotPlanNd.py:245-277 on the oracle: 300 seeds on a soft 24 x 24 image converge in few steps, the last
    two each an order of magnitude (the quadratic phase); a warm start from a neighbouring cloud's weights takes at most
    6; a warm start that empties cells is dropped for the Voronoi start. (The reference's 2D default is its LIMITS step,
    which takes no backtrack here; the oracle's TRIALS take one at the first step.)"""
    rng = np.random.default_rng(41)
    n = 300
    pos = rng.uniform(0.05, 0.95, size=(n, 2))
    vals = 1 + 0.5 * rng.random((24, 24))
    dens = ("image", [0, 0], [1 / 24, 1 / 24], vals * (24 * 24 / vals.sum()))
    s = O.solve(pos, density=dens, tol_abs=1e-10 / n, maxit=60)
    res = s["history"][:, 4] * n
    assert s["stats"]["status"] == 1 and res[-1] < 1e-9 and len(res) < 30
    assert res[-1] < 0.1 * res[-2] < 0.01 * res[-3]
    assert np.abs(s["masses"] - 1 / n).max() < 1e-11
    warm = O.solve(pos + 1e-4 * rng.normal(size=pos.shape), density=dens, tol_abs=1e-10 / n, maxit=60, w0=s["weights"])
    assert warm["stats"]["status"] == 1 and warm["stats"]["start"] == 0 and len(warm["history"]) <= 6
    bad = O.solve(pos, density=dens, tol_abs=1e-10 / n, maxit=60, w0=rng.uniform(-1, 1, n))
    assert bad["stats"]["status"] == 1 and bad["stats"]["start"] == 1


def test_log_and_lin_residuals_reach_the_same_plan():
    """tests/test_SdotPlanNd.py:327-348"""
    rng = np.random.default_rng(2)
    n = 500
    pos = rng.uniform(size=(n, 2))
    a = O.solve(pos, tol_abs=1e-13, residual=1)
    b = O.solve(pos, tol_abs=1e-13, residual=0)
    assert a["stats"]["status"] == 1 and b["stats"]["status"] == 1
    assert np.abs(a["weights"] - b["weights"]).max() < 1e-9 * np.abs(a["weights"]).max()


def test_newton_in_3d():
    rng = np.random.default_rng(5)
    n = 400
    pos = rng.uniform(size=(n, 3))
    s = O.solve(pos, tol_abs=0.0, tol_rel=1e-8)
    assert s["stats"]["status"] == 1
    assert np.abs(s["masses"] * n - 1).max() <= 1e-8


def test_the_similarity_start_when_seeds_are_outside():
    """tests/test_SdotPlanNd.py:279-306: the Voronoi start has empty cells, the similarity start does not"""
    rng = np.random.default_rng(9)
    pos = rng.uniform(0.5, 1.5, size=(200, 2))
    s = O.solve(pos, tol_abs=1e-11)
    assert s["stats"]["start"] == 2
    assert s["stats"]["status"] == 1


@pytest.mark.parametrize("d", [2, 3])
def test_near_coincident_seeds_tile_the_domain(d):
    """two cells of seeds 1e-12 apart share their plane to the bit: the diagram's masses sum to the domain's (the plane
    offset takes the weights' difference before |q|^2, and both faces of an edge make the same crossing point)"""
    from helpers import degenerate_clouds
    for name in ("pair at 1e-9", "pair at 1e-12", "triple at 1e-10"):
        pos, _ = degenerate_clouds(d, 17)[name]
        rng = np.random.default_rng(1)
        for w in (None, 1e-3 * rng.standard_normal(len(pos))):
            for brute in (False, True):
                m = O.cells(pos, w, brute=brute)["mass"]
                assert abs(m.sum() - 1) < 1e-15, (d, name, brute, m.sum() - 1)


@pytest.mark.parametrize("d", [2, 3])
def test_aggregation_merges_what_the_doubles_cannot_separate(d):
    """tests/test_SdotPlanNd.py:1437-1453 on the oracle: with the aggregation the near-coincident groups are merged and
    the solve converges on the clusters (status 7); without it, it stagnates at the floor of the weights' doubles"""
    from helpers import degenerate_clouds
    for name, (pos, groups) in degenerate_clouds(d, 17).items():
        if len(np.unique(pos, axis=0)) < len(pos):
            continue                     # exact duplicates are the API layer's (they never reach a solver)
        n = len(pos)
        tol = 1e-11 / n
        r = O.solve(pos, tol_abs=tol, maxit=60, agg_margin=4.0)
        st = r["stats"]
        assert st["status"] == 7 and st["residual"] <= tol, (d, name, st["status"], st["residual"])
        assert st["nb_clusters"] == len(groups) and st["nb_aggregated"] == sum(len(g) for g, _ in groups), (d, name)
        cl = r["clusters"]
        alone = np.ones(n, dtype=bool)
        for members, _ in groups:
            assert (cl[members] == min(members)).all(), (d, name, cl[members])
            alone[members] = False
            assert abs(r["masses"][members].sum() - len(members) / n) <= len(members) * tol * (1 + 1e-9), (d, name)
        assert (cl[alone] == np.arange(n)[alone]).all()
        assert np.abs(r["masses"][alone] - 1 / n).max() <= tol, (d, name)
        off = O.solve(pos, tol_abs=tol, maxit=60)
        assert off["stats"]["status"] not in (1, 7), (d, name, off["stats"]["status"])
        assert off["stats"]["nb_clusters"] == 0


def test_aggregation_changes_nothing_without_such_seeds():
    """tests/test_SdotPlanNd.py:1486-1507: a cloud without near pairs gives the same plan, to the bit, with or without it"""
    rng = np.random.default_rng(8)
    pos = rng.uniform(size=(1500, 2))
    t = O.max_threads()
    O.set_threads(1)                     # (the threads' reductions would differ in the last bits from run to run)
    try:
        on = O.solve(pos, tol_abs=1e-10 / 1500, agg_margin=4.0)
        off = O.solve(pos, tol_abs=1e-10 / 1500)
    finally:
        O.set_threads(t)
    assert on["stats"]["status"] == 1 and on["stats"]["nb_clusters"] == 0
    assert np.array_equal(on["weights"], off["weights"])


def test_the_image_continuation_solves_what_direct_newton_cannot():
    """tests/test_SdotPlanNd.py:397-405 on the oracle: an almost empty image but for two spots. Direct Newton fails; the
    blur continuation (the image widened on its grid, sdotplan/convolved/Image.h) converges, and `auto` starts it"""
    rng = np.random.default_rng(91)
    pos = rng.uniform(0, 1, size=(400, 2))
    values = np.full((32, 32), 1e-6)
    values[6:10, 6:10] = 1.0
    values[20:26, 18:24] = 0.7
    dens = ("image", [0.0, 0.0], [1 / 32, 1 / 32], values)
    direct = O.solve(pos, density=dens, tol_abs=0.0, tol_rel=1e-6, maxit=60, continuation=0)
    assert direct["stats"]["status"] != 1
    for cont in (1, 2):
        r = O.solve(pos, density=dens, tol_abs=0.0, tol_rel=1e-6, maxit=100, continuation=cont)
        st = r["stats"]
        assert st["status"] == 1 and st["nb_continuation_steps"] > 1, (cont, st)
        nu = np.full(400, st["domain_mass"] / 400)
        assert np.abs(r["masses"] / nu - 1).max() <= 1e-6
        s = r["history"][:, 7]
        assert s[0] > 0 and s[-1] == 0 and (np.diff(s) <= 0).all()
