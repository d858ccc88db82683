"""Parity of the GPU cells (through the C ABI) with the oracle and with the reference's known answers.

Tolerances: FP64 masses within 1e-10 relative of the oracle's (tighter than the reference, which pins its
FP64 card at 1e-9, tests/test_CardCells.py:48-73); neighbour sets of non-degenerate facets bit-exact (a facet
below 1e-9 of its cell's largest is degenerate: its presence is decided by rounding); c_ij within 1e-9.
"""
import numpy as np
import pytest

import oracle as O
import sdot
from helpers import compare_neighbours, degenerate_pairs, neighbour_sets
from sdot import PowerDiagram, box_half_spaces

pytestmark = pytest.mark.gpu


def _pd(pos, w=None, lo=None, hi=None, dist=None, kernel_dtype=None):
    d = pos.shape[1]
    lo = np.zeros(d) if lo is None else lo
    hi = np.ones(d) if hi is None else hi
    return PowerDiagram(pos, w, boundaries=box_half_spaces(lo, hi), distribution=dist, kernel_dtype=kernel_dtype)


def test_known_answers(known_answers):
    for case in known_answers:
        pos = np.array(case["positions"], float)
        w = None if case["weights"] is None else np.array(case["weights"], float)
        m = _pd(pos, w, np.array(case["lo"], float), np.array(case["hi"], float)).measures
        tol = case["atol"]
        if case.get("masses") is not None:
            assert np.abs(m - np.array(case["masses"])).max() < tol, (case["name"], m)
        for k, v in case.get("mass_at", {}).items():
            assert abs(m[int(k)] - v) < tol, (case["name"], m)
        if "total" in case:
            assert abs(m.sum() - case["total"]) < tol * max(1, case["total"]), case["name"]


def _compare(pos, w, dens=None, n_check=None, kernel_dtype=None):
    d = pos.shape[1]
    lo, hi = np.zeros(d), np.ones(d)
    od = None
    dist = None
    if dens is not None:
        od, dist = dens
    ref = O.cells(pos, w, box=(lo, hi), density=od)
    pd = _pd(pos, w, lo, hi, dist, kernel_dtype)
    nb, ids, coef, meas = pd.facets()
    m, bary, cost = pd.barycenters_and_costs()
    assert ref["status"] == 0
    rm = ref["mass"]
    full = rm > 1e-14 * rm.max()
    assert np.abs(m[full] - rm[full]).max() <= 1e-10 * rm[full].max()
    # relative 1e-10 per cell; a cell far in a gaussian's tail (mass 1e4 below the mean) is held to 1e-14 of the mean mass
    assert (np.abs(m - rm) <= 1e-10 * rm + 1e-14 * rm.mean()).mean() > 0.999
    # barycentres: first moment / mass, so a cell in a gaussian's far tail (mass ~1e-20) has an ill-conditioned one;
    # held through its first moment m (b - p), and directly where the cell carries a visible share of the mass
    fm = (bary - pos) * m[:, None]
    fr = (ref["bary"] - pos) * rm[:, None]
    assert np.abs(fm - fr).max() <= 1e-10 * rm.max()
    heavy = rm > 1e-6 * rm.max()
    assert np.abs(bary[heavy] - ref["bary"][heavy]).max() < 1e-9
    assert np.abs(cost - ref["cost"]).max() <= 1e-9 * ref["cost"].max()
    # neighbour sets of the non-degenerate facets, bit-exact
    ga = neighbour_sets(nb, ids, meas)
    gb = neighbour_sets(ref["nb"], ref["nid"], ref["nm"])
    skip = degenerate_pairs(ref["nb"], ref["nid"], ref["nm"]) | degenerate_pairs(nb, ids, meas)
    assert compare_neighbours(ga, gb, skip) == 0
    # c_ij of the non-degenerate facets: relative to the row's largest coefficient (a short facet's own relative
    # error grows as its length shrinks), and the median relative error (tests/test_CardCells.py:259-312)
    worst, rels = 0.0, []
    for i in range(0, len(pos), max(1, len(pos) // 2000)):
        a = {int(j): c for j, c in zip(ids[i, : nb[i]], coef[i, : nb[i]])}
        top = ref["nc"][i, : ref["nb"][i]].max() if ref["nb"][i] else 0
        for j, c in zip(ref["nid"][i, : ref["nb"][i]], ref["nc"][i, : ref["nb"][i]]):
            if int(j) in a and c > 1e-9 * top:
                worst = max(worst, abs(a[int(j)] - c) / top)
                rels.append(abs(a[int(j)] - c) / c)
    assert worst < 1e-10, worst
    assert np.median(rels) < 1e-12
    return m


@pytest.mark.parametrize("n,wscale", [(1000, 0.0), (20000, 0.0), (20000, 2e-5), (100000, 5e-6)])
def test_uniform_cells_match_the_oracle(n, wscale):
    rng = np.random.default_rng(n + int(wscale * 1e7))
    pos = rng.uniform(size=(n, 2))
    w = rng.uniform(0, wscale, size=n) if wscale else None
    m = _compare(pos, w)
    assert abs(m.sum() - 1) < 1e-12


@pytest.mark.parametrize("case", ["uniform", "weights", "image", "gaussians"])
def test_the_fp32_clip_matches_the_oracle(case):
    """precision "mixed" (kernel_dtype FP32: the clip in FP32, a vertex within the FP32 band of a plane re-checked in FP64,
    every vertex re-solved in FP64 before the integration -- the reference's float kernel, gpu/Cell2D.cuh:56-60, 991-1042)
    against the FP64 oracle, with the FP64 clip's tolerances: masses within 1e-10 relative, neighbour sets of the
    non-degenerate facets bit-exact, c_ij within 1e-10 of the row's largest"""
    rng = np.random.default_rng(77)
    n = 20000
    pos = rng.uniform(size=(n, 2))
    w = rng.uniform(0, 2e-5, size=n) if case == "weights" else None
    dens = None
    if case == "image":
        img = sdot.Image(rng.uniform(0.1, 1.0, size=(64, 48)), frame=[1 / 64, 1 / 48])
        dens = (("image", [0, 0], [1 / 64, 1 / 48], img.normalized_version().values), img)
    if case == "gaussians":
        c, s = rng.uniform(0.3, 0.7, size=(4, 2)), rng.uniform(0.05, 0.15, size=4)
        g = sdot.SumOfGaussians(c, s, support_box=(np.zeros(2), np.ones(2)))
        dens = (("gauss", c, s, g.normalized_version().weights), g)
    m = _compare(pos, w, dens, kernel_dtype="FP32")
    if case in ("uniform", "weights"):
        assert abs(m.sum() - 1) < 1e-12


@pytest.mark.parametrize("n,wscale", [(20000, 0.0), (100000, 1.0)])
def test_the_fp32_clip_gives_the_fp64_cells(n, wscale):
    """the FP32 clip decides every vertex as the FP64 one (its band sends the doubtful ones to an FP64 re-check) and
    re-solves every vertex from the same two lines: the same neighbour tables as the FP64 clip, masses, centroids and
    coefficients within 1e-13 relative; the two kernels' times are printed side by side"""
    import time
    from sdot import _lib
    rng = np.random.default_rng(5 + n)
    pos = rng.uniform(size=(n, 2))
    w = rng.uniform(0, wscale * n ** -1.0, size=n) if wscale else None
    out = {}
    for dt in ("FP64", "FP32"):
        pd = _pd(pos, w, kernel_dtype=dt)
        pd.facets()
        _lib.set_timing(True)
        _lib.kernel_stats(reset=True)
        nb, ids, coef, meas = _pd(pos, w, kernel_dtype=dt).facets()
        ms = _lib.kernel_stats()["cells2d"][0]
        _lib.set_timing(False)
        m, bary, _ = _pd(pos, w, kernel_dtype=dt).barycenters_and_costs()
        out[dt] = (nb, ids, coef, m, bary, ms)
    (nb, ids, coef, m, bary, t64), (nb2, ids2, coef2, m2, bary2, t32) = out["FP64"], out["FP32"]
    assert (nb == nb2).all()
    for i in range(n):
        assert set(ids[i, : nb[i]]) == set(ids2[i, : nb2[i]]), i
    assert np.abs(m - m2).max() <= 1e-13 * m.max()
    assert np.abs(bary - bary2).max() <= 1e-12
    assert np.abs(np.sort(coef, axis=1) - np.sort(coef2, axis=1)).max() <= 1e-13 * coef.max()
    print(f"\n2D cells, {n} seeds: FP64 clip {1e6 * t64 / n:.2f} ns per cell, FP32 clip {1e6 * t32 / n:.2f} ns per cell")


@pytest.mark.parametrize("n,wscale", [(500, 0.0), (20000, 0.0), (20000, 2e-4)])
def test_3d_cells_match_the_oracle(n, wscale):
    """3D: volumes, centroids, costs, neighbour sets and face areas (the off-diagonals area / 2|p_i - p_j|)"""
    rng = np.random.default_rng(3 * n + int(wscale * 1e5))
    pos = rng.uniform(size=(n, 3))
    w = rng.uniform(0, wscale, size=n) if wscale else None
    m = _compare(pos, w)
    assert abs(m.sum() - 1) < 1e-12


def test_cells_are_deterministic():
    rng = np.random.default_rng(8)
    pos = rng.uniform(size=(30000, 2))
    w = rng.uniform(0, 1e-5, size=30000)
    a = _pd(pos, w).hessian_rows()
    b = _pd(pos, w).hessian_rows()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_image_density_matches_the_oracle():
    rng = np.random.default_rng(21)
    vals = rng.uniform(0.1, 1.0, size=(64, 48))
    vals[:5, :7] = 0
    img = sdot.Image(vals, frame=[1 / 64, 1 / 48])
    norm = img.normalized_version()
    pos = rng.uniform(size=(3000, 2))
    w = rng.uniform(0, 1e-4, size=3000)
    m = _compare(pos, w, (("image", [0, 0], [1 / 64, 1 / 48], norm.values), img))
    assert abs(m.sum() - 1) < 1e-12


def test_gaussian_density_matches_the_oracle():
    rng = np.random.default_rng(22)
    c = rng.uniform(0.3, 0.7, size=(4, 2))
    s = rng.uniform(0.05, 0.15, size=4)
    g = sdot.SumOfGaussians(c, s, support_box=(np.zeros(2), np.ones(2)))
    ng = g.normalized_version()
    pos = rng.uniform(size=(2000, 2))
    _compare(pos, None, (("gauss", c, s, ng.weights), g))


@pytest.mark.parametrize("n", [400, 1500])
def test_3d_gaussian_density_matches_the_oracle(n):
    """3D sums of gaussians: face integrals (Gauss's theorem, angular Gauss-Legendre) on the GPU against the
    oracle's adaptive tetrahedral quadrature; the total is the mixture's mass inside the cube (erf products)"""
    from scipy.special import erf
    rng = np.random.default_rng(23 + n)
    c = rng.uniform(0.2, 0.8, size=(4, 3))
    s = rng.uniform(0.05, 0.15, size=4)
    g = sdot.SumOfGaussians(c, s, support_box=(np.zeros(3), np.ones(3)))
    ng = g.normalized_version()
    pos = rng.uniform(size=(n, 3))
    m = _compare(pos, None, (("gauss", c, s, ng.weights), g))
    inside = sum(wk * np.prod([0.5 * (erf((1 - c[k, a]) / (s[k] * np.sqrt(2))) - erf(-c[k, a] / (s[k] * np.sqrt(2)))) for a in range(3)])
                 for k, wk in enumerate(ng.weights))
    assert abs(m.sum() - inside) < 1e-12


@pytest.mark.parametrize("d", [2, 3])
def test_a_gaussian_facet_is_the_closed_form(d):
    """tests/test_SumOfGaussians.py:20-43 through the C ABI: the facet x = 1/2 of two seeds under a narrow, a mid and a
    wide gaussian is a product of erf factors; 1e-12 relative (the reference's bar), from both cells, under a rotation
    of the cube about each axis and a reflection (the box of this path is axis-aligned)"""
    from helpers import coefficient, gaussian_facet_case
    maps = [(None, None), ((1, 0), (0, 1))] if d == 2 else [(None, None), ((1, 2, 0), (0, 0, 1)), ((2, 0, 1), (1, 0, 0))]
    for perm, flip in maps:
        pos, c, s, m, ref = gaussian_facet_case(d, perm, flip)
        nb, ids, vals = _pd(pos, dist=sdot.SumOfGaussians(c, s, m)).hessian_rows()
        for i, j in ((0, 1), (1, 0)):
            got = coefficient(nb, ids, vals, i, j)
            assert abs(got - ref) < 1e-12 * ref, (perm, flip, i, got, ref)


def test_3d_gaussian_facets_agree_from_both_sides():
    """tests/test_SumOfGaussians.py:46-61 through the C ABI: 30 seeds under gaussians of widths 0.04, 0.2 and 0.35,
    oblique facets each integrated by both of its cells; symmetric to 1e-12 of the largest entry, and each row's
    coefficients those of the oracle to 1e-10 of that entry"""
    rng = np.random.default_rng(33)
    n = 30
    pos = rng.uniform(0.1, 0.9, size=(n, 3))
    w0 = rng.uniform(-0.01, 0.01, n)
    c = rng.uniform(0.3, 0.7, size=(3, 3))
    s = np.array([0.04, 0.2, 0.35])
    m = np.array([0.5, 1.0, 0.7])
    nb, ids, vals = _pd(pos, w0, dist=sdot.SumOfGaussians(c, s, m)).hessian_rows()
    ref = O.cells(pos, w0, box=(np.zeros(3), np.ones(3)), density=("gauss", c, s, m / m.sum()), want=("facets",))

    def dense(nb, ids, vals):
        H = np.zeros((n, n))
        for i in range(n):
            for q in range(nb[i]):
                H[i, ids[i, q]] -= vals[i, q]
                H[i, i] += vals[i, q]
        return H
    H, R = dense(nb, ids, vals), dense(ref["nb"], ref["nid"], ref["nc"])
    assert (H - np.diag(np.diag(H)) < 0).sum() > 2 * n
    assert np.abs(H - H.T).max() < 1e-12 * np.abs(H).max()
    assert np.abs(H - R).max() < 1e-10 * np.abs(R).max()


def test_the_laplacian_is_bit_symmetric():
    rng = np.random.default_rng(4)
    n = 20000
    pos = rng.uniform(size=(n, 2))
    w = rng.uniform(0, 1e-5, size=n)
    row, cols, vals, dia = _pd(pos, w).laplacian()
    import scipy.sparse as sp
    A = sp.csr_matrix((vals, cols, row[:-1].tolist() + [row[-1]]), shape=(n, n))
    assert (A != A.T).nnz == 0
    assert np.array_equal(A.data, A.T.tocsr().data) or (abs(A - A.T)).max() == 0
    rs = np.asarray(A.sum(axis=1)).reshape(-1)
    full = np.diff(row) > 0                     # an empty row (an empty cell) carries dia = 1 (sdotplan/Laplacian.h:56-61)
    assert np.abs(rs[full] - dia[full]).max() <= 1e-15 * dia.max()
    assert (dia[~full] == 1).all()
    ref = O.cells(pos, w)
    for i in range(0, n, 97):
        a = dict(zip(cols[row[i]:row[i + 1]], vals[row[i]:row[i + 1]]))
        for j, c in zip(ref["nid"][i, : ref["nb"][i]], ref["nc"][i, : ref["nb"][i]]):
            if c > 1e-8 * ref["nc"][i].max():
                assert abs(a[int(j)] - c) <= 1e-10 * ref["nc"][i].max()


def test_the_linear_solve_matches_a_direct_solve():
    rng = np.random.default_rng(5)
    n = 5000
    pos = rng.uniform(size=(n, 2))
    pd = _pd(pos)
    row, cols, vals, dia = pd.laplacian()
    b = rng.standard_normal(n)
    b -= b.mean()
    x = pd.laplacian_solve(b, tol=1e-13)
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    L = sp.diags(dia) - sp.csr_matrix((vals, cols, row), shape=(n, n))
    y = np.zeros(n)
    y[1:] = sla.spsolve(L[1:, 1:].tocsc(), b[1:])
    assert x[0] == 0
    assert np.abs(x - y).max() < 1e-8 * np.abs(y).max()


@pytest.mark.parametrize("d,n", [(2, 40000), (3, 20000)])
def test_both_linear_methods_match_a_direct_solve(d, n):
    """sdot_linear_solve with method 0 (Jacobi-PCG), 1 (multigrid-PCG, FP32 levels), and 2 / 3 (the same with the CG in
    FP32 inside an FP64 iterative refinement) on the Laplacian of a Voronoi diagram, against scipy's direct solve of the
    gauge-fixed system, two right-hand sides: the refinement reaches the FP64 solves' 1e-8 of the solution's size"""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    from sdot import _lib
    rng = np.random.default_rng(50 + d)
    pos = rng.uniform(size=(n, d))
    row, cols, vals, dia = _pd(pos).laplacian()             # Voronoi: no empty cell, one connected graph, a consistent system
    assert (np.diff(row) > 0).all()
    b = rng.standard_normal((2, n))
    b -= b.mean(axis=1, keepdims=True)
    L = sp.diags(dia) - sp.csr_matrix((vals, cols, row), shape=(n, n))
    lu = sla.splu(L[1:, 1:].tocsc())
    y = np.zeros((2, n))
    for k in range(2):
        y[k, 1:] = lu.solve(b[k, 1:])
    its = {}
    for method in (0, 1, 2, 3):
        x, it = _lib.linear_solve(row, cols, vals, dia, b, tol=1e-12, method=method)
        assert (x[:, 0] == 0).all()
        assert np.abs(x - y).max() < 1e-8 * np.abs(y).max(), method
        its[method] = np.asarray(it)
    assert (its[1] > 0).all() and (its[1] < its[0]).all(), its
    assert (its[2] > 0).all() and (its[3] > 0).all() and (its[3] < its[2]).all(), its


def test_the_adjoint_is_the_derivative_of_the_measures():
    rng = np.random.default_rng(6)
    n = 300
    pos = rng.uniform(size=(n, 2))
    w = rng.uniform(0, 1e-3, size=n)
    g = rng.standard_normal(n)
    pd = _pd(pos, w)
    gp, gw = pd.measures_vjp(g)
    h = 1e-7
    for i in range(0, n, 37):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (g @ _pd(pos, wp).measures - g @ _pd(pos, wm).measures) / (2 * h)
        assert abs(fd - gw[i]) < 1e-5 * max(1, abs(fd))
        for a in range(2):
            pp, pm = pos.copy(), pos.copy()
            pp[i, a] += h
            pm[i, a] -= h
            fd = (g @ _pd(pp, w).measures - g @ _pd(pm, w).measures) / (2 * h)
            assert abs(fd - gp[i, a]) < 1e-5 * max(1, abs(fd))


@pytest.mark.parametrize("d", [2, 3])
def test_the_adjoint_of_the_first_moments_is_their_derivative(d):
    """PowerDiagram.py:341-353 (`moment(k)`, k < d, differentiable like the measures): `sdot_cells_vjp_moments` for the
    cotangents of the masses and of the first moments int_cell x rho, against central differences of the GPU cells at
    fixed weights, in the weights and the positions (1e-5 of the largest derivative)"""
    rng = np.random.default_rng(10 + d)
    n = 300
    pos = rng.uniform(size=(n, d))
    w = rng.uniform(0, 1e-3, size=n)
    g = rng.standard_normal(n)
    G = rng.standard_normal((n, d))

    def f(p, ww):
        m, first, _ = _pd(p, ww).moments
        return g @ m + (G * first).sum()
    gp, gw = _pd(pos, w).moments_vjp(g, G)
    gp0, gw0 = _pd(pos, w).moments_vjp(None, G)
    gp1, gw1 = _pd(pos, w).measures_vjp(g)
    assert np.abs(gp0 + gp1 - gp).max() < 1e-12 * np.abs(gp).max() and np.abs(gw0 + gw1 - gw).max() < 1e-12 * np.abs(gw).max()
    assert abs(gw.sum()) < 1e-10 * np.abs(gw).max()          # a constant added to every weight moves no facet
    h = 1e-6
    scale = max(np.abs(gp).max(), np.abs(gw).max())
    for i in range(0, n, 29):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (f(pos, wp) - f(pos, wm)) / (2 * h)
        assert abs(fd - gw[i]) < 1e-5 * scale, (i, fd, gw[i])
        for a in range(d):
            pp, pm = pos.copy(), pos.copy()
            pp[i, a] += h
            pm[i, a] -= h
            fd = (f(pp, w) - f(pm, w)) / (2 * h)
            assert abs(fd - gp[i, a]) < 1e-5 * scale, (i, a, fd, gp[i, a])


@pytest.mark.parametrize("d", [2, 3])
def test_the_search_counters_leave_the_cells_unchanged(d):
    """the gather model's device counters (sdot_context_set_counters): the counting instantiation of the cell kernel gives
    the same cells bit for bit, its counts repeat exactly, every neighbour's seed is among the candidates read, the
    spread weights send the search through the pyramid, and nothing is counted once the counters are off"""
    from sdot import _lib
    rng = np.random.default_rng(30 + d)
    n = 20000
    pos = rng.uniform(size=(n, d))
    w = rng.uniform(0, 1e-3 if d == 2 else 3e-2, n)
    pd = _pd(pos, w)
    m0 = pd.measures
    nb = pd.hessian_rows()[0]
    _lib.gather_counters(d, reset=True)
    _lib.set_counters(True)
    try:
        m1 = pd.measures
        c1 = _lib.gather_counters(d, reset=True)
        m2 = pd.measures
        c2 = _lib.gather_counters(d, reset=True)
    finally:
        _lib.set_counters(False)
    assert np.array_equal(m0, m1) and np.array_equal(m1, m2)
    assert c1 == c2, (c1, c2)
    assert c1["cells"] == n
    assert c1["candidates"] >= nb.sum(), (c1, nb.sum())
    assert c1["grid_ranges"] > 0 and c1["grid_cells"] > 0 and c1["nodes"] > 0, c1
    print(f"\n{d}D n={n}: per cell " + ", ".join(f"{k} {v / n:.1f}" for k, v in c1.items() if k != "cells"))
    pd.measures
    assert _lib.gather_counters(d)["candidates"] == 0


def test_the_3d_adjoint_is_the_derivative_of_the_measures():
    """gpu/Cell3D.cuh:1954-1978: the adjoint of the 3D masses (constant density) against central differences"""
    rng = np.random.default_rng(7)
    n = 400
    pos = rng.uniform(size=(n, 3))
    w = rng.uniform(0, 1e-3, size=n)
    g = rng.standard_normal(n)
    pd = _pd(pos, w)
    gp, gw = pd.measures_vjp(g)
    assert gp.shape == (n, 3) and gw.shape == (n,)
    h = 1e-6
    for i in range(0, n, 41):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (g @ _pd(pos, wp).measures - g @ _pd(pos, wm).measures) / (2 * h)
        assert abs(fd - gw[i]) < 1e-5 * max(1, abs(fd)), (i, fd, gw[i])
        for a in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[i, a] += h
            pm[i, a] -= h
            fd = (g @ _pd(pp, w).measures - g @ _pd(pm, w).measures) / (2 * h)
            assert abs(fd - gp[i, a]) < 1e-5 * max(1, abs(fd)), (i, a, fd, gp[i, a])
    # the weights' part is the Laplacian's action: grad_w = L g (rows of c_ij)
    row, cols, vals, dia = pd.laplacian()
    Lg = dia * g - np.array([vals[row[i]:row[i + 1]] @ g[cols[row[i]:row[i + 1]]] for i in range(n)])
    assert np.abs(gw - Lg).max() < 1e-9 * np.abs(Lg).max()


def test_a_seed_with_hundreds_of_neighbours_is_solved():
    """tests/test_SdotPlanNd.py:1280-1300: a ring of 600 seeds around one seed -- its cell has 600 vertices, far past
    the 32 a warp holds in registers: the global-memory pass rebuilds it, and the facet table grows to hold its row"""
    k = 600
    ang = 2 * np.pi * np.arange(k) / k
    pos = np.r_[[[0.5, 0.5]], np.c_[0.5 + 0.3 * np.cos(ang), 0.5 + 0.3 * np.sin(ang)]]
    pd = _pd(pos)
    m = pd.measures
    ref = O.cells(pos)
    assert np.abs(m - ref["mass"]).max() <= 1e-10 * ref["mass"].max()
    nb, ids, coef = pd.hessian_rows()
    assert nb[0] == k
    assert set(ids[0, :k].tolist()) == set(range(1, k + 1))
    row, cols, vals, dia = pd.laplacian()
    assert row[1] - row[0] == k


def test_a_cell_past_every_capacity_is_a_kernel_failure():
    """a ring of 5000 seeds: the centre cell needs 5000 vertices, past the 4096 of the global-memory pass"""
    k = 5000
    ang = 2 * np.pi * np.arange(k) / k
    pos = np.r_[[[0.5, 0.5]], np.c_[0.5 + 0.3 * np.cos(ang), 0.5 + 0.3 * np.sin(ang)]]
    with pytest.raises(sdot.KernelFailure) as e:
        _pd(pos).measures
    assert e.value.seed == 0


def test_big_cells_in_a_solve():
    """a gaussian far from most seeds: low-density cells grow huge during the continuation"""
    rng = np.random.default_rng(44)
    g = sdot.SumOfGaussians([[0.25, 0.3]], [0.05], support_box=(np.zeros(2), np.ones(2)))
    pos = rng.uniform(size=(3000, 2))
    plan = sdot.OtProblem(sdot.SumOfDiracs(pos), g).solve(sdot.Iterative(tol=0.0, tuning=sdot.Tuning(mass_rtol=1e-8)))
    assert plan.converged
    assert np.abs(plan.cell_masses / plan.target_masses - 1).max() <= 1e-8
