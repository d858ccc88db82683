"""The host side of the drop-in API, without a GPU: domains, normalisation, settings and refusals."""
import numpy as np
import pytest

import sdot
from sdot import Box, Image, Iterative, OtProblem, SumOfDiracs, SumOfGaussians, Tuning, box_half_spaces
from sdot.PowerDiagram import _domain_box, axis_aligned_box
from sdot.SdotPlanNd import exact_duplicates, solver_options


def test_box_half_spaces_round_trip():
    d, o = box_half_spaces([0, -1], [2, 3])
    mi, ma, kept = axis_aligned_box(d, o)
    assert np.allclose(mi, [0, -1]) and np.allclose(ma, [2, 3]) and not kept.any()
    assert np.allclose(_domain_box((d, o), 2)[0], [0, -1])


def test_a_polytope_domain_is_refused():
    d, o = box_half_spaces([0, 0], [1, 1])
    d = np.vstack([d, [[1, 1]]])
    o = np.concatenate([o, [1.5]])
    with pytest.raises(NotImplementedError):
        _domain_box((d, o), 2)
    # a plane that does not cut the box is harmless
    o[-1] = 2.5
    assert np.allclose(_domain_box((d, o), 2)[1], [1, 1])


def test_distributions_normalise_like_the_reference():
    s = SumOfDiracs(np.zeros((4, 2))).normalized_version()
    assert np.allclose(s.weights, 0.25)
    s = SumOfDiracs(np.zeros((2, 2)), [1, 3]).normalized_version()
    assert np.allclose(s.weights, [0.25, 0.75])
    im = Image(np.ones((4, 2)), frame=[0.5, 1.0]).normalized_version()
    assert abs(im.mass - 1) < 1e-15
    assert np.allclose(im.box()[1], [2.0, 2.0])
    g = SumOfGaussians([[0.5, 0.5], [0.2, 0.3]], [0.1, 0.05], [2, 6]).normalized_version()
    assert np.allclose(g.weights, [0.25, 0.75])
    lo, hi = g.box()
    assert np.allclose(lo, [-0.1, -0.1]) and np.allclose(hi, [1.1, 1.1])
    b = Box().normalized_version(nb_dims=3)
    assert b._sdot_density() == ("uniform", 1.0)


def test_settings_map_onto_the_option_vector():
    o = solver_options(Iterative(tol=0, tuning=Tuning(mass_rtol=1e-8, residual="lin")), 10)
    assert o["tol_abs"] == 0 and o["tol_rel"] == 1e-8 and o["residual"] == 0 and o["continuation"] == 1
    assert o["lin_method"] == 1 and solver_options(Iterative(tuning=Tuning(linear_solver="cg")), 10)["lin_method"] == 0
    assert solver_options(Iterative(tuning=Tuning(step="limits")), 10)["step"] == 1
    assert solver_options(Iterative(tuning=Tuning(step="trials")), 10)["step"] == 0
    assert solver_options(Iterative(tuning=Tuning(step="limits")), 10, 2)["step"] == 1
    assert solver_options(Iterative(), 10, 2)["step"] == 1          # "auto": the limits in 2D (SdotPlanNd.py:462)
    with pytest.raises(ValueError):                    # SdotPlanNd.py:461-465: the limits step is 2D only
        solver_options(Iterative(tuning=Tuning(step="limits")), 10, 3)
    assert solver_options(Iterative(), 10, 3)["step"] == 0
    with pytest.raises(ValueError):
        solver_options(Iterative(tuning=Tuning(step="bisection")), 10)
    assert solver_options(Iterative(precision="mixed"), 10, 2)["precision"] == 1     # the FP32 clip (2D)
    with pytest.raises(NotImplementedError):
        solver_options(Iterative(precision="mixed"), 10, 3)
    with pytest.raises(ValueError):
        Iterative(precision="fp16")
    with pytest.raises(ValueError):
        Iterative(ot_plan=object(), weights0=np.zeros(3))


def test_the_problem_refuses_what_it_does_not_solve():
    pb = OtProblem(SumOfDiracs(np.zeros((3, 1))), Image(np.ones(4)))
    with pytest.raises(NotImplementedError):
        pb.solve()
    with pytest.raises(TypeError):
        OtProblem(Image(np.ones((2, 2))), Image(np.ones((2, 2))))


def test_exact_duplicates():
    p = np.array([[0, 0], [1, 1], [0, 0], [2, 2], [1, 1.0]])
    dup, rep = exact_duplicates(p)
    assert list(dup) == [2, 4] and list(rep) == [0, 1]
    assert len(exact_duplicates(np.random.default_rng(0).uniform(size=(100, 2)))[0]) == 0


def test_public_names():
    for name in ("PowerDiagram", "Voronoi", "OtProblem", "Iterative", "Tuning", "OtNotConverged", "ot_solve", "SdotPlanNd", "SumOfDiracs",
                 "Image", "SumOfGaussians", "Box", "box_half_spaces", "KernelFailure"):
        assert hasattr(sdot, name)


def test_quantization_draws_its_start_in_the_support():
    """quantization.py:113-130: rejection in the bounding box of the support's polytope"""
    import sdot
    from sdot.quantization import uniform_in_support
    img = sdot.Image(np.ones((4, 3)), frame=[0.5, 0.25])
    x = uniform_in_support(img, 300, seed=3)
    assert x.shape == (300, 2) and (x >= 0).all() and (x[:, 0] <= 2).all() and (x[:, 1] <= 0.75).all()
    assert np.array_equal(x, uniform_in_support(img, 300, seed=3))
    assert x[:, 0].max() > 1.9 and x[:, 1].max() > 0.7


def test_exact_duplicates_are_written_back_with_empty_cells():
    """SdotPlanNd.py:124-148, sdotplan/Aggregation.h:24-31: the solve runs without the duplicates; each gets an empty cell,
    its representative's weight minus k gaps (k its rank among the representative's duplicates), its cluster the
    representative's; the other outputs are the solve's, in the caller's order"""
    from sdot.SdotPlanNd import SdotPlanNd
    pos = np.array([[0.1, 0.2], [0.5, 0.5], [0.1, 0.2], [0.9, 0.3], [0.1, 0.2]])
    dup, rep = exact_duplicates(pos)
    assert list(dup) == [2, 4] and list(rep) == [0, 0]
    plan = SdotPlanNd.__new__(SdotPlanNd)
    plan.problem = OtProblem(SumOfDiracs(pos), Box(nb_dims=2))
    plan._dups = (dup, rep)
    plan._keep = np.array([0, 1, 3])
    r = dict(weights=np.array([0.0, 0.25, -0.125]), masses=np.array([0.6, 0.2, 0.2]),
             barycentres=np.array([[0.2, 0.2], [0.5, 0.6], [0.8, 0.3]]), clusters=np.array([0, 1, 2]))
    out = plan._expand(r)
    w, m, b, cl = out["weights"], out["masses"], out["barycentres"], out["clusters"]
    assert np.array_equal(m, [0.6, 0.2, 0.0, 0.2, 0.0])
    assert np.array_equal(cl, [0, 1, 0, 3, 0])
    assert w[0] == 0 and w[1] == 0.25 and w[3] == -0.125
    assert w[4] < w[2] < w[0] and np.isclose(w[0] - w[2], w[2] - w[4])
    assert np.array_equal(b[[0, 1, 3]], r["barycentres"]) and np.array_equal(b[2], pos[2]) and np.array_equal(b[4], pos[4])


@pytest.mark.parametrize("d", [2, 3])
def test_the_weights_derivative_is_the_derivative_of_the_solve(d):
    """SdotPlanNd.py:1018-1050, tests/test_SdotPlanNd.py:2068-2104: the implicit-function derivative of the fitted
    weights (`torch_ops.weights_vjp`, the backward of `weights_batch`), driven here by the oracle's diagram, a dense
    solve and a finite-difference adjoint of the masses, against central differences of the whole oracle solve in the
    positions and in the target masses (1e-7 of the largest component)"""
    import oracle as O
    from sdot.torch_ops import weights_vjp
    rng = np.random.default_rng(d)
    n = 16 if d == 2 else 10
    pos = rng.uniform(0.2, 0.8, size=(n, d))
    nu = rng.uniform(0.5, 1.5, n)

    def solve(p, q):
        s = O.solve(p, nu=q / q.sum(), tol_abs=1e-15, maxit=100)
        assert s["stats"]["status"] == 1
        return s["weights"]

    def laplacian(p, w):
        r = O.cells(p, w)
        row, cols, vals = [0], [], []
        for i in range(n):
            k = r["nb"][i]
            cols += list(r["nid"][i, :k])
            vals += list(r["nc"][i, :k])
            row.append(row[-1] + k)
        return np.array(row), np.array(cols), np.array(vals), np.array([r["nc"][i, : r["nb"][i]].sum() for i in range(n)])

    def dense_solve(row, cols, vals, dia, rhs):
        L = np.diag(dia)
        for i in range(n):
            L[i, cols[row[i]:row[i + 1]]] -= vals[row[i]:row[i + 1]]
        return np.linalg.lstsq(0.5 * (L + L.T), rhs, rcond=None)[0]

    def masses_vjp(p, w, lam, h=1e-7):
        out = np.zeros_like(p)
        for k in range(n):
            for a in range(d):
                pp, pm = p.copy(), p.copy()
                pp[k, a] += h
                pm[k, a] -= h
                out[k, a] = lam @ (O.cells(pp, w)["mass"] - O.cells(pm, w)["mass"]) / (2 * h)
        return out

    w = solve(pos, nu)
    g = rng.standard_normal(n)
    gp, gn = weights_vjp(pos, w, nu, g, laplacian, dense_solve, masses_vjp, 1.0)
    h = 1e-6
    fp = np.zeros_like(pos)
    for k in range(n):
        for a in range(d):
            pp, pm = pos.copy(), pos.copy()
            pp[k, a] += h
            pm[k, a] -= h
            fp[k, a] = g @ (solve(pp, nu) - solve(pm, nu)) / (2 * h)
    fn = np.array([g @ (solve(pos, nu + h * e) - solve(pos, nu - h * e)) / (2 * h) for e in np.eye(n)])
    assert np.abs(gp - fp).max() < 1e-7 * np.abs(fp).max()
    assert np.abs(gn - fn).max() < 1e-7 * np.abs(fn).max()


@pytest.mark.parametrize("d", [2, 3])
def test_the_barycentres_derivative_is_the_derivative_of_the_solve(d):
    """SdotPlanNd.py:1051-1070: the barycentres' derivative (`torch_ops.barycentres_vjp`, the backward of
    `barycentres_batch`: the adjoint of the masses and first moments at fixed weights, then the weights' implicit
    derivative), driven by the oracle's diagram and finite-difference adjoints, against central differences of the whole
    oracle solve's barycentres in the positions and the target masses (1e-6 of the largest component)"""
    import oracle as O
    from sdot.torch_ops import barycentres_vjp
    rng = np.random.default_rng(20 + d)
    n = 12 if d == 2 else 8
    pos = rng.uniform(0.2, 0.8, size=(n, d))
    nu = rng.uniform(0.5, 1.5, n)

    def solve(p, q):
        s = O.solve(p, nu=q / q.sum(), tol_abs=1e-15, maxit=100)
        assert s["stats"]["status"] == 1
        return s

    def laplacian(p, w):
        r = O.cells(p, w)
        row, cols, vals = [0], [], []
        for i in range(n):
            k = r["nb"][i]
            cols += list(r["nid"][i, :k])
            vals += list(r["nc"][i, :k])
            row.append(row[-1] + k)
        return np.array(row), np.array(cols), np.array(vals), np.array([r["nc"][i, : r["nb"][i]].sum() for i in range(n)])

    def dense_solve(row, cols, vals, dia, rhs):
        L = np.diag(dia)
        for i in range(n):
            L[i, cols[row[i]:row[i + 1]]] -= vals[row[i]:row[i + 1]]
        return np.linalg.lstsq(0.5 * (L + L.T), rhs, rcond=None)[0]

    def fd_adjoint(p, w, f, h=1e-7):
        """(grad_p, grad_w) of the scalar f(cells at p, w) by central differences"""
        gp, gw = np.zeros_like(p), np.zeros(n)
        for k in range(n):
            wp, wm = w.copy(), w.copy()
            wp[k] += h
            wm[k] -= h
            gw[k] = (f(O.cells(p, wp)) - f(O.cells(p, wm))) / (2 * h)
            for a in range(d):
                pp, pm = p.copy(), p.copy()
                pp[k, a] += h
                pm[k, a] -= h
                gp[k, a] = (f(O.cells(pp, w)) - f(O.cells(pm, w))) / (2 * h)
        return gp, gw

    def moments_vjp(p, w, gm, gF):
        return fd_adjoint(p, w, lambda r: gm @ r["mass"] + (gF * r["mass"][:, None] * r["bary"]).sum())

    def masses_vjp(p, w, lam):
        return fd_adjoint(p, w, lambda r: lam @ r["mass"])[0]

    s = solve(pos, nu)
    g = rng.standard_normal((n, d))
    gp, gn = barycentres_vjp(pos, s["weights"], nu, s["masses"], s["bary"], g, moments_vjp, laplacian, dense_solve, masses_vjp,
                             float(s["masses"].sum()))
    h = 1e-6
    fp = np.zeros_like(pos)
    for k in range(n):
        for a in range(d):
            pp, pm = pos.copy(), pos.copy()
            pp[k, a] += h
            pm[k, a] -= h
            fp[k, a] = ((solve(pp, nu)["bary"] - solve(pm, nu)["bary"]) * g).sum() / (2 * h)
    fn = np.array([((solve(pos, nu + h * e)["bary"] - solve(pos, nu - h * e)["bary"]) * g).sum() / (2 * h) for e in np.eye(n)])
    assert np.abs(gp - fp).max() < 1e-6 * np.abs(fp).max(), np.abs(gp - fp).max()
    assert np.abs(gn - fn).max() < 1e-6 * np.abs(fn).max(), np.abs(gn - fn).max()


def test_the_domain_comes_from_the_density_alone():
    """tests/test_SdotPlanNd.py:409-438 (its host part): the domain of a gaussian target is the support it declares,
    `centres +- 6 sigma`, not the envelope of the diracs; a target that declares no support is refused"""
    from sdot.SdotPlanNd import _box_of
    pos = np.random.default_rng(3).uniform(0.4, 0.6, size=(60, 2))
    g = SumOfGaussians(np.array([[0.5, 0.5]]), np.array([0.15]), weights=np.array([1.0]))
    lo, hi = _box_of(OtProblem(SumOfDiracs(pos), g))
    assert np.allclose(lo, [0.5 - 0.9] * 2) and np.allclose(hi, [0.5 + 0.9] * 2)
    with pytest.raises(ValueError):
        OtProblem(SumOfDiracs(pos), SumOfGaussians(np.array([[0.5, 0.5]]), np.array([0.15]), support_sigmas=None)).solve()
