"""Parity of the GPU damped Newton (sdot_solve / sdot_solve_batch through the C ABI) with the oracle's.

The bar (the reference's card-vs-CPU tests tests/test_SdotPlanNd.py:612-656, 966-1072, tightened):
the solve converges to `max |m - nu| / nu <= 1e-8`; an independent oracle diagram at the GPU's weights
confirms the masses; the weights agree with the oracle's converged weights within 1e-7 of max|w|; masses,
barycentres and cost agree; a solve in a batch is bitwise the solve alone.
"""
import numpy as np
import pytest

import oracle as O
import sdot
from sdot import Iterative, OtProblem, SumOfDiracs, Tuning
from sdot.SdotPlanNd import SdotPlanNd

pytestmark = pytest.mark.gpu


def _solve(pos, target=None, rtol=1e-8, **kw):
    target = target or sdot.Box()
    return OtProblem(SumOfDiracs(pos), target).solve(Iterative(tol=0.0, tuning=Tuning(mass_rtol=rtol), **kw))


def test_plain_2d_fp64_n10000_matches_the_oracle():
    """config: N = 10,000 uniform in [0,1]^2, uniform density, nu = 1/N, w0 = 0, FP64, max rel mass error <= 1e-8"""
    n = 10000
    rng = np.random.default_rng(20260101)
    pos = rng.uniform(size=(n, 2))
    plan = _solve(pos, rtol=1e-10)
    assert plan.converged, plan.stats
    nu = 1.0 / n
    assert np.abs(plan.cell_masses - nu).max() / nu <= 1e-10
    assert plan.weights[0] == 0
    # independent check: the oracle's diagram at the GPU's weights
    chk = O.cells(pos, plan.weights)["mass"]
    assert np.abs(chk - nu).max() / nu <= 1e-8
    ref = O.solve(pos, tol_abs=0.0, tol_rel=1e-10)
    assert ref["stats"]["status"] == 1
    assert np.abs(plan.weights - ref["weights"]).max() <= 1e-7 * np.abs(ref["weights"]).max()
    assert np.abs(plan.barycenters - ref["bary"]).max() < 1e-9
    assert abs(plan.cost - ref["cost"]) <= 1e-9 * ref["cost"]
    assert plan.stats["start"] == "voronoi"
    assert len(plan.history) >= plan.stats["nb_iter"] + 1


@pytest.mark.parametrize("target", ["uniform", "gaussians"])
def test_the_fp32_clip_solve_reaches_the_fp64_plan(target):
    """precision "mixed" (the clip in FP32 with FP64 re-checks, every vertex re-solved in FP64): the 2D Newton converges to
    max |m - nu| / nu <= 1e-8 as the FP64 one; the oracle's diagram at its weights confirms it; its weights agree with
    the FP64 solve's within 1e-9 of max|w|"""
    n = 10000
    rng = np.random.default_rng(20260303)
    pos = rng.uniform(size=(n, 2))
    dst = None
    od = None
    if target == "gaussians":
        c, s = rng.uniform(0.3, 0.7, size=(4, 2)), rng.uniform(0.05, 0.15, size=4)
        dst = sdot.SumOfGaussians(c, s, support_box=(np.zeros(2), np.ones(2)))
        od = ("gauss", c, s, dst.normalized_version().weights)
    a = _solve(pos, dst)
    b = _solve(pos, dst, precision="mixed")
    assert a.converged and b.converged, (a.stats["status"], b.stats["status"])
    nu = np.asarray(b.target_masses).reshape(-1)
    assert np.abs(b.cell_masses / nu - 1).max() <= 1e-8
    chk = O.cells(pos, b.weights, density=od)["mass"]
    assert np.abs(chk / nu - 1).max() <= 1e-8 * (1 + 1e-6)
    assert np.abs(a.weights - b.weights).max() <= 1e-9 * np.abs(a.weights).max()


@pytest.mark.parametrize("lin", ["cg", "mg"])
@pytest.mark.parametrize("lp", ["fp64", "mixed"])
def test_both_linear_solvers_reach_the_same_plan(lin, lp):
    """tests/test_SdotPlanNd.py:536-561: the multigrid reaches the plan of the reference solver; so does each of them with
    its CG in FP32 inside an FP64 iterative refinement (`linear_precision = "mixed"`)"""
    rng = np.random.default_rng(50)
    n = 20000
    pos = rng.uniform(size=(n, 2))
    plan = OtProblem(SumOfDiracs(pos), sdot.Box()).solve(
        Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-10, linear_solver=lin, linear_precision=lp)))
    assert plan.converged
    ref = O.solve(pos, tol_abs=0.0, tol_rel=1e-10)
    assert np.abs(plan.weights - ref["weights"]).max() <= 1e-7 * np.abs(ref["weights"]).max()


@pytest.mark.parametrize("d,gauss", [(2, True), (3, False), (3, True)])
def test_the_mixed_cg_reaches_the_fp64_plan(d, gauss):
    """`linear_precision = "mixed"` (the Newton systems' CG in FP32, refined in FP64) against the FP64 CG: both converge
    to max |m - nu| / nu <= 1e-8, to the same weights within 1e-7 of max |w|, and the oracle's diagram at the mixed
    solve's weights confirms its masses (a constant density: the oracle's 3D gaussian quadrature is too slow here)"""
    rng = np.random.default_rng(60 + d)
    n = 6000 if d == 2 else 3000
    pos = rng.uniform(size=(n, d))
    target = sdot.Box(nb_dims=d)
    if gauss:
        c = rng.uniform(0.3, 0.7, size=(3, d))
        target = sdot.SumOfGaussians(c, np.array([0.1, 0.15, 0.12]), np.full(3, 1 / 3), support_box=(np.zeros(d), np.ones(d)))
    plans = {lp: OtProblem(SumOfDiracs(pos), target).solve(Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-8, linear_precision=lp)))
             for lp in ("fp64", "mixed")}
    for lp, plan in plans.items():
        assert plan.converged, (lp, plan.stats["status"])
        nu = np.asarray(plan.target_masses).reshape(-1)
        assert np.abs(plan.cell_masses / nu - 1).max() <= 1e-8, lp
    w64, wmx = plans["fp64"].weights, plans["mixed"].weights
    assert np.abs(wmx - w64).max() <= 1e-7 * np.abs(w64).max()
    if not gauss:
        chk = O.cells(pos, wmx)["mass"]
        assert np.abs(chk * n - 1).max() <= 1e-8


def test_a_solve_in_a_batch_is_the_solve_alone():
    rng = np.random.default_rng(3)
    pbs = [OtProblem(SumOfDiracs(rng.uniform(size=(n, 2))), sdot.Box()) for n in (1500, 4000, 700, 2500)]
    s = Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-9))
    batch = SdotPlanNd._solve_many(pbs, s)
    for pb, b in zip(pbs, batch):
        a = SdotPlanNd._solve(pb, s)
        assert np.array_equal(a.weights, b.weights)
        assert np.array_equal(a.cell_masses, b.cell_masses)
        assert a.stats["nb_diag"] == b.stats["nb_diag"]


def test_the_multigrid_cuts_the_cg_iterations():
    """2D uniform, N = 100,000: the Newton solves' CG iterations per Newton step with the aggregation multigrid stay
    a small fraction of the Jacobi-preconditioned ones (both reach the same plan)"""
    rng = np.random.default_rng(41)
    pos = rng.uniform(size=(100000, 2))
    per = {}
    for lin in ("cg", "mg"):
        plan = OtProblem(SumOfDiracs(pos), sdot.Box()).solve(Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-8, linear_solver=lin)))
        assert plan.converged
        per[lin] = plan.stats["lin_nb_iter"] / max(1, plan.stats["nb_iter"])
    assert per["mg"] < 0.2 * per["cg"], per


def test_a_cell_past_every_capacity_fails_its_solve_only():
    """a ring of 5000 seeds around one (its cell has 5000 vertices, past the 4096 of the global-memory pass) in the
    same batch as two ordinary problems: it ends with status 5 ("card capacity", SdotPlanNd.py:106-107), and the
    others are the solves alone, bit for bit"""
    k = 5000
    ang = 2 * np.pi * np.arange(k) / k
    ring = np.r_[[[0.5, 0.5]], np.c_[0.5 + 0.3 * np.cos(ang), 0.5 + 0.3 * np.sin(ang)]]
    rng = np.random.default_rng(12)
    others = [rng.uniform(size=(n, 2)) for n in (2000, 900)]
    s = Iterative(tol=0.0, on_failure="ignore", tuning=Tuning(mass_rtol=1e-9))
    pbs = [OtProblem(SumOfDiracs(p), sdot.Box()) for p in (others[0], ring, others[1])]
    batch = SdotPlanNd._solve_many(pbs, s)
    assert batch[1].stats["status"] == "card capacity" and not batch[1].converged
    for i in (0, 2):
        alone = SdotPlanNd._solve(pbs[i], s)
        assert batch[i].converged
        assert np.array_equal(alone.weights, batch[i].weights)


def test_an_image_target_matches_the_oracle():
    rng = np.random.default_rng(31)
    xs = (np.arange(128) + 0.5) / 128
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    vals = 0.2 + np.exp(-((X - 0.3) ** 2 + (Y - 0.6) ** 2) / 0.02) + 0.5 * np.exp(-((X - 0.7) ** 2 + (Y - 0.3) ** 2) / 0.01)
    img = sdot.Image(vals, frame=[1 / 128, 1 / 128])
    n = 3000
    pos = rng.uniform(size=(n, 2))
    plan = _solve(pos, img, rtol=1e-10)
    assert plan.converged
    norm = img.normalized_version()
    ref = O.solve(pos, tol_abs=0.0, tol_rel=1e-10, density=("image", [0, 0], [1 / 128, 1 / 128], norm.values))
    assert ref["stats"]["status"] == 1
    assert np.abs(plan.weights - ref["weights"]).max() <= 1e-7 * np.abs(ref["weights"]).max()
    assert abs(plan.cost - ref["cost"]) <= 1e-9 * ref["cost"]
    assert np.abs(plan.barycenters - ref["bary"]).max() < 1e-8


def test_gaussians_with_the_continuation_match_the_oracle():
    rng = np.random.default_rng(33)
    c = rng.uniform(0.2, 0.8, size=(4, 2))
    s = rng.uniform(0.05, 0.15, size=4)
    g = sdot.SumOfGaussians(c, s, support_box=(np.zeros(2), np.ones(2)))
    n = 800
    pos = rng.uniform(size=(n, 2))
    plan = _solve(pos, g, rtol=1e-9)
    assert plan.converged
    ng = g.normalized_version()
    ref = O.solve(pos, tol_abs=0.0, tol_rel=1e-9, density=("gauss", c, s, ng.weights))
    assert ref["stats"]["status"] == 1
    assert plan.stats["nb_continuation_steps"] == ref["stats"]["nb_continuation_steps"]
    assert abs(plan.stats["domain_mass"] - ref["stats"]["domain_mass"]) < 1e-10
    assert np.abs(plan.weights - ref["weights"]).max() <= 1e-6 * np.abs(ref["weights"]).max()
    assert abs(plan.cost - ref["cost"]) <= 1e-8 * ref["cost"]


def test_a_3d_gaussian_target_is_solved():
    """3D, 4 gaussians (the continuation runs): the plan reaches 1e-8, and the oracle's cells at the plan's weights
    give the same masses (1e-9 relative) and barycentres"""
    rng = np.random.default_rng(34)
    c = rng.uniform(0.2, 0.8, size=(4, 3))
    s = rng.uniform(0.05, 0.15, size=4)
    g = sdot.SumOfGaussians(c, s, support_box=(np.zeros(3), np.ones(3)))
    n = 1200
    pos = rng.uniform(size=(n, 3))
    plan = _solve(pos, g, rtol=1e-8)
    assert plan.converged
    assert np.abs(plan.cell_masses / plan.target_masses - 1).max() <= 1e-8
    ng = g.normalized_version()
    ref = O.cells(pos, plan.weights, box=(np.zeros(3), np.ones(3)), density=("gauss", c, s, ng.weights))
    assert ref["status"] == 0
    assert np.abs(ref["mass"] / plan.cell_masses - 1).max() <= 1e-9
    assert np.abs(ref["bary"] - plan.barycenters).max() <= 1e-9


def test_the_similarity_start():
    rng = np.random.default_rng(9)
    pos = rng.uniform(0.5, 1.5, size=(500, 2))
    plan = _solve(pos, rtol=1e-9)
    assert plan.stats["start"] == "similarity"
    assert plan.converged


def test_a_solve_that_misses_its_tolerance_raises():
    rng = np.random.default_rng(10)
    pos = rng.uniform(size=(1000, 2))
    with pytest.raises(sdot.OtNotConverged) as e:
        OtProblem(SumOfDiracs(pos), sdot.Box()).solve(Iterative(tol=1e-14, max_iter=1))
    assert e.value.solution.stats["status"] == "max iterations"


def test_the_warm_start_is_the_last_plan():
    rng = np.random.default_rng(12)
    pos = rng.uniform(size=(2000, 2))
    pb = OtProblem(SumOfDiracs(pos), sdot.Box())
    a = pb.solve(Iterative(tol=1e-12))
    pb.source = SumOfDiracs(pos + 1e-4 * rng.standard_normal(pos.shape))
    b = pb.solve(Iterative(tol=1e-12))
    assert b.stats["warm_start"] == "ot_plan"
    assert b.stats["nb_iter"] <= a.stats["nb_iter"]


def test_the_envelope_gradient_by_finite_differences():
    """tests/test_SdotPlanNd.py:500-534: d cost / d p = 2 m (p - b), central differences h = 1e-4"""
    rng = np.random.default_rng(13)
    n = 200
    pos = rng.uniform(0.1, 0.9, size=(n, 2))
    plan = _solve(pos, rtol=1e-12)
    _, grad = plan.cost_and_position_grad()
    h = 1e-4
    for i in range(0, n, 41):
        for a in range(2):
            pp, pm = pos.copy(), pos.copy()
            pp[i, a] += h
            pm[i, a] -= h
            fd = (_solve(pp, rtol=1e-12).cost - _solve(pm, rtol=1e-12).cost) / (2 * h)
            assert abs(fd - grad[i, a]) < 1e-4 * max(1, abs(fd))


def test_a_3d_solve_matches_the_oracle():
    """tests/test_SdotPlanNd.py:308-325 and 1621-1660: 3D uniform, the card against the CPU"""
    rng = np.random.default_rng(41)
    n = 3000
    pos = rng.uniform(size=(n, 3))
    plan = _solve(pos, rtol=1e-10)
    assert plan.converged
    assert np.abs(plan.cell_masses * n - 1).max() <= 1e-10
    ref = O.solve(pos, tol_abs=0.0, tol_rel=1e-10)
    assert ref["stats"]["status"] == 1
    assert np.abs(plan.weights - ref["weights"]).max() <= 1e-7 * np.abs(ref["weights"]).max()
    assert np.abs(plan.barycenters - ref["bary"]).max() < 1e-9
    assert abs(plan.cost - ref["cost"]) <= 1e-9 * ref["cost"]


def _check_aggregated(name, plan, pos, groups, tol):
    """tests/test_SdotPlanNd.py:1407-1432: converged (aggregated, unless the groups are exact duplicates only), the clusters
    found, each cluster's mass its target, every other cell its own, an exact duplicate's cell empty"""
    n = len(pos)
    st = plan.stats
    nu = np.asarray(plan.target_masses).reshape(-1)
    m = np.asarray(plan.cell_masses).reshape(-1)
    w = np.asarray(plan.weights).reshape(-1)
    assert plan.converged, (name, st["status"], st["residual"])
    only_exact = all(exact for _, exact in groups)
    assert st["status"] == ("converged" if only_exact else "converged (aggregated)"), (name, st["status"])
    assert st["residual"] <= tol, (name, st["residual"])
    cl = np.asarray(plan.clusters).reshape(-1)
    alone = np.ones(n, dtype=bool)
    for members, exact in groups:
        assert (cl[members] == min(members)).all(), (name, members, cl[members])
        alone[members] = False
        assert abs(m[members].sum() - nu[members].sum()) <= len(members) * tol * (1 + 1e-9), (name, m[members].sum() - nu[members].sum())
        if exact:
            assert (m[members[1:]] == 0).all() and (w[members[1:]] < w[members[0]]).all(), name
    assert (cl[alone] == np.arange(n)[alone]).all(), name
    assert np.abs(m[alone] - nu[alone]).max() <= tol, (name, np.abs(m[alone] - nu[alone]).max())
    assert st["nb_clusters"] == len(groups) and st["nb_aggregated"] == sum(len(g) for g, _ in groups), (name, st["aggregation"])


# the clouds of the aggregation tests (the 2D pair 1e-12 apart puts c_ij ~ 1e10 next to couplings ~ 1 in the first Newton
# system; in 3D the triple 1e-10 apart makes three near-coincident bisector planes)
_CLOUDS = [(d, name) for d in (2, 3) for name in ("exact pair", "exact triple", "pair at 1e-9", "pair at 1e-12", "triple at 1e-10",
                                                   "pair and duplicate")]


@pytest.mark.parametrize("d,name", _CLOUDS)
def test_the_card_aggregates_as_the_cpu(d, name):
    """tests/test_SdotPlanNd.py:1510-1535, 1785-1805: seeds the doubles cannot separate are merged, and the oracle's
    diagram at the GPU's weights gives each cluster its mass and every other cell its own"""
    from helpers import degenerate_clouds
    pos, groups = degenerate_clouds(d, 17)[name]
    n = len(pos)
    tol = (1e-9 if "1e-12" in name else 1e-11) / n
    plan = OtProblem(SumOfDiracs(pos), sdot.Box()).solve(Iterative(tol=tol, max_iter=60, on_failure="ignore"))
    assert plan.converged, (plan.stats["status"], plan.stats["nb_iter"], plan.stats["residual"])
    _check_aggregated(f"{d}D {name}", plan, pos, groups, tol)
    if plan.stats["status"] == "converged (aggregated)":
        # the re-splitting ran (sdotplan/Newton.h:434-471): its diagrams are counted, and the full residual it left is
        # the one reported
        assert plan.stats["nb_polish"] >= 1 and plan.stats["residual_full"] > tol, (name, plan.stats["nb_polish"])
    g = O.cells(pos, np.asarray(plan.weights).reshape(-1))["mass"]
    nu = np.asarray(plan.target_masses).reshape(-1)
    alone = np.ones(n, dtype=bool)
    for members, exact in groups:
        alone[members] = False
        if not exact:                # (two equal points: the oracle counts their cell twice)
            assert abs(g[members].sum() - nu[members].sum()) < 1e-8 / n, (name, g[members].sum() - nu[members].sum())
    assert np.abs(g[alone] - nu[alone]).max() < 1e-8 / n, name
    if any(exact for _, exact in groups) or len(np.unique(pos, axis=0)) < n:
        return
    # without the aggregation: the floor of the weights' doubles
    off = OtProblem(SumOfDiracs(pos), sdot.Box()).solve(Iterative(tol=tol, max_iter=60, aggregate=False, on_failure="ignore"))
    assert not off.converged and off.stats["aggregation"] == "off" and off.clusters is None, (name, off.stats["status"])


def test_the_aggregation_changes_nothing_without_such_seeds():
    """tests/test_SdotPlanNd.py:1544-1552: a cloud without near pairs, the same plan to the bit"""
    rng = np.random.default_rng(8)
    pos = rng.uniform(size=(4000, 2))
    on, off = [OtProblem(SumOfDiracs(pos), sdot.Box()).solve(Iterative(tol=1e-10 / 4000, max_iter=60, aggregate=agg)) for agg in (True, False)]
    assert on.clusters is None and on.stats["aggregation"] == "none" and on.stats["duplicates"] == "checked"
    assert np.array_equal(np.asarray(on.weights), np.asarray(off.weights))


@pytest.mark.parametrize("continuation", ["auto", "always"])
def test_an_image_with_a_hole_takes_the_blur_continuation(continuation):
    """tests/test_SdotPlanNd.py:1032-1040: a contrasted image with zeros; the image blurred on its grid, stage by stage,
    as the oracle does it: the same stages and the same plan"""
    rng = np.random.default_rng(201)
    n = 1500
    pos = rng.uniform(0.001, 0.999, size=(n, 2))
    nu = rng.uniform(0.5, 1.5, n)
    nu /= nu.sum()
    vals = 0.1 + 0.9 * rng.random((32, 32))
    vals[4:12, 18:28] = 0
    vals[20:23, :] += 4
    img = sdot.Image(vals, frame=[1 / 32, 1 / 32])
    plan = OtProblem(SumOfDiracs(pos, nu), img).solve(Iterative(tol=1e-10 / n, max_iter=80, continuation=continuation))
    assert plan.converged and plan.stats["nb_continuation_steps"] > 1, plan.stats
    norm = img.normalized_version()
    ref = O.solve(pos, nu=nu, tol_abs=1e-10 / n, maxit=80, continuation={"auto": 1, "always": 2}[continuation],
                  density=("image", [0, 0], [1 / 32, 1 / 32], norm.values))
    assert ref["stats"]["status"] == 1
    assert plan.stats["nb_continuation_steps"] == ref["stats"]["nb_continuation_steps"]
    assert np.abs(plan.weights - ref["weights"]).max() <= 1e-7 * np.abs(ref["weights"]).max()
    ss = [h["s"] for h in plan.history]
    assert ss[0] > 0 and ss[-1] == 0 and all(b <= a for a, b in zip(ss, ss[1:]))


def test_an_almost_empty_image_takes_the_blur_continuation():
    """tests/test_SdotPlanNd.py:397-405: two spots on a 1e-6 floor; `auto` starts the continuation and the plan converges"""
    rng = np.random.default_rng(91)
    pos = rng.uniform(0, 1, size=(400, 2))
    values = np.full((32, 32), 1e-6)
    values[6:10, 6:10] = 1.0
    values[20:26, 18:24] = 0.7
    img = sdot.Image(values, frame=[1 / 32, 1 / 32])
    plan = OtProblem(SumOfDiracs(pos), img).solve(Iterative(max_iter=100, tuning=Tuning(mass_rtol=1e-6)))
    assert plan.converged and plan.stats["nb_continuation_steps"] > 1, plan.stats
    assert np.allclose(plan.cell_masses, plan.target_masses, rtol=1e-5)


def _scattered_target(d, nb_gaussians, seed, sigma=0.13):
    """tests/test_SdotPlanNd.py:24-32: narrow, separate bumps over [0.3, 0.7]^d (the hard case of the damping)"""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.3, 0.7, size=(nb_gaussians, d))
    return sdot.SumOfGaussians(pos, np.full(nb_gaussians, sigma), weights=rng.uniform(0.7, 1.3, nb_gaussians))


def test_the_limits_step_reaches_the_same_plan_with_fewer_diagrams():
    """tests/test_SdotPlanNd.py:349-371: `step = "limits"` gives the weights of the trials with fewer diagrams, the step
    brought under the limits of the cells below the floor instead of halved"""
    rng = np.random.default_rng(81)
    pos = rng.uniform(0.1, 0.9, size=(60, 2))
    dst = _scattered_target(2, 4, seed=6)
    it = dict(max_iter=200, tol=1e-12, continuation="never")
    a = OtProblem(SumOfDiracs(pos), dst).solve(Iterative(**it, tuning=Tuning(step="trials", residual="lin")))
    b = OtProblem(SumOfDiracs(pos), dst).solve(Iterative(**it, tuning=Tuning(step="limits", residual="lin")))
    assert a.converged and b.converged, (a.stats, b.stats)
    assert np.allclose(a.weights, b.weights, atol=1e-9)
    assert b.stats["nb_diag"] <= a.stats["nb_diag"], (a.stats["nb_diag"], b.stats["nb_diag"])
    assert b.stats["nb_cell_lim"] > 0 and b.stats["nb_limit_rounds"] > 0, b.stats


@pytest.mark.parametrize("continuation", ["never", "auto"])
def test_the_limits_step_reaches_the_oracle_plan(continuation):
    """tests/test_SdotPlanNd.py:1023-1040: a soft image directly, and an image with a hole through the continuation, with
    the limits step: the plan of the oracle's trials"""
    rng = np.random.default_rng(201)
    n = 1500
    pos = rng.uniform(0.001, 0.999, size=(n, 2))
    nu = rng.uniform(0.5, 1.5, n)
    nu /= nu.sum()
    if continuation == "never":
        vals = 1 + 2 * rng.random((24, 17))
    else:
        vals = 0.1 + 0.9 * rng.random((32, 32))
        vals[4:12, 18:28] = 0
        vals[20:23, :] += 4
    step = [1 / vals.shape[0], 1 / vals.shape[1]]
    img = sdot.Image(vals, frame=step)
    plan = OtProblem(SumOfDiracs(pos, nu), img).solve(Iterative(tol=1e-10 / n, max_iter=80, continuation=continuation,
                                                                tuning=Tuning(step="limits")))
    assert plan.converged, plan.stats
    norm = img.normalized_version()
    ref = O.solve(pos, nu=nu, tol_abs=1e-10 / n, maxit=80, continuation={"never": 0, "auto": 1}[continuation],
                  density=("image", [0, 0], step, norm.values))
    assert ref["stats"]["status"] == 1
    assert np.abs(plan.weights - ref["weights"]).max() <= 1e-7 * np.abs(ref["weights"]).max()
