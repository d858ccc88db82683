"""Two of the stated workloads at their full sizes, through the public API, checked against the oracle on a random
subset of their cells (the oracle builds the whole diagram's search grid, then computes only those cells).

* The 3D power diagram: N = 1,000,000 seeds uniform in [0,1]^3, weights uniform in [0, 1e-4], uniform density on the
  unit cube; every cell's neighbour set, volume, centroid and face areas (FP64 clipping: the FP32-clip variant is not
  built).  Bar: the volumes sum to 1 within 1e-12; on 10,000 random cells, volumes within 1e-10 relative (of the mean
  volume for the hidden and sliver cells that weights of the size of the spacing squared make), centroids within
  1e-9, neighbour sets of non-degenerate facets bit-exact, face areas within 1e-10 of the cell's largest.
* The 2D Newton on an image: N = 1,000,000 seeds uniform in [0,1]^2; the target a 1024 x 1024 piecewise-constant image,
  the sum of 16 isotropic gaussians (centres uniform, sigma uniform in [0.02, 0.1], amplitudes uniform in [0.5, 2]) at
  the pixel centres plus 1 % of the peak, normalised to mass 1; nu = 1/N; the Newton systems' CG in FP32 inside an FP64
  iterative refinement (a system on which the refinement stalls -- condition number times the FP32 rounding past 1 --
  is solved again by the FP64 CG over FP32 multigrid levels).  Bar: converged to max |m - nu| / nu <= 1e-8 (a cluster of
  seeds the doubles cannot separate by its sum); the oracle's masses of 10,000 random unclustered cells at the GPU's
  weights within 1.1e-8 relative of nu as well.
"""
import time

import numpy as np
import pytest

import oracle as O
import sdot
from helpers import neighbour_sets
from sdot import Iterative, OtProblem, SumOfDiracs, Tuning

pytestmark = pytest.mark.gpu


def test_3d_power_diagram_of_a_million_seeds():
    n, d = 1_000_000, 3
    rng = np.random.default_rng(20260302)
    pos = rng.uniform(size=(n, d))
    w = rng.uniform(0, 1e-4, size=n)
    pd = sdot.PowerDiagram(pos, w, boundaries=sdot.box_half_spaces(np.zeros(d), np.ones(d)))
    t0 = time.perf_counter()
    nb, ids, coef, meas = pd.facets()
    m, bary, _ = pd.barycenters_and_costs()
    secs = time.perf_counter() - t0
    assert abs(m.sum() - 1) < 1e-12, m.sum() - 1
    rows = np.sort(rng.choice(n, size=10_000, replace=False))
    ref = O.cells_rows(pos, rows, w)
    assert ref["status"] == 0
    rm = ref["mass"]
    err_v = np.abs(m[rows] - rm)
    assert (err_v <= 1e-10 * rm + 1e-14 / n).all(), err_v.max()
    full = rm > 1e-6 / n
    assert np.abs(bary[rows][full] - ref["bary"][full]).max() < 1e-9
    sub_nb, sub_ids, sub_meas = nb[rows], ids[rows], meas[rows]
    ga = neighbour_sets(sub_nb, sub_ids, sub_meas)
    gb = neighbour_sets(ref["nb"], ref["nid"], ref["nm"])
    # the neighbours whose facet sits in the ambiguous band [1e-9, 1e-6] of its cell's largest (presence decided by rounding)
    skip = set()
    for i in range(len(rows)):
        k = int(ref["nb"][i])
        top = ref["nm"][i, :k].max() if k else 0.0
        for j, v in zip(ref["nid"][i, :k], ref["nm"][i, :k]):
            if 1e-9 * top <= v <= 1e-6 * top:
                skip.add(int(j))
    bad = 0
    worst_area = 0.0
    for i in range(len(rows)):
        diff = {j for j in ga[i] ^ gb[i] if j not in skip}
        bad += bool(diff)
        a = {int(j): v for j, v in zip(sub_ids[i, : sub_nb[i]], sub_meas[i, : sub_nb[i]])}
        k = int(ref["nb"][i])
        top = ref["nm"][i, :k].max() if k else 0.0
        for j, v in zip(ref["nid"][i, :k], ref["nm"][i, :k]):
            if v > 1e-9 * top and int(j) in a:
                worst_area = max(worst_area, abs(a[int(j)] - v) / top)
    assert bad == 0, bad
    assert worst_area < 1e-10, worst_area
    print(f"\n3D power diagram, 1e6 seeds, w in [0, 1e-4]: facets + moments in {secs:.2f} s through the API; "
          f"sum of volumes - 1 = {m.sum() - 1:.1e}; on 1e4 cells: volume error max {err_v.max():.1e} "
          f"(relative {(err_v / np.maximum(rm, 1e-300))[full].max():.1e}), face areas {worst_area:.1e} of the cell's largest, "
          f"{int((rm == 0).sum())} hidden cells")


def _sixteen_gaussians_image(rng, res=1024):
    c = rng.uniform(size=(16, 2))
    s = rng.uniform(0.02, 0.1, size=16)
    a = rng.uniform(0.5, 2.0, size=16)
    xs = (np.arange(res) + 0.5) / res
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    v = np.zeros((res, res))
    for k in range(16):
        v += a[k] * np.exp(-((X - c[k, 0]) ** 2 + (Y - c[k, 1]) ** 2) / (2 * s[k] ** 2))
    v += 0.01 * v.max()
    return v


def test_2d_newton_on_a_1024_image_with_a_million_seeds():
    n = 1_000_000
    rng = np.random.default_rng(20260303)
    vals = _sixteen_gaussians_image(rng)
    img = sdot.Image(vals, frame=[1 / 1024, 1 / 1024])
    pos = rng.uniform(size=(n, 2))
    t0 = time.perf_counter()
    plan = OtProblem(SumOfDiracs(pos), img).solve(
        Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-8, linear_precision="mixed")))
    secs = time.perf_counter() - t0
    assert plan.converged, plan.stats["status"]
    nu = 1.0 / n
    # seeds the doubles of the weights cannot separate (status "converged (aggregated)") meet the tolerance as clusters
    # (tests/test_SdotPlanNd.py:1407-1432): each cluster's mass is its members' target
    m = np.asarray(plan.cell_masses).reshape(-1)
    cl = np.asarray(plan.clusters).reshape(-1)
    size = np.bincount(cl, minlength=n)
    alone = size[cl] == 1
    err = np.abs(m[alone] / nu - 1).max()
    if (~alone).any():
        sums = np.bincount(cl[~alone], weights=m[~alone], minlength=n)
        reps = np.unique(cl[~alone])
        err = max(err, np.abs(sums[reps] / (size[reps] * nu) - 1).max())
    assert err <= 1e-8, err
    norm = img.normalized_version()
    rows = np.sort(rng.choice(np.flatnonzero(alone), size=10_000, replace=False))
    ref = O.cells_rows(pos, rows, plan.weights, density=("image", [0, 0], [1 / 1024, 1 / 1024], norm.values))
    assert ref["status"] == 0
    oerr = np.abs(ref["mass"] / nu - 1).max()
    assert oerr <= 1.1e-8, oerr                    # (the two integrations of the image agree to ~1e-12 of a cell's mass)
    st = plan.stats
    print(f"\n2D Newton, 1e6 seeds, 1024^2 image of 16 gaussians, mixed CG: {secs:.2f} s, status {st['status']!r}, "
          f"{st['nb_iter']} Newton steps, {st['nb_diag']} diagrams, {st['nb_continuation_steps']} continuation stages, "
          f"{st['lin_nb_iter']} CG iterations, {int((~alone).sum())} seeds in clusters; max |m - nu| / nu = {err:.1e} (GPU), "
          f"{oerr:.1e} (oracle on 1e4 cells)")
