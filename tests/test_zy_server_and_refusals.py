"""The C ABI's serving layer, its refusals, the weights' derivative and the grid clouds, on a device.

The server (sdot_server_*: continuous batching) against the batched solve of the same requests; the precision variants
this build does not have, refused before any launch; the implicit-function derivative of the fitted weights against
differences of the solve; seeds on grids, whose cells are the grid's boxes."""
import numpy as np
import pytest

import sdot
from sdot import Iterative, Tuning

pytestmark = pytest.mark.gpu


def _pd(pos):
    d = pos.shape[1]
    return sdot.PowerDiagram(pos, boundaries=sdot.box_half_spaces(np.zeros(d), np.ones(d)))


def test_the_server_returns_the_plans_of_the_batched_solve():
    """continuous batching (sdot_server_*): requests submitted one after the other, admitted while the others run, come
    back with the plans the batched solve gives them -- weights, masses, status and the clusters of near-coincident
    seeds (a pair 1e-9 apart, merged)"""
    from helpers import degenerate_clouds
    from sdot import _lib
    from sdot.PowerDiagram import _domain_box
    from sdot.SdotPlanNd import solver_options
    from sdot.server import Server
    rng = np.random.default_rng(61)
    pair, _ = degenerate_clouds(2, 17)["pair at 1e-9"]
    g = sdot.SumOfGaussians(rng.uniform(0.3, 0.7, size=(3, 2)), [0.1, 0.12, 0.08], support_box=(np.zeros(2), np.ones(2)))
    cases = [(rng.uniform(size=(3000, 2)), sdot.Box()), (rng.uniform(size=(1500, 3)), sdot.Box()), (rng.uniform(size=(1000, 2)), g),
             (pair, sdot.Box())]
    settings = [Iterative(tol=0.0, max_iter=60, tuning=Tuning(mass_rtol=1e-9))] * 3 + [Iterative(tol=1e-11 / len(pair), max_iter=60)]
    srv = Server()
    try:
        tickets = [srv.submit(pos, tg, settings=st) for (pos, tg), st in zip(cases, settings)]
        served = [srv.result(t) for t in tickets]
    finally:
        srv.close()
    for (pos, tg), st, r in zip(cases, settings, served):
        n, d = pos.shape
        t = tg.normalized_version(nb_dims=d)
        lo, hi = _domain_box(t.bounding_half_spaces(), d)
        b = _lib.solve_batch([(pos, None, None, lo, hi, t._sdot_density())], [solver_options(st, n, d)])[0]
        assert r["stats"][0] == b["stats"][0] and b["stats"][0] in (1, 7), (r["stats"][0], b["stats"][0])
        assert np.abs(r["weights"] - b["weights"]).max() <= 1e-12 * np.abs(b["weights"]).max()
        assert np.abs(r["masses"] - b["masses"]).max() <= 1e-12 / n
        assert np.array_equal(r["clusters"], b["clusters"])
    assert served[-1]["stats"][0] == 7 and (served[-1]["clusters"] != np.arange(len(pair))).sum() == 1


def test_the_unbuilt_precisions_are_refused():
    """no silent FP64 in place of an FP32 clip that is not built: in 3D, `precision` 1 of a cells call, and the
    `precision` option of a solve, are SDOT_ERR_UNSUPPORTED (NotImplementedError), before any launch; `lin_precision` 2
    is an argument error"""
    import ctypes
    from sdot import _lib
    from sdot.SdotPlanNd import solver_options
    pos = np.random.default_rng(3).uniform(size=(200, 3))
    lo, hi = np.zeros(3), np.ones(3)
    keep = []
    desc = _lib.diagram_desc(pos, None, lo, hi, ("uniform", 1.0), keep)
    m = np.zeros(200)
    out = _lib.CellsOut(masses=m.ctypes.data, precision=1)
    st = _lib.Status()
    assert _lib.load().sdot_cells(_lib.context(), ctypes.byref(desc), ctypes.byref(out), ctypes.byref(st)) == _lib.SDOT_ERR_UNSUPPORTED
    opts = dict(solver_options(Iterative(), 200), precision=1)
    r = _lib.solve_batch([(pos, None, None, lo, hi, ("uniform", 1.0))], [opts])[0]
    assert isinstance(r, NotImplementedError), r
    opts = dict(solver_options(Iterative(), 200), lin_precision=2)
    r = _lib.solve_batch([(pos, None, None, lo, hi, ("uniform", 1.0))], [opts])[0]
    assert isinstance(r, ValueError), r
    assert np.abs(_pd(pos[:, :2]).measures.sum() - 1) < 1e-12   # the context is still usable


def test_the_weights_are_differentiable():
    """SdotPlanNd.py:1018-1050: `torch_ops.weights_batch`'s backward (one Laplacian solve and one adjoint of the masses
    through the C ABI) against central differences of the GPU solve itself, in the positions and in the target masses"""
    import torch
    from sdot.torch_ops import weights_batch
    rng = np.random.default_rng(7)
    n = 200
    pos = torch.tensor(rng.uniform(0.2, 0.8, size=(1, n, 2)), dtype=torch.float64, device="cuda", requires_grad=True)
    nu = torch.tensor(rng.uniform(0.5, 1.5, size=(1, n)), dtype=torch.float64, device="cuda", requires_grad=True)
    settings = Iterative(tol=0.0, max_iter=100, tuning=Tuning(mass_rtol=1e-12))
    g = torch.tensor(rng.standard_normal((1, n)), dtype=torch.float64, device="cuda")
    (weights_batch(pos, nu, settings=settings) * g).sum().backward()

    def loss(p, q):
        with torch.no_grad():
            return float((weights_batch(p, q, settings=settings) * g).sum())
    h = 1e-5
    for k, a in ((3, 0), (50, 1), (117, 0), (199, 1)):
        e = torch.zeros_like(pos)
        e[0, k, a] = h
        fd = (loss(pos.detach() + e, nu.detach()) - loss(pos.detach() - e, nu.detach())) / (2 * h)
        assert abs(float(pos.grad[0, k, a]) - fd) < 1e-5 * max(1.0, abs(fd)), (k, a, float(pos.grad[0, k, a]), fd)
    for k in (0, 77, 150):
        e = torch.zeros_like(nu)
        e[0, k] = h
        fd = (loss(pos.detach(), nu.detach() + e) - loss(pos.detach(), nu.detach() - e)) / (2 * h)
        assert abs(float(nu.grad[0, k]) - fd) < 1e-5 * max(1.0, abs(fd)), (k, float(nu.grad[0, k]), fd)


@pytest.mark.parametrize("d", [2, 3])
def test_the_barycentres_are_differentiable(d):
    """SdotPlanNd.py:1051-1070 (the barycentres first / mass at the live weights, with their implicit derivative):
    `torch_ops.barycentres_batch`'s backward (the adjoint of the masses and first moments, then the weights' implicit
    derivative) against central differences of the GPU solve's barycentres, in the positions and the target masses"""
    import torch
    from sdot.torch_ops import barycentres_batch
    rng = np.random.default_rng(8 + d)
    n = 200 if d == 2 else 80
    pos = torch.tensor(rng.uniform(0.2, 0.8, size=(1, n, d)), dtype=torch.float64, device="cuda", requires_grad=True)
    nu = torch.tensor(rng.uniform(0.5, 1.5, size=(1, n)), dtype=torch.float64, device="cuda", requires_grad=True)
    settings = Iterative(tol=0.0, max_iter=100, tuning=Tuning(mass_rtol=1e-12))
    g = torch.tensor(rng.standard_normal((1, n, d)), dtype=torch.float64, device="cuda")
    (barycentres_batch(pos, nu, settings=settings) * g).sum().backward()

    def loss(p, q):
        with torch.no_grad():
            return float((barycentres_batch(p, q, settings=settings) * g).sum())
    h = 1e-5
    scale = max(1.0, float(pos.grad.abs().max()))
    for k, a in ((3, 0), (50, 1), (71, d - 1), (n - 1, 0)):
        e = torch.zeros_like(pos)
        e[0, k, a] = h
        fd = (loss(pos.detach() + e, nu.detach()) - loss(pos.detach() - e, nu.detach())) / (2 * h)
        assert abs(float(pos.grad[0, k, a]) - fd) < 1e-5 * scale, (k, a, float(pos.grad[0, k, a]), fd)
    scale = max(1.0, float(nu.grad.abs().max()))
    for k in (0, 41, n - 2):
        e = torch.zeros_like(nu)
        e[0, k] = h
        fd = (loss(pos.detach(), nu.detach() + e) - loss(pos.detach(), nu.detach() - e)) / (2 * h)
        assert abs(float(nu.grad[0, k]) - fd) < 1e-5 * scale, (k, float(nu.grad[0, k]), fd)


@pytest.mark.parametrize("shape", [(40, 30), (12, 10, 8), (20, 20, 20)])
def test_grids_give_the_exact_boxes(shape):
    """tests/test_CardCells.py:166-187, 900-941: seeds on a grid (cuts through vertices already on the cell, the ties a
    clip must survive) have the grid's boxes as cells, 1e-10 relative"""
    d = len(shape)
    g = np.stack(np.meshgrid(*[(np.arange(k) + 0.5) / k for k in shape], indexing="ij"), axis=-1).reshape(-1, d)
    m = _pd(g).measures
    assert np.abs(m * len(g) - 1).max() < 1e-10 and abs(m.sum() - 1) < 1e-12
