"""W2 of a batch of semi-discrete transports as a differentiable torch op.

    cost = w2_batch(positions, nu=None, target=None)        # positions [B, N, d] on a CUDA device, FP32 or FP64
    cost.sum().backward()                                   # positions.grad, nu.grad
    w = weights_batch(positions, nu)                        # the fitted weights [B, N], differentiable too
    b = barycentres_batch(positions, nu)                    # the cells' barycentres [B, N, d], differentiable too

Forward: ONE call of the C ABI (`sdot_solve_batch`) on the device pointers -- the B problems advance together.
Backward: the hand-written kernel `sdot_w2_backward` -- the envelope theorem at the fitted weights,
d W2 / d p_i = 2 m_i (p_i - b_i) and d W2 / d nu_i = w_i projected on sum(d nu) = 0 (SdotPlanNd.py:1037-1040,
1107-1122).  The weights' backward is the implicit-function derivative (SdotPlanNd.py:1018-1050): one Laplacian solve
and one adjoint of the masses a problem, `weights_vjp`.  The barycentres' backward (SdotPlanNd.py:1051-1070: first / mass at
the live weights) adds the adjoint of the masses and first moments at fixed weights (`sdot_cells_vjp_moments`) to the
weights' own.  PyTorch only owns the device memory and the autograd graph.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .OtProblem import Iterative, Tuning


def _options(settings):
    from .SdotPlanNd import solver_options
    return solver_options(settings, 0)


def _target_density(target, d):
    from .PowerDiagram import _domain_box
    from .distributions import Box
    t = (target or Box(nb_dims=d)).normalized_version(nb_dims=d)
    lo, hi = _domain_box(t.bounding_half_spaces(), d)
    return t._sdot_density(), lo, hi


class _W2Batch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, nu, target, settings):
        B, N, d = positions.shape
        dev = positions.device
        pos = positions.detach().to(torch.float64).contiguous()
        nuv = None if nu is None else (nu.detach().to(torch.float64) / nu.detach().to(torch.float64).sum(dim=1, keepdim=True)).contiguous()
        dens, lo, hi = _target_density(target, d)
        if dens[0] != "uniform":
            raise NotImplementedError("w2_batch: uniform targets (the differentiable batch); other targets through OtProblem")
        weights = torch.empty(B, N, dtype=torch.float64, device=dev)
        masses = torch.empty(B, N, dtype=torch.float64, device=dev)
        bary = torch.empty(B, N, d, dtype=torch.float64, device=dev)
        cost = torch.empty(B, dtype=torch.float64, device=dev)
        opts = _options(settings)
        descs, outs = (_lib.SolveDesc * B)(), (_lib.SolveOut * B)()
        for b in range(B):
            sd = _lib.SolveDesc()
            sd.diagram.dim, sd.diagram.n = d, N
            sd.diagram.positions = pos[b].data_ptr()
            sd.diagram.weights = None
            for a in range(d):
                sd.diagram.box_lo[a], sd.diagram.box_hi[a] = float(lo[a]), float(hi[a])
            sd.diagram.density.kind, sd.diagram.density.value = _lib.DENSITY_UNIFORM, float(dens[1])
            sd.diagram.memory = _lib.SDOT_DEVICE
            sd.nu = None if nuv is None else nuv[b].data_ptr()
            for q, name in enumerate(_lib.OPTIONS):
                sd.options[q] = float(opts[name])
            descs[b] = sd
            so = _lib.SolveOut()
            so.weights, so.masses = weights[b].data_ptr(), masses[b].data_ptr()
            so.barycentres, so.cost = bary[b].data_ptr(), cost[b:b + 1].data_ptr()
            outs[b] = so
        torch.cuda.synchronize(dev)
        sts = (_lib.Status * B)()
        code = _lib.load().sdot_solve_batch(_lib.context(dev.index), B, descs, outs, sts)
        for b in range(B):
            if sts[b].code:
                _lib.raise_for(sts[b].code, sts[b], "w2_batch")
        if code:
            raise RuntimeError("w2_batch: the batch failed")
        stats = np.array([outs[b].stats[:] for b in range(B)])
        failed = ~np.isin(stats[:, 0], (1, 7))          # converged, or converged on the clusters of near-coincident seeds
        if settings.on_failure == "raise" and failed.any():
            raise RuntimeError(f"w2_batch: {failed.sum()} of {B} solves did not converge")
        ctx.save_for_backward(positions, masses, bary, weights)
        ctx.has_nu = nu is not None
        ctx.nu_dtype = None if nu is None else nu.dtype
        ctx.stats = stats
        return cost

    @staticmethod
    def backward(ctx, grad_cost):
        positions, masses, bary, weights = ctx.saved_tensors
        B, N, d = positions.shape
        pos = positions.detach().contiguous()
        fp32 = pos.dtype == torch.float32
        gpos = torch.empty_like(pos)
        gnu = torch.empty(B, N, dtype=pos.dtype, device=pos.device)
        g = grad_cost.detach().to(torch.float64).contiguous()
        torch.cuda.synchronize(pos.device)
        st = _lib.Status()
        _lib.raise_for(_lib.load().sdot_w2_backward(_lib.context(pos.device.index), B, N, d, pos.data_ptr(), int(fp32), masses.data_ptr(),
                                                    bary.data_ptr(), weights.data_ptr(), g.data_ptr(), gpos.data_ptr(), gnu.data_ptr(),
                                                    ctypes.byref(st)), st, "sdot_w2_backward")
        _lib.load().sdot_context_synchronize(_lib.context(pos.device.index), ctypes.byref(st))
        return gpos, (gnu.to(ctx.nu_dtype) if ctx.has_nu else None), None, None


def weights_vjp(pos, w, nu, grad_w, laplacian, solve, masses_vjp, domain_mass=1.0):
    """the implicit-function derivative of the fitted weights of one transport (SdotPlanNd.py:1018-1050).

    At the fitted weights m(w, p) = nu_eff = M nu / sum(nu) (M the domain's mass, fixed), with the gauge w[0] = 0. The
    jacobian of the masses in the weights is the Laplacian L, so dw = P L^+ (d nu_eff - J_p dp), P = I - 1 e_0^T. For a
    cotangent g of the weights: lambda solves L lambda = P^T g = g - e_0 sum(g) (of zero sum), then
        grad_p = - J_p^T lambda,     grad_nu = M / sum(nu) (lambda - (nu . lambda) / sum(nu)).
    `laplacian(pos, w)` gives the CSR (row_ptr, cols, vals, dia) at the fitted weights, `solve(row_ptr, cols, vals, dia,
    rhs)` one solution of L x = rhs, `masses_vjp(pos, w, lam)` J_p^T lam ([n, d]). Returns (grad_p, grad_nu or None)."""
    g = np.asarray(grad_w, dtype=np.float64).reshape(-1)
    rhs = g.copy()
    rhs[0] -= g.sum()
    row, cols, vals, dia = laplacian(pos, w)
    lam = np.asarray(solve(row, cols, vals, dia, rhs), dtype=np.float64).reshape(-1)
    gp = -np.asarray(masses_vjp(pos, w, lam), dtype=np.float64)
    gnu = None
    if nu is not None:
        nu = np.asarray(nu, dtype=np.float64).reshape(-1)
        s = nu.sum()
        gnu = domain_mass / s * (lam - (nu @ lam) / s)
    return gp, gnu


def barycentres_vjp(pos, w, nu, masses, bary, grad_b, moments_vjp, laplacian, solve, masses_vjp, domain_mass=1.0):
    """the derivative of the barycentres of one transport at its fitted weights (SdotPlanNd.py:1051-1070).

    b_i = F_i / m_i with F_i = int_cell x rho; an empty cell keeps its seed. For a cotangent g of the barycentres:
    g_F = g / m and g_m = - (g . b) / m; `moments_vjp(pos, w, g_m, g_F)` gives (grad_p, grad_w) of m and F at fixed
    weights; the weights' cotangent grad_w is carried to the positions and target masses by `weights_vjp` (its other
    arguments). Returns (grad_p [n, d], grad_nu [n] or None)."""
    g = np.asarray(grad_b, dtype=np.float64)
    m = np.asarray(masses, dtype=np.float64).reshape(-1)
    full = m > 0
    inv = np.where(full, 1.0 / np.where(full, m, 1.0), 0.0)
    gF = g * inv[:, None]
    gm = -(g * np.asarray(bary, dtype=np.float64)).sum(axis=1) * inv
    gpe, gwe = moments_vjp(pos, w, gm, gF)
    gp, gnu = weights_vjp(pos, w, nu, gwe, laplacian, solve, masses_vjp, domain_mass)
    gp = gp + np.asarray(gpe, dtype=np.float64)
    gp[~full] += g[~full]
    return gp, gnu


def _solve_one(row, cols, vals, dia, rhs):
    x, its = _lib.linear_solve(row, cols, vals, dia, rhs, tol=1e-12, method=1)
    if its[0] < 0:
        raise RuntimeError("weights_batch backward: the Laplacian solve did not converge")
    return x[0]


def _pullback(pos, w, nub, grad_w, lo, hi, dens, domain_mass):
    """`weights_vjp` through the C ABI: the Laplacian, its CG solve and the masses adjoint of one problem"""
    return weights_vjp(pos, w, nub, grad_w, lambda p, ww: _lib.laplacian(p, ww, lo, hi, dens), _solve_one,
                       lambda p, ww, lam: _lib.cells_vjp(p, ww, lo, hi, dens, lam)[0], domain_mass)


def _forward_saved(positions, nu, target, settings):
    """the batched solve on detached inputs: (weights, masses, barycentres), all [B, N(, d)] on the device"""
    with torch.enable_grad():
        p = positions.detach().requires_grad_(True)
        cost = _W2Batch.apply(p, None if nu is None else nu.detach(), target, settings)
    node = cost.grad_fn
    return node.saved_tensors[3], node.saved_tensors[1], node.saved_tensors[2]


class _WeightsBatch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, nu, target, settings):
        weights, masses, _ = _forward_saved(positions, nu, target, settings)
        ctx.save_for_backward(positions, weights, masses, nu if nu is not None else torch.empty(0, device=positions.device))
        ctx.has_nu, ctx.target = nu is not None, target
        return weights.clone()

    @staticmethod
    def backward(ctx, grad_w):
        positions, weights, masses, nu = ctx.saved_tensors
        B, N, d = positions.shape
        _, lo, hi = _target_density(ctx.target, d)
        dens = _target_density(ctx.target, d)[0]
        gp = torch.empty(B, N, d, dtype=torch.float64)
        gn = torch.empty(B, N, dtype=torch.float64) if ctx.has_nu else None
        for b in range(B):
            pos = positions[b].detach().to(torch.float64).cpu().numpy()
            w = weights[b].cpu().numpy()
            nub = nu[b].detach().to(torch.float64).cpu().numpy() if ctx.has_nu else None
            x, xn = _pullback(pos, w, nub, grad_w[b].detach().to(torch.float64).cpu().numpy(), lo, hi, dens, float(masses[b].sum()))
            gp[b] = torch.from_numpy(x)
            if ctx.has_nu:
                gn[b] = torch.from_numpy(xn)
        gp = gp.to(device=positions.device, dtype=positions.dtype)
        gn = None if gn is None else gn.to(device=positions.device, dtype=nu.dtype)
        return gp, gn, None, None


class _BarycentresBatch(torch.autograd.Function):
    """b_i = F_i / m_i (F_i = int_cell x rho) at the fitted weights; an empty cell keeps its seed (SdotPlanNd.py:1066-1068).
    For a cotangent g_b: g_F = g_b / m, g_m = - (g_b . b) / m; the adjoint at fixed weights gives the explicit part and a
    cotangent of the weights, which the implicit function theorem carries to the positions and target masses."""

    @staticmethod
    def forward(ctx, positions, nu, target, settings):
        weights, masses, bary = _forward_saved(positions, nu, target, settings)
        ctx.save_for_backward(positions, weights, masses, bary, nu if nu is not None else torch.empty(0, device=positions.device))
        ctx.has_nu, ctx.target = nu is not None, target
        return bary.clone()

    @staticmethod
    def backward(ctx, grad_b):
        positions, weights, masses, bary, nu = ctx.saved_tensors
        B, N, d = positions.shape
        dens, lo, hi = _target_density(ctx.target, d)
        gp = torch.empty(B, N, d, dtype=torch.float64)
        gn = torch.empty(B, N, dtype=torch.float64) if ctx.has_nu else None
        for b in range(B):
            pos = positions[b].detach().to(torch.float64).cpu().numpy()
            w, m, bb = weights[b].cpu().numpy(), masses[b].cpu().numpy(), bary[b].cpu().numpy()
            g = grad_b[b].detach().to(torch.float64).cpu().numpy()
            nub = nu[b].detach().to(torch.float64).cpu().numpy() if ctx.has_nu else None
            x, xn = barycentres_vjp(pos, w, nub, m, bb, g, lambda p, ww, gm, gF: _lib.cells_vjp(p, ww, lo, hi, dens, gm, gF),
                                    lambda p, ww: _lib.laplacian(p, ww, lo, hi, dens), _solve_one,
                                    lambda p, ww, lam: _lib.cells_vjp(p, ww, lo, hi, dens, lam)[0], float(m.sum()))
            gp[b] = torch.from_numpy(x)
            if ctx.has_nu:
                gn[b] = torch.from_numpy(xn)
        gp = gp.to(device=positions.device, dtype=positions.dtype)
        gn = None if gn is None else gn.to(device=positions.device, dtype=nu.dtype)
        return gp, gn, None, None


def barycentres_batch(positions, nu=None, target=None, settings=None):
    """the barycentres of the cells of the B transports [B, N, d] (FP64) at the fitted weights, differentiable wrt
    `positions` [B, N, d] and `nu` [B, N] (a constant density): the adjoint of the masses and first moments, then the
    weights' implicit derivative, one Laplacian solve a problem"""
    settings = settings or Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-12))
    return _BarycentresBatch.apply(positions, nu, target, settings)


def weights_batch(positions, nu=None, target=None, settings=None):
    """the fitted weights of the B transports [B, N] (FP64, gauge w[0] = 0), differentiable wrt `positions` [B, N, d] and
    `nu` [B, N] by the implicit function theorem (`weights_vjp`: one Laplacian solve and one masses adjoint a problem,
    through the C ABI)"""
    settings = settings or Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-12))
    return _WeightsBatch.apply(positions, nu, target, settings)


def w2_batch(positions, nu=None, target=None, settings=None):
    """W2^2 of each of the B transports [B] (FP64), differentiable wrt `positions` [B, N, d] and `nu` [B, N]"""
    settings = settings or Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-10))
    return _W2Batch.apply(positions, nu, target, settings)


def solve_batch(positions, nu=None, target=None, settings=None):
    """the batched forward alone: (cost [B], weights [B, N], masses [B, N], barycentres [B, N, d]), all on the device"""
    settings = settings or Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-10))
    with torch.enable_grad():
        p = positions.detach().requires_grad_(True)
        cost = _W2Batch.apply(p, nu, target, settings)
    node = cost.grad_fn
    return cost.detach(), node.saved_tensors[3], node.saved_tensors[1], node.saved_tensors[2]
