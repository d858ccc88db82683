"""W2 of a batch of semi-discrete transports as a differentiable torch op.

    cost = w2_batch(positions, nu=None, target=None)        # positions [B, N, d] on a CUDA device, FP32 or FP64
    cost.sum().backward()                                   # positions.grad, nu.grad

Forward: ONE call of the C ABI (`sdot_solve_batch`) on the device pointers -- the B problems advance together.
Backward: the hand-written kernel `sdot_w2_backward` -- the envelope theorem at the fitted weights,
d W2 / d p_i = 2 m_i (p_i - b_i) and d W2 / d nu_i = w_i projected on sum(d nu) = 0 (SdotPlanNd.py:1037-1040,
1107-1122).  PyTorch only owns the device memory and the autograd graph.
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
