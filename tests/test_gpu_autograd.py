"""The differentiable batch: 64 independent 2D problems of N = 4096 FP32 positions against a uniform density;
forward solve and the backward of W2 wrt positions and target masses through the autograd.Function, checked by
central finite differences (h = 1e-4, FP64) on 32 random coordinates, then 50 gradient-descent steps.

The finite differences solve the 64 perturbed problems (32 coordinates x +-h) as ONE batch.  Gradient bar:
|fd - g| <= 1e-3 |g| + 1e-10 (the cost is solved to max |m - nu| / nu <= 1e-11)."""
import numpy as np
import pytest
import torch

from sdot import Iterative, Tuning
from sdot.torch_ops import solve_batch, w2_batch

pytestmark = pytest.mark.gpu

TIGHT = Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-11))


def test_the_gradient_of_a_batch_of_64_by_finite_differences():
    B, N = 64, 4096
    g = torch.Generator().manual_seed(7)
    pos = torch.rand(B, N, 2, generator=g, dtype=torch.float32).cuda().requires_grad_(True)
    nu = torch.full((B, N), 1.0 / N, dtype=torch.float64, device="cuda", requires_grad=True)
    cost = w2_batch(pos, nu, settings=TIGHT)
    assert cost.shape == (B,)
    cost.sum().backward()
    gp, gn = pos.grad.double().cpu().numpy(), nu.grad.cpu().numpy()
    assert np.isfinite(gp).all() and np.isfinite(gn).all()
    # 32 random coordinates: 24 positions and 8 target masses (perturbed by +-h on i and -+h on j: sum(d nu) = 0)
    rng = np.random.default_rng(11)
    h = 1e-4
    base = pos.detach().double()
    pp, nn, expect = [], [], []
    for k in range(32):
        b = int(rng.integers(B))
        if k < 24:
            i, a = int(rng.integers(N)), int(rng.integers(2))
            for s in (1, -1):
                q = base[b].clone()
                q[i, a] += s * h
                pp.append(q)
                nn.append(torch.full((N,), 1.0 / N, dtype=torch.float64, device="cuda"))
            expect.append(gp[b, i, a])
        else:
            i, j = rng.choice(N, size=2, replace=False)
            for s in (1, -1):
                v = torch.full((N,), 1.0 / N, dtype=torch.float64, device="cuda")
                v[int(i)] += s * h / N
                v[int(j)] -= s * h / N
                pp.append(base[b].clone())
                nn.append(v)
            expect.append((gn[b, i] - gn[b, j]) / N)
    c, _, _, _ = solve_batch(torch.stack(pp), torch.stack(nn), settings=TIGHT)
    c = c.cpu().numpy()
    fd = (c[0::2] - c[1::2]) / (2 * h)
    expect = np.array(expect)
    assert (np.abs(fd - expect) <= 1e-3 * np.abs(expect) + 1e-10).all(), np.c_[fd, expect][np.abs(fd - expect) > 1e-3 * np.abs(expect)]


def test_fifty_descent_steps_lower_the_cost():
    """50 gradient steps x <- x - grad / (2 m), i.e. the Lloyd step x <- b(x) (quantization.py:1-12)"""
    B, N = 64, 4096
    g = torch.Generator().manual_seed(8)
    pos = torch.rand(B, N, 2, generator=g, dtype=torch.float32).cuda()
    costs = []
    for step in range(50):
        p = pos.clone().requires_grad_(True)
        c = w2_batch(p, settings=Iterative(tol=0.0, tuning=Tuning(mass_rtol=1e-8)))
        c.sum().backward()
        costs.append(c.detach().cpu().numpy())
        with torch.no_grad():
            pos = (pos - p.grad * (N / 2.0)).clamp(0, 1)
    costs = np.array(costs)
    assert (costs[-1] < 0.5 * costs[0]).all()
    assert (np.diff(costs, axis=0) <= 1e-12).mean() > 0.95
