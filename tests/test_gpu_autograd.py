"""torch.autograd of arrival times through the GPU adjoint, checked by central finite differences."""
import numpy as np
import pytest

from hamiltonfastmarching_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _fd_check(params, cost0, receivers, cells, rel_tol):
    import torch
    from hamiltonfastmarching_b200.autograd import arrival_times
    rng = np.random.default_rng(0)
    t_obs = None

    def loss_of(c):
        T = arrival_times(params, c)
        tr = T.reshape(-1)[receivers]
        return ((tr - t_obs) ** 2).sum()

    with torch.no_grad():
        base = arrival_times(params, torch.from_numpy(cost0))
    t_obs = base.reshape(-1)[receivers] * torch.from_numpy(1.0 + 0.05 * rng.standard_normal(len(receivers)))
    c = torch.from_numpy(cost0.copy()).requires_grad_(True)
    L = loss_of(c)
    L.backward()
    g = c.grad.numpy().reshape(-1)
    for cell in cells:
        h = 1e-6 * cost0.reshape(-1)[cell]
        cp, cm = cost0.copy().reshape(-1), cost0.copy().reshape(-1)
        cp[cell] += h
        cm[cell] -= h
        with torch.no_grad():
            fd = (loss_of(torch.from_numpy(cp.reshape(cost0.shape))) -
                  loss_of(torch.from_numpy(cm.reshape(cost0.shape)))).item() / (2 * h)
        scale = max(abs(fd), 1e-3 * np.max(np.abs(g)))
        assert abs(g[cell] - fd) <= rel_tol * scale, (cell, g[cell], fd)


def test_riemann2_cost_multiplier_gradient_matches_finite_differences():
    p = W.riemann2_case(48, aniso=4.0, seed=2)
    rng = np.random.default_rng(1)
    cost = 1.0 + 0.3 * rng.uniform(size=(48, 48))
    receivers = rng.choice(48 * 48, 16, replace=False)
    # cells on the upwind paths of the receivers carry gradient; pick some with nonzero gradient
    import torch
    from hamiltonfastmarching_b200.autograd import arrival_times
    c = torch.from_numpy(cost.copy()).requires_grad_(True)
    arrival_times(p, c).reshape(-1)[receivers].sum().backward()
    g = c.grad.numpy().reshape(-1)
    cells = np.flatnonzero(np.abs(g) > 1e-3 * np.abs(g).max())[::37][:8]
    _fd_check(p, cost, receivers, cells, rel_tol=2e-3)


def test_reedsshepp2_cost_gradient_matches_finite_differences():
    p = W.curvature2_case(32, 24, "ReedsShepp2", n_curves=5)
    cost = np.ascontiguousarray(p.pop("cost"))
    rng = np.random.default_rng(3)
    receivers = rng.choice(32 * 32 * 24, 12, replace=False)
    import torch
    from hamiltonfastmarching_b200.autograd import arrival_times
    c = torch.from_numpy(cost.copy()).requires_grad_(True)
    arrival_times(p, c).reshape(-1)[receivers].sum().backward()
    g = c.grad.numpy().reshape(-1)
    cells = np.flatnonzero(np.abs(g) > 1e-3 * np.abs(g).max())[::13][:8]
    _fd_check(p, cost, receivers, cells, rel_tol=2e-3)
