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


def test_tti3_velocity_gradient_matches_finite_differences():
    """d loss / d vp with loss = sum over top-face receivers of (T - T_obs)^2, T_obs from a perturbed
    vp (Gaussian blob), through the TTI3 adjoint; vp enters as the norm multiplier vp_ref / vp."""
    import torch
    from hamiltonfastmarching_b200.autograd import arrival_times
    n, h = 24, 0.01
    p = W.tti3_case(n, h=h, seed=4)
    vp0 = p.pop("_vp")
    obs = W.tti3_case(n, h=h, seed=4, blob=((0.12, 0.12, 0.12), 0.04, 0.05))
    vp_obs = obs.pop("_vp")
    rng = np.random.default_rng(5)
    rx = rng.integers(0, n, (16, 2))
    receivers = np.ravel_multi_index((rx[:, 0], rx[:, 1], np.zeros(16, int)), (n, n, n))
    with torch.no_grad():
        t_obs = arrival_times(p, torch.from_numpy(vp0 / vp_obs)).reshape(-1)[receivers]

    def loss_of(vp):
        T = arrival_times(p, torch.from_numpy(vp0) / vp)
        return ((T.reshape(-1)[receivers] - t_obs) ** 2).sum()

    vp = torch.from_numpy(vp0.copy()).requires_grad_(True)
    loss_of(vp).backward()
    g = vp.grad.numpy().reshape(-1)
    assert np.all(np.isfinite(g)) and np.abs(g).max() > 0
    cells = np.flatnonzero(np.abs(g) > 1e-2 * np.abs(g).max())
    cells = rng.choice(cells, min(8, len(cells)), replace=False)
    for cell in cells:
        d = 1e-6 * vp0.reshape(-1)[cell]
        vpp, vpm = vp0.copy().reshape(-1), vp0.copy().reshape(-1)
        vpp[cell] += d
        vpm[cell] -= d
        with torch.no_grad():
            fd = (loss_of(torch.from_numpy(vpp.reshape(vp0.shape))) -
                  loss_of(torch.from_numpy(vpm.reshape(vp0.shape)))).item() / (2 * d)
        scale = max(abs(fd), 1e-3 * np.abs(g).max())
        assert abs(g[cell] - fd) <= 5e-3 * scale, (cell, g[cell], fd)


@pytest.mark.parametrize("model", ["Isotropic2", "Diagonal2"])
def test_isotropic_and_diagonal_cost_gradient_matches_finite_differences(model):
    """cost is the model's cost field (per axis for Diagonal2, shape dims + (2,)); the gradient is
    the costSensitivity of the retained solve, d(values)/d(cost)."""
    import torch
    from hamiltonfastmarching_b200.autograd import arrival_times
    n = 40
    rng = np.random.default_rng(7)
    shape = (n, n) if model == "Isotropic2" else (n, n, 2)
    cost = 1.0 + 0.5 * rng.random(shape)
    walls = np.zeros((n, n))
    walls[20, 5:30] = 1.0
    p = {"model": model, "arrayOrdering": "RowMajor", "dims": np.array([n, n], float), "gridScale": 1.0 / n,
         "walls": walls, "seeds": np.array([[0.3, 0.2], [0.7, 0.15]])}
    receivers = rng.choice(np.flatnonzero(walls.ravel() == 0), 12, replace=False)
    c = torch.from_numpy(cost.copy()).requires_grad_(True)
    arrival_times(p, c).reshape(-1)[receivers].sum().backward()
    assert c.grad.shape == cost.shape
    g = c.grad.numpy().reshape(-1)
    cells = np.flatnonzero(np.abs(g) > 1e-3 * np.abs(g).max())[::11][:8]
    _fd_check(p, cost, receivers, cells, rel_tol=2e-3)


@pytest.mark.parametrize("name", ["riemann2_64", "fv_diag2_30x26"])
def test_retained_solve_sensitivity_equals_one_shot(name):
    """hfm_run with retainState then hfm_run_sensitivity gives what one hfm_run with the inspection
    keys gives (same solve, deterministic reverse sweep), and matches the reference fixture (a
    Diagonal2 one among them: its per-axis speeds are part of the retained state)."""
    import hamiltonfastmarching_b200 as H
    from conftest import load_golden
    params, ref, _ = load_golden(name)
    keys = ("inspectSensitivity", "inspectSensitivityWeights", "inspectSensitivityLengths")
    base = {k: v for k, v in params.items() if k not in keys and k != "exportActiveNeighs"}
    io = H.HFMIO("RowMajor")
    io.set_dict(dict(base, retainState=1.0, verbosity=0.0))
    io.run()
    for k in keys:
        io.set_array(k, params[k])
    io.run_sensitivity()
    s1 = io.get_array("costSensitivity_0")
    one = H.run(dict(base, **{k: params[k] for k in keys}))["costSensitivity_0"]
    assert np.array_equal(s1, one)
    rs = ref["costSensitivity_0"]
    assert s1.shape == rs.shape
    assert np.max(np.abs(s1 - rs)) <= 1e-8 * np.max(np.abs(rs))
    io2 = H.HFMIO("RowMajor")
    io2.set_dict(dict(base, verbosity=0.0))
    io2.run()
    for k in keys:
        io2.set_array(k, params[k])
    with pytest.raises(H.PyExp):
        io2.run_sensitivity()
