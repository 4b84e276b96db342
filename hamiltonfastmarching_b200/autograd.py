"""Arrival times as a differentiable function of a cost field (torch.autograd).

Forward: the GPU solve of ``params`` with the cost field applied; backward: the reverse first
variation of the reference (``Headers/ExtraAlgorithms/FirstVariation.h:341-385``) run on the GPU
with the incoming gradient as the weights of the inspected points, i.e. one ``inspectSensitivity``
group whose ``costSensitivity_0`` is the vector-Jacobian product.

Cost semantics follow the reference:

* curvature models (ReedsShepp2, ReedsSheppForward2, Elastica2) and Isotropic2/3: ``cost`` is the
  model's cost field (the reference's ``cost`` key, speed = 1/cost); the reference's
  costSensitivity is d(values)/d(cost).
* Diagonal2/3: ``cost`` is the per-axis cost field, shape dims + (ndim,) (speed_i = 1/cost_i), and the
  costSensitivity holds d(values)/d(cost_i).
* Riemann2/Riemann3: ``cost`` is a positive local multiplier rho(x) of the norm, the metric used
  being rho^2 * metric; the reference's costSensitivity is the derivative with respect to a relative
  change of the local norm, so d/d(rho) = costSensitivity / rho.
* TTI3: ``cost`` is a positive local multiplier c(x) of the norm (c = vp_ref / vp for a velocity
  change at fixed anisotropy and tilt): the dual unit ball <l, q> + 1/2 <q, Q q> = 1 becomes
  <l / c^2, q> + 1/2 <q, Q / c^4 q> = 1. The reference's costSensitivity (semi-Lagrangian
  ValueVariation, FirstVariation.h:169-196) is the derivative with respect to c at c = 1; here the
  multiplier is applied to the metric, so d/dc = costSensitivity / c.

Sensitivities are exact for the discrete scheme (piecewise linear in the cost); the gradient is
that of the discrete arrival times.
"""
from __future__ import annotations

from typing import Dict

import numpy as np
import torch

from . import HFMIO

__all__ = ["EikonalSolve", "arrival_times"]

_CURVATURE = ("ReedsShepp2", "ReedsSheppForward2", "Elastica2")
_COST_KEY = _CURVATURE + ("Isotropic2", "Isotropic3", "Diagonal2", "Diagonal3")


def _with_cost(params: Dict, cost: np.ndarray) -> Dict:
    p = {k: v for k, v in params.items() if not k.startswith("_")}
    p.setdefault("arrayOrdering", "RowMajor")
    p["verbosity"] = 0.0
    p["exportValues"] = 1.0
    if p["model"] in _COST_KEY:
        p["cost"] = cost
        p.pop("speed", None)
    elif p["model"] == "TTI3":
        metric = np.array(p["metric"], dtype=np.float64)
        c2 = (cost * cost)[..., None]
        metric[..., 0:2] /= c2
        metric[..., 2:5] /= c2 * c2
        p["metric"] = metric
    else:
        metric = np.asarray(p["metric"], dtype=np.float64)
        p["metric"] = metric * (cost[..., None] ** 2)
    return p


def _cell_centres(params: Dict, idx: np.ndarray) -> np.ndarray:
    """Physical points at the centres of RowMajor linear indices (ReDim(PointFromIndex))."""
    dims = tuple(int(round(d)) for d in np.asarray(params["dims"]).ravel())
    sub = np.stack(np.unravel_index(idx, dims), axis=1).astype(np.float64) + 0.5
    if params["model"] in _CURVATURE:
        h = float(params["gridScale"])
        ds = (np.pi if params.get("projective", 0) else 2 * np.pi) / dims[2] if params["model"] == "ReedsShepp2" \
            else 2 * np.pi / dims[2]
        o = np.asarray(params.get("origin", [0.0, 0.0]), float)
        return np.stack([o[0] + sub[:, 0] * h, o[1] + sub[:, 1] * h, -ds / 2 + sub[:, 2] * ds], axis=1)
    hs = np.asarray(params.get("gridScales", [params.get("gridScale", 1.0)] * len(dims)), float)
    hs = np.broadcast_to(hs, (len(dims),))
    o = np.asarray(params.get("origin", np.zeros(len(dims))), float)
    return o + sub * hs


class EikonalSolve(torch.autograd.Function):
    """values = solve(params, cost); backward through the GPU adjoint. The forward solve keeps its
    device state (retainState), so the backward pass is one reverse sweep, not a second solve."""

    @staticmethod
    def forward(ctx, cost: torch.Tensor, params: Dict):
        c = cost.detach().to("cpu", torch.float64).numpy()
        io = HFMIO("RowMajor")
        io.set_dict(_with_cost(params, c), views=True)
        io.set_scalar("retainState", 1.0)
        io.run()
        values = io.get_array("values")
        ctx.params, ctx.io = params, io
        ctx.save_for_backward(cost)
        return torch.from_numpy(values).to(device=cost.device, dtype=cost.dtype)

    @staticmethod
    def backward(ctx, grad: torch.Tensor):
        (cost,) = ctx.saved_tensors
        params, io = ctx.params, ctx.io
        ctx.io = None  # the device state is released with the store
        c = cost.detach().to("cpu", torch.float64).numpy()
        g = grad.detach().to("cpu", torch.float64).numpy().ravel()
        idx = np.flatnonzero(g)
        if idx.size == 0:
            return torch.zeros_like(cost), None
        io.set_array("inspectSensitivity", _cell_centres(params, idx))
        io.set_array("inspectSensitivityWeights", g[idx])
        io.set_array("inspectSensitivityLengths", np.array([float(idx.size)]))
        io.run_sensitivity()
        sens = io.get_array("costSensitivity_0")
        if params["model"] in _COST_KEY:
            gc = sens
            if gc.shape != c.shape:  # physical (x, y) cost field: sum over the angular axis
                gc = gc.sum(axis=2)
        else:
            gc = sens / c
        return torch.from_numpy(np.array(gc)).to(device=cost.device, dtype=cost.dtype), None


def arrival_times(params: Dict, cost: torch.Tensor) -> torch.Tensor:
    """Differentiable arrival times of ``params`` under the cost field ``cost``."""
    return EikonalSolve.apply(cost, params)
