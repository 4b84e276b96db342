"""Regenerate the golden fixtures of this directory by running the reference's own FileHFM
executables (``make -C oracle ref`` builds them from the reference sources into ``oracle/_ref``).

    python tests/golden/make_golden.py

Each fixture stores the inputs (hfmIn keys, RowMajor) and the reference outputs: exact float64
``values``, ``activeNeighs``, ``nAccepted``, ``MaxStencilWidth``, ``costSensitivity_0`` /
``seedSensitivity_0`` where an ``inspectSensitivity`` group is given, and for the stencil fixtures
the reference's ``getStencils`` answer (integer offsets exactly; weights as printed, 6 digits).
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.refrun import run_reference  # noqa: E402
from hamiltonfastmarching_b200 import workloads as W  # noqa: E402

def parse_stencils(text: str, ndim: int):
    """Parse the reference's ``stencils`` string into per-point (offsets, weights) arrays.

    The string nests ``{index, {"forward" -> {{diffs}}, "symmetric" -> {{diffs}}}}`` per point,
    each diff being ``{weight, {offset}}``; braces are turned into JSON lists.
    """
    import json
    s = text.replace('"forward" -> ', "").replace('"symmetric" -> ', "")
    s = re.sub(r",\s*}", "}", s).replace("{", "[").replace("}", "]")
    out = []
    for point in json.loads(s):
        _, (fw, sym) = point
        diffs = [d for grp in fw for d in grp] + [d for grp in sym for d in grp]
        out.append((np.array([d[1] for d in diffs], np.int64), np.array([d[0] for d in diffs], float)))
    return out


def random_spd(rng, n, ndim, amax=100.0):
    """Random SPD matrices, anisotropy log-uniform in [1, amax], plus diagonal and tie cases."""
    mats = []
    for i in range(n):
        if ndim == 2:
            th = rng.uniform(0, np.pi)
            a = np.exp(rng.uniform(0, np.log(amax)))
            R = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
            M = R @ np.diag([1.0, a ** -2]) @ R.T
            if i % 17 == 0:
                M = np.diag(rng.uniform(0.5, 2.0, 2))
            if i % 23 == 0:   # exact tie <b_i, M b_j> = 0 on the canonical superbase
                M = np.array([[2.0, -1.0], [-1.0, 2.0]])
            mats.append([M[0, 0], M[0, 1], M[1, 1]])
        else:
            Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
            a1 = np.exp(rng.uniform(0, np.log(amax)))
            a2 = np.exp(rng.uniform(0, np.log(amax)))
            M = Q @ np.diag([1.0, a1 ** -2, a2 ** -2]) @ Q.T
            if i % 17 == 0:
                M = np.diag(rng.uniform(0.5, 2.0, 3))
            if i % 23 == 0:
                M = np.array([[2.0, -1.0, 0.0], [-1.0, 2.0, -1.0], [0.0, -1.0, 2.0]])
            mats.append([M[0, 0], M[0, 1], M[1, 1], M[0, 2], M[1, 2], M[2, 2]])
    return np.array(mats)


def stencil_fixture(name, ndim, side, seed, dual):
    rng = np.random.default_rng(seed)
    dims = (side,) * ndim
    ncell = side ** ndim
    mats = random_spd(rng, ncell, ndim).reshape(dims + (-1,))
    h = 1.0 / side
    params = {
        "model": "Riemann2" if ndim == 2 else "Riemann3",
        "arrayOrdering": "RowMajor",
        "dims": np.array(dims, float),
        "gridScale": h,
        "dualMetric" if dual else "metric": mats,
        "seeds": np.full((1, ndim), 0.5),
        "exportValues": 1.0,
        "exportActiveNeighs": 1.0,
    }
    grid = np.stack(np.meshgrid(*[(np.arange(side) + 0.5) * h] * ndim, indexing="ij"), -1).reshape(-1, ndim)
    params["getStencils"] = grid
    out = run_reference(params)
    assert out["retcode"] == 0, out["log"]
    st = parse_stencils(out["stencils"], ndim)
    assert len(st) == ncell, (len(st), ncell)
    nk = 3 if ndim == 2 else 6
    offs = np.zeros((ncell, nk, ndim), np.int8)
    ws = np.zeros((ncell, nk))
    for i, (o, w) in enumerate(st):
        offs[i] = o
        ws[i] = w
    del params["getStencils"]
    save(name, params, out, stencil_offsets=offs, stencil_weights_6digits=ws)


def save(name, params, out, **extra):
    blob = {}
    for k, v in params.items():
        blob["in_" + k] = np.asarray(v) if not isinstance(v, str) else np.array(v)
    for k in ("values", "activeNeighs", "nAccepted", "MaxStencilWidth", "costSensitivity_0",
              "seedSensitivity_0", "spreadedSeeds", "spreadedSeedValues", "geodesicPoints", "geodesicLengths",
              "geodesicPoints_Unoriented", "geodesicLengths_Unoriented", "geodesicFlow", "valueVariation",
              "factoringValues", "factoringGradients", "factoringIndexShift"):
        if k in out:
            blob["out_" + k] = np.asarray(out[k])
    blob.update(extra)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **blob)
    print(name, {k: getattr(v, "shape", None) for k, v in blob.items() if k.startswith("out_")})


def solve_fixture(name, params, inspect=None):
    params = dict(params)
    params["exportActiveNeighs"] = 1.0
    if inspect is not None:
        pts, wts = inspect
        params["inspectSensitivity"] = np.asarray(pts, float)
        params["inspectSensitivityWeights"] = np.asarray(wts, float)
        params["inspectSensitivityLengths"] = np.array([len(wts)], float)
    out = run_reference(params)
    assert out["retcode"] == 0, out["log"]
    save(name, params, out)


def main():
    rng = np.random.default_rng(1234)
    stencil_fixture("selling2_32", 2, 32, 11, dual=False)
    stencil_fixture("selling2_dual_24", 2, 24, 12, dual=True)
    stencil_fixture("selling3_10", 3, 10, 13, dual=False)
    solve_fixture("riemann2_64", W.riemann2_case(64),
                  (rng.uniform(0.05, 0.95, (6, 2)), rng.uniform(0.5, 2.0, 6)))
    p = W.riemann2_case(48, aniso=10.0, seed=5, n_seeds=3)
    p["seedValues"] = np.array([0.0, 0.1, 0.05])
    solve_fixture("riemann2_48_seeds", p)
    solve_fixture("riemann3_16_walls", W.riemann3_case(16, n_spheres=5, n_seeds=3, rmin=0.1, rmax=0.25),
                  (rng.uniform(0.05, 0.95, (4, 3)), rng.uniform(0.5, 2.0, 4)))
    pts = np.c_[rng.uniform(0.1, 0.9, (4, 2)), rng.uniform(0, 6, (4, 1))]
    solve_fixture("reedsshepp2_32x24", W.curvature2_case(32, 24, "ReedsShepp2", n_curves=6),
                  (pts, rng.uniform(0.5, 2.0, 4)))
    p = W.curvature2_case(24, 16, "ReedsShepp2", seed=7, n_curves=4)
    p["walls"] = (np.random.default_rng(8).uniform(size=(24, 24)) < 0.08).astype(float)
    solve_fixture("reedsshepp2_24x16_walls", p)
    solve_fixture("elastica2_24x16", W.curvature2_case(24, 16, "Elastica2", seed=9, n_curves=5),
                  (pts[:2], rng.uniform(0.5, 2.0, 2)))


def tti_fixtures():
    """TTI3 16^3 (Thomsen parameters, tilted axis) with 6 weighted receivers on the top face."""
    p = W.tti3_case(16, h=0.01, seed=4)
    p.pop("_vp")
    rng = np.random.default_rng(77)
    pts = np.c_[rng.uniform(0.0, 0.16, (6, 2)), np.full((6, 1), 0.005)]
    solve_fixture("tti3_16", p, (pts, rng.uniform(0.5, 2.0, 6)))


def geodesic_fixtures():
    """Discrete geodesics (tips, tips_Unoriented) and the geodesic flow of every model family."""
    rng = np.random.default_rng(2024)
    p = W.riemann2_case(48, aniso=10.0, seed=21)
    p["walls"] = np.zeros((48, 48))
    p["walls"][20, 6:40] = 1.0
    p["tips"] = rng.uniform(0.05, 0.95, (6, 2))
    p["exportGeodesicFlow"] = 1.0
    solve_fixture("geo_riemann2_48_walls", p)
    p = W.riemann3_case(16, n_spheres=3, n_seeds=2, rmin=0.1, rmax=0.2, seed=22)
    p["tips"] = rng.uniform(0.05, 0.95, (4, 3))
    p["exportGeodesicFlow"] = 1.0
    solve_fixture("geo_riemann3_16_walls", p)
    for model, name in (("ReedsShepp2", "geo_reedsshepp2_24x16"), ("Elastica2", "geo_elastica2_24x16")):
        p = W.curvature2_case(24, 16, model, seed=23, n_curves=4)
        p["tips"] = np.c_[rng.uniform(0.1, 0.9, (3, 2)), rng.uniform(0, 6.2, (3, 1))]
        p["tips_Unoriented"] = rng.uniform(0.1, 0.9, (3, 2))
        p["exportGeodesicFlow"] = 1.0
        solve_fixture(name, p)
    p = W.tti3_case(12, h=0.01, seed=24)
    p.pop("_vp")
    p["tips"] = np.c_[rng.uniform(0.0, 0.12, (3, 2)), rng.uniform(0.03, 0.12, (3, 1))]
    p["exportGeodesicFlow"] = 1.0
    solve_fixture("geo_tti3_12", p)


def ode_fixtures():
    """ODE geodesic solver (geodesicSolver = 'ODE') on every family; one Riemann3 tip stalls (the
    reference's failure message)."""
    rng = np.random.default_rng(1)
    n = 48
    m = np.zeros((n, n, 3))
    m[..., 0] = 1 + rng.random((n, n))
    m[..., 2] = 1 + rng.random((n, n))
    m[..., 1] = 0.4 * (rng.random((n, n)) - 0.5)
    walls = np.zeros((n, n))
    walls[20, 5:40] = 1.0
    tips = rng.random((6, 2))
    solve_fixture("ode_riemann2_48_walls", {"model": "Riemann2", "arrayOrdering": "RowMajor", "dims": np.array([n, n], float),
                                            "gridScale": 1.0 / n, "metric": m, "seeds": np.array([[0.5, 0.3]]),
                                            "tips": tips, "walls": walls, "geodesicSolver": "ODE"})
    rng.random((n, n))  # keeps the generator sequence of the fixtures below
    p = W.riemann3_case(16, n_spheres=3, n_seeds=2, rmin=0.1, rmax=0.2, seed=22)
    p["tips"] = rng.uniform(0.05, 0.95, (4, 3))
    p["geodesicSolver"] = "ODE"
    solve_fixture("ode_riemann3_16_walls", p)
    for model, name in (("ReedsShepp2", "ode_reedsshepp2_24x16"), ("Elastica2", "ode_elastica2_24x16")):
        p = W.curvature2_case(24, 16, model, seed=23, n_curves=4)
        p["tips"] = np.c_[rng.uniform(0.1, 0.9, (3, 2)), rng.uniform(0, 6.2, (3, 1))]
        p["tips_Unoriented"] = rng.uniform(0.1, 0.9, (3, 2))
        p["geodesicSolver"] = "ODE"
        solve_fixture(name, p)
    p = W.tti3_case(12, h=0.01, seed=24)
    p.pop("_vp")
    p["tips"] = np.c_[rng.uniform(0.0, 0.12, (3, 2)), rng.uniform(0.03, 0.12, (3, 1))]
    p["geodesicSolver"] = "ODE"
    solve_fixture("ode_tti3_12", p)


def stopping_fixtures():
    """Stopping criteria: the run stops at the first cell popped that meets one (that cell is
    counted in nAccepted but not accepted); the other cells keep their tentative values."""
    p = W.riemann2_case(48, aniso=6.0, seed=5, n_seeds=2)
    solve_fixture("stop_riemann2_distance", dict(p, stopAtDistance=0.12))
    solve_fixture("stop_riemann2_nmax", dict(p, nMaxAccepted=700.0))
    solve_fixture("stop_riemann2_any_all", dict(p, stopWhenAnyAccepted=np.array([[0.9, 0.9], [0.1, 0.8]]),
                                                stopWhenAllAccepted=np.array([[0.7, 0.2], [0.3, 0.35]])))
    p3 = W.riemann3_case(16, n_spheres=3, n_seeds=2, rmin=0.1, rmax=0.2, seed=22)
    solve_fixture("stop_riemann3_walls_nmax", dict(p3, stopAtDistance=0.5, nMaxAccepted=2500.0))
    c = W.curvature2_case(24, 16, "ReedsShepp2", seed=23, n_curves=4)
    solve_fixture("stop_reedsshepp2_unoriented", dict(c, stopWhenAnyAccepted_Unoriented=np.array([[0.8, 0.2]])))
    t = W.tti3_case(14, h=0.01, seed=5)
    t.pop("_vp")
    solve_fixture("stop_tti3_distance", dict(t, stopAtDistance=0.02))
    solve_fixture("stop_tti3_all", dict(t, stopWhenAllAccepted=np.array([[0.02, 0.03, 0.12], [0.11, 0.1, 0.1]])))


def spreading_fixtures():
    """seedRadius > 0: seeds spread to the cells within that many cells, with values from the
    model's norm at the seed and at the cell (spreadedSeeds, spreadedSeedValues)."""
    rng = np.random.default_rng(4)
    p = W.riemann2_case(40, aniso=6.0, seed=5, n_seeds=2)
    m = p.pop("metric")
    solve_fixture("spread_riemann2_dual", dict(p, dualMetric=m, seedRadius=1.5))
    p3 = W.riemann3_case(16, n_spheres=2, n_seeds=2, rmin=0.1, rmax=0.2, seed=22)
    solve_fixture("spread_riemann3_walls", dict(p3, seedRadius=2.0))
    n = 30
    solve_fixture("spread_isotropic2", {"model": "Isotropic2", "arrayOrdering": "RowMajor",
                                        "dims": np.array([n, n], float), "gridScale": 1.0 / n,
                                        "cost": 1 + rng.random((n, n)), "seeds": np.array([[0.31, 0.52], [0.01, 0.5]]),
                                        "seedRadius": 3.0, "exportValues": 1.0})
    solve_fixture("spread_diagonal3", {"model": "Diagonal3", "arrayOrdering": "RowMajor",
                                       "dims": np.array([12, 10, 8], float), "gridScales": np.array([0.1, 0.12, 0.15]),
                                       "speed": 0.5 + rng.random((12, 10, 8, 3)), "seeds": np.array([[0.55, 0.61, 0.33]]),
                                       "seedRadius": 2.2, "exportValues": 1.0})


def dubins_fixtures():
    """Dubins2 (two stencils of 6 forward differences, the value the smaller of their solutions):
    values, activeNeighs (with the bit naming the stencil), nAccepted, MaxStencilWidth; the last
    one also geodesics, the geodesic flow and both first variations."""
    solve_fixture("dubins2_32x24", W.curvature2_case(32, 24, "Dubins2", seed=14, n_curves=6))
    p = W.curvature2_case(24, 16, "Dubins2", seed=15, n_curves=4)
    p["walls"] = (np.random.default_rng(16).uniform(size=(24, 24)) < 0.06).astype(float)
    solve_fixture("dubins2_24x16_walls", p)
    rng = np.random.default_rng(17)
    p = W.curvature2_case(24, 16, "Dubins2", seed=18, n_curves=4)
    p["tips"] = np.c_[rng.uniform(0.1, 0.9, (3, 2)), rng.uniform(0, 6.2, (3, 1))]
    p["tips_Unoriented"] = rng.uniform(0.1, 0.9, (3, 2))
    p["exportGeodesicFlow"] = 1.0
    p["costVariation"] = rng.standard_normal((24, 24, 16, 1))
    p["seedValueVariation"] = np.array([[0.7]])
    pts = np.c_[rng.uniform(0.1, 0.9, (3, 2)), rng.uniform(0, 6, (3, 1))]
    solve_fixture("dubins2_24x16_geo", p, (pts, rng.uniform(0.5, 2.0, 3)))


def stencil_step_spreading_fixtures():
    """seedRadius < 0 on Riemann models: the spread cells plus one step of the reversed stencils."""
    p = W.riemann2_case(40, aniso=6.0, seed=9, n_seeds=1)
    solve_fixture("spread_riemann2_step", dict(p, seeds=np.array([[0.41, 0.57], [0.62, 0.33]]), seedRadius=-1.5))
    p3 = W.riemann3_case(14, n_spheres=1, n_seeds=1, rmin=0.05, rmax=0.08, seed=23)
    p3.pop("walls", None)
    solve_fixture("spread_riemann3_step", dict(p3, seeds=np.array([[0.52, 0.47, 0.55]]), seedRadius=-1.0))
    rng = np.random.default_rng(31)
    n = 30
    solve_fixture("spread_isotropic2_step", {"model": "Isotropic2", "arrayOrdering": "RowMajor",
                                             "dims": np.array([n, n], float), "gridScale": 1.0 / n,
                                             "cost": 1 + rng.random((n, n)), "seeds": np.array([[0.31, 0.52], [0.02, 0.5]]),
                                             "seedRadius": -2.0, "exportValues": 1.0})
    solve_fixture("spread_diagonal3_step", {"model": "Diagonal3", "arrayOrdering": "RowMajor",
                                            "dims": np.array([12, 10, 8], float), "gridScales": np.array([0.1, 0.12, 0.15]),
                                            "speed": 0.5 + rng.random((12, 10, 8, 3)),
                                            "seeds": np.array([[0.55, 0.61, 0.33]]), "seedRadius": -1.2, "exportValues": 1.0})


def tti_spreading_fixtures():
    """seedRadius > 0 on TTI3: the guess is the TTI norm of the metric interpolated at the seed and
    of the metric at the cell (the transform's columns scaled by the grid scales)."""
    p = W.tti3_case(12, h=0.01, seed=6)
    p.pop("_vp")
    solve_fixture("spread_tti3", dict(p, seeds=np.array([[0.043, 0.061, 0.052], [0.021, 0.093, 0.011]]),
                                      seedRadius=2.0))
    q = {k: v for k, v in W.tti3_case(10, h=0.01, seed=7).items() if k not in ("_vp", "gridScale")}
    solve_fixture("spread_tti3_scales", dict(q, gridScales=np.array([0.01, 0.012, 0.009]),
                                             seeds=np.array([[0.0512, 0.0433, 0.0017]]), seedRadius=1.5))


def tti_factoring_fixtures():
    """Static factoring of TTI3 (StaticFactoring.hxx): computed over a subdomain box (radius 4, one
    grid scale; radius 5, three grid scales), over the whole domain (radius < 0), and imported from
    arrays (values, gradients in physical units, mask, index shift). The computed factors are
    exported (exportFactoring), as are the spread seeds (seedRadius defaults to 2 with factoring)."""
    p = W.tti3_case(16, h=0.01, seed=4)
    p.pop("_vp")
    solve_fixture("fac_tti3_16_r4", dict(p, factoringRadius=4.0, exportFactoring=1.0))
    q = {k: v for k, v in W.tti3_case(14, h=0.01, seed=8).items() if k not in ("_vp", "gridScale")}
    q = dict(q, gridScales=np.array([0.01, 0.012, 0.009]), seeds=np.array([[0.071, 0.052, 0.0313]]))
    solve_fixture("fac_tti3_14_scales_r5", dict(q, factoringRadius=5.0, exportFactoring=1.0))
    r = W.tti3_case(10, h=0.01, seed=9)
    r.pop("_vp")
    solve_fixture("fac_tti3_10_whole", dict(r, factoringRadius=-1.0, exportFactoring=1.0))
    # imported: the radius-4 factor of the first case, gradients in physical units, half the box masked
    z = np.load(os.path.join(HERE, "fac_tti3_16_r4.npz"))
    fv, fg, sh = z["out_factoringValues"], z["out_factoringGradients"], z["out_factoringIndexShift"]
    mask = np.ones(fv.shape)
    mask[: fv.shape[0] // 2] = 0.0
    solve_fixture("fac_tti3_16_import", dict(p, factoringValues=fv, factoringGradients=fg / 0.01,
                                             factoringMask=mask, factoringIndexShift=sh))


def diagonal_variation_fixtures():
    """First variations of the Diagonal models, per axis: costSensitivity dims + (D,), costVariation
    dims + (nVar, D)."""
    rng = np.random.default_rng(7)
    for model, dims, name in (("Diagonal2", (30, 26), "fv_diag2_30x26"), ("Diagonal3", (12, 10, 8), "fv_diag3_12x10x8")):
        nd = len(dims)
        walls = np.zeros(dims)
        walls[dims[0] // 2, 2:] = 1.0
        p = {"model": model, "arrayOrdering": "RowMajor", "dims": np.array(dims, float),
             "gridScales": np.linspace(0.02, 0.03, nd), "speed": 0.5 + rng.random(dims + (nd,)), "walls": walls,
             "seeds": np.array([[0.3] * nd, [0.1] * nd]), "seedValues": np.array([0.0, 0.05]),
             "costVariation": rng.standard_normal(dims + (2, nd)), "seedValueVariation": rng.standard_normal((2, 2)),
             "exportValues": 1.0}
        solve_fixture(name, p, (rng.uniform(0.05, 0.25, (3, nd)), np.array([1.0, 2.0, 0.5])))


def variation_fixtures():
    """Forward first variation (costVariation, seedValueVariation -> valueVariation)."""
    rng = np.random.default_rng(2025)
    p = W.riemann2_case(40, aniso=6.0, seed=5, n_seeds=3)
    p["costVariation"] = rng.standard_normal((40, 40, 2))
    p["seedValueVariation"] = rng.standard_normal((2, 3))
    solve_fixture("fwd_riemann2_40_seeds", p)
    p = W.riemann3_case(16, n_spheres=3, n_seeds=2, rmin=0.1, rmax=0.2, seed=9)
    p["costVariation"] = rng.standard_normal((16, 16, 16, 2))
    solve_fixture("fwd_riemann3_16_walls", p)
    for model, name in (("ReedsShepp2", "fwd_reedsshepp2_20x12"), ("Elastica2", "fwd_elastica2_20x12")):
        p = W.curvature2_case(20, 12, model, seed=4, n_curves=3)
        p["costVariation"] = rng.standard_normal((20, 20, 12, 1))
        p["seedValueVariation"] = np.array([[0.7]])
        solve_fixture(name, p)
    p = W.tti3_case(12, h=0.01, seed=2)
    p.pop("_vp")
    p["costVariation"] = rng.standard_normal((12, 12, 12, 2))
    p["seedValueVariation"] = rng.standard_normal((2, 1))
    solve_fixture("fwd_tti3_12", p)


def isotropic_fixtures():
    """Isotropic2 / Isotropic3 and Diagonal2 / Diagonal3 with walls, two seeds, distinct grid scales:
    values, activeNeighs, costSensitivity (isotropic), valueVariation, geodesics and the geodesic flow."""
    rng = np.random.default_rng(2026)
    for model, dims, name in (("Isotropic2", (40, 36), "iso2_40x36_walls"), ("Isotropic3", (14, 12, 10), "iso3_14x12x10_walls")):
        nd = len(dims)
        walls = np.zeros(dims)
        walls[dims[0] // 2, 2:] = 1.0
        p = {"model": model, "arrayOrdering": "RowMajor", "dims": np.array(dims, float),
             "gridScales": np.linspace(0.02, 0.03, nd), "cost": 1 + rng.random(dims), "walls": walls,
             "seeds": np.array([[0.3] * nd, [0.1] * nd]), "seedValues": np.array([0.0, 0.05]),
             "costVariation": rng.standard_normal(dims + (2,)), "tips": rng.uniform(0.0, 0.3, (3, nd)),
             "exportGeodesicFlow": 1.0, "exportValues": 1.0}
        solve_fixture(name, p, (rng.uniform(0.05, 0.25, (3, nd)), np.array([1.0, 2.0, 0.5])))
    # Diagonal2 / Diagonal3: a speed vector per point (no first variation of the multiplier here)
    for model, dims, name in (("Diagonal2", (40, 36), "diag2_40x36_walls"), ("Diagonal3", (14, 12, 10), "diag3_14x12x10_walls")):
        nd = len(dims)
        walls = np.zeros(dims)
        walls[dims[0] // 2, 2:] = 1.0
        p = {"model": model, "arrayOrdering": "RowMajor", "dims": np.array(dims, float),
             "gridScales": np.linspace(0.02, 0.03, nd), "speed": 0.5 + rng.random(dims + (nd,)), "walls": walls,
             "seeds": np.array([[0.3] * nd, [0.1] * nd]), "seedValues": np.array([0.0, 0.05]),
             "seedValueVariation": rng.standard_normal((2, 2)), "tips": rng.uniform(0.0, 0.3, (3, nd)),
             "exportGeodesicFlow": 1.0, "exportValues": 1.0}
        solve_fixture(name, p)


def forward_curvature_fixtures():
    """ReedsSheppForward2 (3 forward differences and 1 symmetric angular one per angle): values,
    activeNeighs, costSensitivity; with walls, geodesics (tips, tips_Unoriented), the geodesic flow
    and a forward variation."""
    rng = np.random.default_rng(2027)
    pts = np.c_[rng.uniform(0.1, 0.9, (4, 2)), rng.uniform(0, 6, (4, 1))]
    solve_fixture("rsf2_32x24", W.curvature2_case(32, 24, "ReedsSheppForward2", seed=11, n_curves=6),
                  (pts, rng.uniform(0.5, 2.0, 4)))
    p = W.curvature2_case(24, 16, "ReedsSheppForward2", seed=12, n_curves=4)
    p["walls"] = (np.random.default_rng(13).uniform(size=(24, 24)) < 0.06).astype(float)
    p["tips"] = np.c_[rng.uniform(0.1, 0.9, (3, 2)), rng.uniform(0, 6.2, (3, 1))]
    p["tips_Unoriented"] = rng.uniform(0.1, 0.9, (3, 2))
    p["exportGeodesicFlow"] = 1.0
    p["costVariation"] = rng.standard_normal((24, 24, 16, 1))
    p["seedValueVariation"] = np.array([[0.7]])
    solve_fixture("rsf2_24x16_walls", p)



def reedsshepp3_fixtures():
    """ReedsShepp3 (Curvature3.h:29-70): primal and dual, projective, each kind of cost field; and
    ReedsSheppForward3 (Curvature3.h:72-107)."""
    solve_fixture("rs3_10x6", W.reedsshepp3_case(10, 6, seed=31))
    solve_fixture("rs3_8x4_dual", W.reedsshepp3_case(8, 4, seed=32, dual=True, cost="full"))
    solve_fixture("rs3_8x4_projective", W.reedsshepp3_case(8, 4, seed=33, projective=True, cost="angular"))
    solve_fixture("rs3_12x6_xi1", W.reedsshepp3_case(12, 6, seed=34, xi=1.0, eps=0.2, cost="constant", n_seeds=2))
    for name, kw in (("rsf3_10x6", dict(seed=35, cost="full")),
                     ("rsf3_8x4_angular", dict(seed=36, cost="angular", xi=1.0, eps=0.3, n_seeds=2))):
        n, nt = (10, 6) if name == "rsf3_10x6" else (8, 4)
        p = W.reedsshepp3_case(n, nt, **kw)
        p["model"] = "ReedsSheppForward3"
        del p["dual"], p["projective"]
        solve_fixture(name, p)
    # seeds given beyond the pole (theta > pi, reflected with phi turned by pi) and an origin
    p = W.reedsshepp3_case(8, 4, seed=38, cost="spatial")
    ds = 2 * np.pi / 8
    p["origin"] = np.array([0.25, -0.5, 0.125])
    p["seeds"] = np.array([[0.8, -0.1, 0.6, np.pi + 0.5 * ds, 0.3], [0.5, 0.2, 0.4, -0.5 * ds, 1.0]])
    p["seedValues"] = np.array([0.0, 0.05])
    solve_fixture("rs3_8x4_pole_seeds", p)
    # getStencils on the sphere bundle: the reference's `stencils` string at a few cells, the poles'
    # classes included
    for name, model in (("rs3_stencils_6x4", "ReedsShepp3"), ("rsf3_stencils_6x4", "ReedsSheppForward3")):
        p = W.reedsshepp3_case(6, 4, seed=37, cost="constant")
        if model != "ReedsShepp3":
            p["model"] = model
            del p["dual"], p["projective"]
        ds = 2 * np.pi / 8
        p["getStencils"] = np.array([[0.5, 0.5, 0.5, 0.5 * ds, 0.0], [0.1, 0.9, 0.3, 3.5 * ds, 5 * ds],
                                     [0.7, 0.2, 0.6, 1.5 * ds, 2 * ds], [0.3, 0.3, 0.3, 2.5 * ds, 7 * ds]])
        out = run_reference(p)
        assert out["retcode"] == 0, out["log"]
        save(name, p, out, ref_stencils=np.array(out["stencils"]))

if __name__ == "__main__":
    # `make_golden.py tti|geodesic|variation|isotropic|ode|stopping|spreading|diagvar|rsf2|ttispread|dubins|
    # spreadstep|factoring|rs3`
    # regenerates only those fixtures
    if sys.argv[1:] == ["tti"]:
        tti_fixtures()
    elif sys.argv[1:] == ["geodesic"]:
        geodesic_fixtures()
    elif sys.argv[1:] == ["variation"]:
        variation_fixtures()
    elif sys.argv[1:] == ["isotropic"]:
        isotropic_fixtures()
    elif sys.argv[1:] == ["ode"]:
        ode_fixtures()
    elif sys.argv[1:] == ["stopping"]:
        stopping_fixtures()
    elif sys.argv[1:] == ["spreading"]:
        spreading_fixtures()
    elif sys.argv[1:] == ["diagvar"]:
        diagonal_variation_fixtures()
    elif sys.argv[1:] == ["rsf2"]:
        forward_curvature_fixtures()
    elif sys.argv[1:] == ["ttispread"]:
        tti_spreading_fixtures()
    elif sys.argv[1:] == ["dubins"]:
        dubins_fixtures()
    elif sys.argv[1:] == ["spreadstep"]:
        stencil_step_spreading_fixtures()
    elif sys.argv[1:] == ["factoring"]:
        tti_factoring_fixtures()
    elif sys.argv[1:] == ["rs3"]:
        reedsshepp3_fixtures()
    else:
        main()
        tti_fixtures()
        geodesic_fixtures()
        variation_fixtures()
        isotropic_fixtures()
        ode_fixtures()
        stopping_fixtures()
        spreading_fixtures()
        diagonal_variation_fixtures()
