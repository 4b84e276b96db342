"""Batched solves (hfm_run_batch): many uneven instances in one launch sequence.

Every instance's arrival times are the fixed point of its own local solves (each value is
determined by strictly smaller neighbour values of the same instance), so a batch returns,
instance by instance, what a solve of that instance alone returns, up to rounding: a cell keeps
the smallest value it was computed at, and the order of the computations depends on the batch.
The tests check that equality (1e-12 relative for FP64, 1e-6 for FP32), the FP64 oracle on a
sample of instances, errors that stay with their own instance, and mixed families (grouped into
one launch sequence per family).
"""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as hfm
from hamiltonfastmarching_b200 import workloads as W

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10
FP32_RTOL = 1e-5
SAME = {"float64": 1e-12, "float32": 1e-6}


def _same(a, b, prec="float64"):
    return _rel(a, b) <= SAME[prec]


def _ragged_riemann2(n0, n1, seed, aniso=5.0, n_seeds=1, walls=False):
    n = max(n0, n1)
    p = W.riemann2_case(n, aniso=aniso, seed=seed, n_seeds=n_seeds)
    p["metric"] = np.ascontiguousarray(p["metric"][:n0, :n1])
    p["dims"] = np.array([n0, n1], float)
    h = p["gridScale"]
    rng = np.random.default_rng(seed + 100)
    p["seeds"] = np.stack([rng.uniform(0.1, 0.9, n_seeds) * n0 * h, rng.uniform(0.1, 0.9, n_seeds) * n1 * h], 1)
    if walls:
        w = np.zeros((n0, n1))
        w[n0 // 3, : (2 * n1) // 3] = 1
        w[(2 * n0) // 3, n1 // 3:] = 1
        seeds_ij = np.floor(p["seeds"] / h).astype(int)
        w[seeds_ij[:, 0], seeds_ij[:, 1]] = 0
        p["walls"] = w
    return p


def _alone(p):
    return hfm.run(p)["values"]


def _rel(a, b):
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    return np.max(np.abs(a[fin] - b[fin])) / np.max(np.abs(b[fin]))


def test_batch_riemann2_ragged_equals_alone():
    shapes = [(64, 64), (97, 33), (8, 200), (150, 150), (1, 77), (40, 41), (256, 31)]
    cases = [_ragged_riemann2(a, b, seed=i, aniso=1 + 2 * i, n_seeds=1 + i % 3, walls=(i % 2 == 1))
             for i, (a, b) in enumerate(shapes)]
    out = hfm.run_batch(cases)
    for p, o in zip(cases, out):
        ref = _alone(p)
        assert o["values"].shape == ref.shape
        assert _same(o["values"], ref), _rel(o["values"], ref)
        assert o["nAccepted"] == hfm.run(p)["nAccepted"]


def test_batch_fp32_equals_alone_and_oracle_tolerance():
    from oracle import oracle as O
    cases = []
    for i, (a, b) in enumerate([(96, 96), (50, 130), (128, 64)]):
        p = _ragged_riemann2(a, b, seed=10 + i, aniso=8.0)
        p["solverPrecision"] = "float32"
        cases.append(p)
    out = hfm.run_batch(cases)
    for p, o in zip(cases, out):
        assert _same(o["values"], _alone(p), "float32")
        q = dict(p)
        q.pop("solverPrecision")
        ref = O.solve(q)["values"]
        assert _rel(o["values"], ref) <= FP32_RTOL


def test_batch_curvature_models_equal_alone():
    rs = [W.curvature2_case(n, 24, "ReedsShepp2", seed=20 + n, n_curves=4) for n in (32, 48, 20)]
    el = [W.curvature2_case(n, 16, "Elastica2", seed=30 + n, n_curves=4) for n in (24, 40)]
    cases = [rs[0], el[0], rs[1], el[1], rs[2]]
    out = hfm.run_batch(cases)
    for p, o in zip(cases, out):
        assert _same(o["values"], _alone(p))


def test_batch_mixed_families_and_oracle_sample():
    from oracle import oracle as O
    cases = [
        _ragged_riemann2(70, 90, seed=40),
        W.riemann3_case(24, seed=41, n_spheres=3, n_seeds=2),
        W.curvature2_case(32, 24, "ReedsShepp2", seed=42, n_curves=4),
        _ragged_riemann2(33, 128, seed=43, n_seeds=2),
        W.riemann3_case(20, seed=44, n_spheres=0, n_seeds=1),
    ]
    out = hfm.run_batch(cases)
    for p, o in zip(cases, out):
        assert _same(o["values"], _alone(p))
    for k in (0, 1, 2):  # FP64 oracle on a sample of the instances
        assert _rel(out[k]["values"], O.solve(cases[k])["values"]) <= FP64_RTOL


def test_batch_error_stays_with_its_instance():
    good = [_ragged_riemann2(64, 64, seed=50), _ragged_riemann2(40, 72, seed=51)]
    bad = _ragged_riemann2(48, 48, seed=52)
    bad["metric"] = bad["metric"].copy()
    bad["metric"][10, 10] = [1.0, 2.0, 1.0]  # not positive definite
    missing = {"model": "Riemann2", "arrayOrdering": "RowMajor"}
    out = hfm.run_batch([good[0], bad, missing, good[1]], raise_errors=False)
    assert isinstance(out[1], hfm.PyExp) and out[1].code == 2
    assert isinstance(out[2], hfm.PyExp) and out[2].code == 1
    for p, o in zip(good, (out[0], out[3])):
        assert _same(o["values"], _alone(p))


def test_batch_with_sensitivity_request_runs_it_alone():
    p = _ragged_riemann2(48, 48, seed=60)
    q = dict(p)
    q["inspectSensitivity"] = np.array([[0.1, 0.12]])
    out = hfm.run_batch([p, q])
    ref = hfm.run(q)
    assert _same(out[1]["values"], ref["values"])
    assert _rel(out[1]["costSensitivity_0"], ref["costSensitivity_0"]) <= 1e-10
    assert _same(out[0]["values"], _alone(p))


def test_autotuner_picks_a_valid_schedule_and_values_do_not_change():
    """Tile shape, sweeps and queue policy change the speed, not the fixed point."""
    from hamiltonfastmarching_b200.autotune import Autotuner
    cases = [_ragged_riemann2(n, n, seed=70 + n) for n in (64, 96, 80)]
    for p in cases:
        p["solverPrecision"] = "float32"
    at = Autotuner(repeats=1, device="test")
    res = at.tune(cases, sweeps=1)
    assert np.isfinite(res["seconds"]) and res["seconds"] <= res["default_seconds"]
    assert len(at.trials) >= 8
    for p in cases:
        q = at.apply(p)
        assert "tileShape" in q
        assert _rel(hfm.run(q)["values"], _alone(p)) <= SAME["float32"]
    # a non-default tile shape on each domain kind gives the same values
    for p, shape in ((cases[0], [16, 4]), (W.riemann3_case(24, seed=3, n_spheres=3), [2, 4, 8]),
                     (W.curvature2_case(32, 24, "ReedsShepp2", seed=4, n_curves=4), [2, 2, 16])):
        assert _same(hfm.run(dict(p, tileShape=np.array(shape, float)))["values"], _alone(p),
                     p.get("solverPrecision", "float64"))


def test_batch_tti3_instances_equal_alone():
    cases = []
    for n, seed in ((16, 1), (24, 2), (12, 3)):
        p = W.tti3_case(n, h=0.01, seed=seed)
        p.pop("_vp")
        cases.append(p)
    out = hfm.run_batch(cases)
    for p, o in zip(cases, out):
        assert _same(o["values"], _alone(p))
