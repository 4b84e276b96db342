"""Serving loop (hfm_server_*): continuous batching, memory admission, alone-vs-mix equality.

Each request's fixed point depends only on its own inputs, so a request served in a mix of other
models and sizes must return what it returns alone (asserted within the stated tolerances:
1e-10 relative max-norm for FP64, 1e-5 for FP32).
"""
import threading
import time

import numpy as np
import pytest

import hamiltonfastmarching_b200 as hfm
from hamiltonfastmarching_b200 import workloads as W
from hamiltonfastmarching_b200.serving import Server

pytestmark = pytest.mark.gpu

TOL = {"float64": 1e-10, "float32": 1e-5}


def _rel(a, b):
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    return float(np.max(np.abs(a[fin] - b[fin])) / np.max(np.abs(b[fin])))


def _mix(prec, seed=0):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(10):
        n = int(rng.integers(24, 160))
        reqs.append(W.riemann2_case(n, aniso=float(rng.uniform(1, 10)), seed=seed * 100 + k,
                                    n_seeds=int(rng.integers(1, 5))))
    for k in range(3):
        reqs.append(W.riemann3_case(int(rng.integers(16, 40)), seed=seed * 100 + 20 + k, n_spheres=4,
                                    n_seeds=int(rng.integers(1, 5))))
    for k in range(3):
        reqs.append(W.curvature2_case(int(rng.integers(24, 48)), 24, "ReedsShepp2", seed=seed * 100 + 30 + k,
                                      n_curves=4, n_seeds=int(rng.integers(1, 5))))
    order = rng.permutation(len(reqs))
    reqs = [reqs[i] for i in order]
    for p in reqs:
        p["solverPrecision"] = prec
        p["verbosity"] = 0.0
    return reqs


@pytest.mark.parametrize("prec", ["float64", "float32"])
def test_served_in_mix_equals_alone(prec):
    reqs = _mix(prec)
    alone = [hfm.run(p)["values"] for p in reqs]
    with Server(lanes=2, max_batch=8) as srv:
        tickets = []
        for i, p in enumerate(reqs):  # a burst, then staggered arrivals while batches run
            tickets.append(srv.submit(p))
            if i >= len(reqs) // 2:
                time.sleep(0.002)
        outs = [t.result(timeout=120) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["max_batch"] > 1  # several instances were resident at once
    for o, a in zip(outs, alone):
        assert o["values"].shape == a.shape
        assert _rel(o["values"], a) <= TOL[prec]
        assert o["nAccepted"] == float(np.isfinite(a).sum())


def test_fp32_served_within_tolerance_of_fp64():
    r32 = _mix("float32", seed=1)
    r64 = _mix("float64", seed=1)
    with Server(lanes=2) as srv:
        t32 = [srv.submit(p) for p in r32]
        t64 = [srv.submit(p) for p in r64]
        for a, b in zip(t32, t64):
            assert _rel(a.result(timeout=120)["values"], b.result(timeout=120)["values"]) <= TOL["float32"]


def test_admission_respects_memory_budget():
    reqs = [W.riemann2_case(256, seed=k) for k in range(6)]  # ~10.5 MB estimated each
    budget = 25e6  # at most two of them on the device at a time
    with Server(lanes=3, hbm_budget_bytes=budget) as srv:
        ts = [srv.submit(p) for p in reqs]
        for t in ts:
            t.result(timeout=120)
        st = srv.stats()
        assert st["peak_bytes"] <= budget
        big = W.riemann2_case(1024, seed=9)
        with pytest.raises(hfm.PyExp) as e:
            srv.submit(big)
        assert e.value.code == 6


def test_errors_stay_with_their_request():
    good = [W.riemann2_case(64, seed=k) for k in range(3)]
    bad = W.riemann2_case(64, seed=5)
    bad["metric"] = bad["metric"].copy()
    bad["metric"][3, 3] = [1.0, 2.0, 1.0]
    with Server(lanes=1, max_batch=8) as srv:
        ts = [srv.submit(p) for p in (good[0], bad, good[1], good[2])]
        with pytest.raises(hfm.PyExp) as e:
            ts[1].result(timeout=60)
        assert e.value.code == 2
        for t, p in zip((ts[0], ts[2], ts[3]), good):
            assert _rel(t.result(timeout=60)["values"], hfm.run(p)["values"]) <= TOL["float64"]


def test_concurrent_clients():
    reqs = _mix("float32", seed=2)
    alone = [hfm.run(p)["values"] for p in reqs]
    results = [None] * len(reqs)
    with Server(lanes=2) as srv:
        def client(idx):
            for i in idx:
                results[i] = srv.submit(reqs[i]).result(timeout=120)["values"]
        th = [threading.Thread(target=client, args=(list(range(j, len(reqs), 3)),)) for j in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    for r, a in zip(results, alone):
        assert _rel(r, a) <= TOL["float32"]


def test_small_request_released_before_a_large_one_admitted_earlier():
    """Continuous batching: a small request that arrives while a large one runs joins the running
    solver and is released as soon as its own tiles converge."""
    big = dict(W.riemann3_case(160, seed=3), solverPrecision="float64", verbosity=0.0)
    small = dict(W.riemann2_case(64, seed=4), solverPrecision="float64", verbosity=0.0)
    alone_small = hfm.run(small)["values"]
    alone_big = hfm.run(big)["values"]
    with Server(max_batch=8) as srv:
        tb = srv.submit(big)
        t0 = time.time()
        while srv.stats()["running_batches"] < 1 and time.time() - t0 < 60:  # the big one is resident
            time.sleep(0.0005)
        ts = srv.submit(small)
        out_s, out_b = ts.result(timeout=120), tb.result(timeout=120)
    assert ts.times[2] < tb.times[2], (ts.times, tb.times)
    assert _rel(out_s["values"], alone_small) <= TOL["float64"]
    assert _rel(out_b["values"], alone_big) <= TOL["float64"]


def test_requests_beyond_arrival_times_are_served_in_the_mix():
    """Geodesics, activeNeighs and other models run through the single-solve path between slices."""
    reqs = _mix("float64", seed=3)[:6]
    geo = dict(W.riemann2_case(48, seed=11), tips=np.array([[0.2, 0.3], [0.8, 0.7]]), exportActiveNeighs=1.0,
               verbosity=0.0)
    iso = {"model": "Isotropic2", "arrayOrdering": "RowMajor", "dims": np.array([40.0, 30.0]), "gridScale": 0.025,
           "cost": np.linspace(1.0, 2.0, 1200).reshape(40, 30), "seeds": np.array([[0.5, 0.4]]),
           "exportValues": 1.0, "verbosity": 0.0}
    reqs = reqs[:3] + [geo] + reqs[3:] + [iso]
    alone = [hfm.run(p) for p in reqs]
    with Server(max_batch=8) as srv:
        outs = [t.result(timeout=120) for t in [srv.submit(p) for p in reqs]]
    for o, a in zip(outs, alone):
        assert _rel(o["values"], a["values"]) <= TOL["float64"]
    np.testing.assert_array_equal(outs[3]["activeNeighs"], alone[3]["activeNeighs"])
    np.testing.assert_array_equal(outs[3]["geodesicLengths"], alone[3]["geodesicLengths"])


def test_plain_loop_mode_serves_one_at_a_time():
    reqs = _mix("float32", seed=4)[:5]
    alone = [hfm.run(p)["values"] for p in reqs]
    with Server(max_batch=1) as srv:
        outs = [t.result(timeout=120)["values"] for t in [srv.submit(p) for p in reqs]]
        assert srv.stats()["max_batch"] == 0  # nothing resident: every request through hfm_run
    for o, a in zip(outs, alone):
        assert _rel(o, a) <= TOL["float32"]
