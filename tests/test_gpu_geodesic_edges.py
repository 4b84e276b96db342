"""Edge cases of geodesic backtracking and stopping criteria on the GPU, each checked against the
oracle run on the GPU's own arrival times (or against the reference semantics stated inline):
tips outside the domain, inside a wall, on a seed, on the boundary; the ODE solver on the same
tips; stopping criteria whose targets are unreachable or beyond the number of reached cells."""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as hfm
from hamiltonfastmarching_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _case():
    p = W.riemann2_case(64, aniso=5.0, seed=17, seed_points=np.array([[0.5, 0.5]]))
    walls = np.zeros((64, 64))
    walls[20:24, 10:50] = 1.0
    p["walls"] = walls
    return p


TIPS = np.array([[1.5, 0.5],          # outside the domain: the geodesic is the tip alone
                 [-0.2, 0.3],
                 [0.3, 22.0 / 64],    # inside the wall band
                 [0.5, 0.5],          # on the seed
                 [0.0, 0.0],          # corner
                 [0.999, 0.5]])       # last column


@pytest.mark.parametrize("solver", ["Discrete", "ODE"])
def test_edge_tips_match_oracle(solver):
    p = dict(_case(), tips=TIPS, geodesicSolver=solver, exportValues=1.0, exportActiveNeighs=1.0, verbosity=0.0)
    out = hfm.run(p)
    res = {"values": np.ascontiguousarray(out["values"]),
           "activeNeighs": np.ascontiguousarray(out["activeNeighs"].astype(np.uint64).ravel()),
           "problem": O.Problem(p)}
    geo = O.geodesics(res, p)
    np.testing.assert_array_equal(out["geodesicLengths"], geo["geodesicLengths"])
    assert np.max(np.abs(out["geodesicPoints"] - geo["geodesicPoints"])) <= 1e-11
    # tips outside the domain give a geodesic of one point, the tip itself
    assert out["geodesicLengths"][0] == 1 and out["geodesicLengths"][1] == 1
    np.testing.assert_allclose(out["geodesicPoints"][0], TIPS[0])


def test_stopping_edge_cases_match_oracle():
    base = _case()
    cases = [dict(base, nMaxAccepted=1e9),                                   # more than reached: no stop
             dict(base, nMaxAccepted=1.0),                                   # stops on the seed itself
             dict(base, stopWhenAllAccepted=np.array([[0.3, 22.0 / 64], [0.9, 0.9]])),  # a wall target
             dict(base, stopWhenAnyAccepted=np.array([[0.3, 22.0 / 64], [0.9, 0.9]])),
             dict(base, stopAtDistance=-1.0)]                                # stops at the first cell
    for p in cases:
        out = hfm.run(dict(p, exportValues=1.0, verbosity=0.0))
        ref = O.solve(p)
        assert int(out["nAccepted"]) == ref["nAccepted"], {k: p[k] for k in p if k.startswith(("stop", "nMax"))}
        a, b = out["values"], ref["values"]
        fin = np.isfinite(b)
        assert np.array_equal(np.isfinite(a), fin)
        if fin.any():
            assert np.max(np.abs(a[fin] - b[fin])) <= 1e-10 * max(1.0, np.max(np.abs(b[fin])))


@pytest.mark.parametrize("solver", ["Discrete", "ODE"])
def test_bypass_from_previous_values(solver):
    """values and activeNeighs of a previous run given back (the reference's bypass of the solve,
    HFMInterface.hxx:399-427): the geodesics equal those computed in the run itself."""
    p = dict(_case(), exportValues=1.0, exportActiveNeighs=1.0, verbosity=0.0)
    tips = np.array([[0.9, 0.1], [0.15, 0.85], [0.6, 0.95]])
    first = hfm.run(dict(p, tips=tips, geodesicSolver=solver))
    q = {k: v for k, v in p.items() if k not in ("seeds", "exportActiveNeighs")}
    again = hfm.run(dict(q, values=np.array(first["values"]), activeNeighs=np.array(first["activeNeighs"]),
                         tips=tips, geodesicSolver=solver))
    np.testing.assert_array_equal(again["geodesicLengths"], first["geodesicLengths"])
    np.testing.assert_array_equal(again["geodesicPoints"], first["geodesicPoints"])
    np.testing.assert_array_equal(again["values"], first["values"])
