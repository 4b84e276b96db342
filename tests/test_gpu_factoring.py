"""TTI3 with static factoring on the GPU (StaticFactoring.hxx with TTI.hpp:160-276).

The corrected update u(x + e) + <grad(x), e> + F(x) - F(x + e) is not causal: fast marching takes
it in acceptance order, and a cell can be updated below values accepted before it. Fast marching's
factored result is then not a fixed point of the update at those cells (the oracle's
fmo_tti_prefix_solve finds 6-9 such cells on each reference fixture, where the unfactored result
is a fixed point everywhere), and fixed points of the corrected update are not unique. The
parallel solver iterates the update; what is pinned here:

* on the reference fixtures (a computed factor over a subdomain box, with distinct grid scales,
  over the whole domain, an imported factor with a mask) its arrival times are within 3e-2 of the
  reference's in max-norm relative to the largest value (the oracle's own Jacobi fixed point of
  the same update is 1.4e-3 to 2.1e-2 away), with the same reached set and nAccepted;
* it is a fixed point of the oracle's order-independent form of the update (each neighbour's value
  triggering a solve over the neighbours at or below it, while below the result so far) except at
  a few cells (at most 4, each within 1e-2 of its max-norm), recomputed from the GPU's own values;
* at 32^3 with a radius-4 box, the same two properties against the oracle's factored fast
  marching fed the factor and spread seeds that the library exported.
"""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as H
from hamiltonfastmarching_b200 import workloads as W
from conftest import load_golden
from oracle import oracle as O
from test_factoring import oracle_inputs

pytestmark = pytest.mark.gpu

FIXTURES = ["fac_tti3_16_r4", "fac_tti3_14_scales_r5", "fac_tti3_10_whole", "fac_tti3_16_import"]
FIXED_POINT_RTOL = 1e-2
FIXED_POINT_CELLS = 4
REFERENCE_RTOL = 3e-2


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert np.array_equal(np.isinf(a), np.isinf(b)), "reached sets differ"
    fin = np.isfinite(a)
    return float(np.max(np.abs(a[fin] - b[fin])) / np.max(np.abs(a[fin])))


def _check_fixed_point(v, again):
    fin = np.isfinite(v)
    moved = np.abs(again[fin] - v[fin]) > 1e-12 * np.max(np.abs(v[fin]))
    assert int(moved.sum()) <= FIXED_POINT_CELLS
    assert _rel(v, again) <= FIXED_POINT_RTOL


def _oracle_result_with_values(name, values):
    """The oracle's problem of a fixture (factor, spread seeds) carrying the given values."""
    q, _ = oracle_inputs(name)
    res = O.tti_solve(q)
    res = dict(res, values=np.asarray(values, float).reshape(res["values"].shape))
    return res


@pytest.mark.parametrize("name", FIXTURES)
def test_factored_tti3_is_a_fixed_point_and_close_to_the_reference(name):
    params, ref, _ = load_golden(name)
    out = H.run(dict(params, verbosity=0.0))
    v = out["values"]
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    res = _oracle_result_with_values(name, v)
    again = O.tti_prefix_solve(res)
    _check_fixed_point(v, again)
    assert _rel(ref["values"], v) <= REFERENCE_RTOL


def test_factored_tti3_at_32_fixed_point_and_close_to_oracle():
    p = W.tti3_case(32, h=0.01, seed=12)
    p.pop("_vp")
    p.update(factoringRadius=4.0, exportFactoring=1.0, verbosity=0.0)
    out = H.run(p)
    q = {k: v for k, v in p.items() if not k.startswith("factoring") and k != "exportFactoring"}
    q.update(seeds=out["spreadedSeeds"], seedValues=out["spreadedSeedValues"],
             _factor=(out["factoringValues"], out["factoringGradients"], out["factoringIndexShift"]))
    fm = O.tti_solve(q)
    v = out["values"]
    again = O.tti_prefix_solve(dict(fm, values=v))
    _check_fixed_point(v, again)
    assert _rel(fm["values"], v) <= REFERENCE_RTOL
