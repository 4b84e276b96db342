"""Stopping criteria on the GPU (stopAtDistance, nMaxAccepted, stopWhenAnyAccepted,
stopWhenAllAccepted, stopWhenAnyAccepted_Unoriented) against the reference's golden fixtures:
nAccepted exactly (it counts the cell that stopped the run), the same unreached cells, values of the
accepted cells and tentative values of the others within 1e-10 (relative), activeNeighs on more than
99 % of the cells."""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as hfm
from conftest import load_golden

pytestmark = pytest.mark.gpu

GOLDEN = ["stop_riemann2_distance", "stop_riemann2_nmax", "stop_riemann2_any_all", "stop_riemann3_walls_nmax",
          "stop_reedsshepp2_unoriented", "stop_tti3_distance", "stop_tti3_all"]


@pytest.mark.parametrize("name", GOLDEN)
def test_stopping_matches_reference(name):
    params, ref, _ = load_golden(name)
    out = hfm.run(dict(params))
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    a, b = out["values"], ref["values"]
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    assert np.max(np.abs(a[fin] - b[fin])) <= 1e-10 * np.max(np.abs(b[fin]))
    if params["model"] != "TTI3":  # TTI3 activeNeighs hold the extremum t (see test_gpu_tti.py)
        assert np.mean(out["activeNeighs"] == ref["activeNeighs"]) > 0.99


def test_distance_beyond_every_value_accepts_all():
    params, ref, _ = load_golden("stop_riemann2_distance")
    full = hfm.run(dict(params, stopAtDistance=1e9))
    plain = dict(params)
    plain.pop("stopAtDistance")
    out = hfm.run(plain)
    assert int(full["nAccepted"]) == int(out["nAccepted"])
    np.testing.assert_allclose(full["values"], out["values"], rtol=1e-12)


def test_stopping_then_geodesic_from_the_target():
    """A common use: stop once a target is reached, then backtrack the geodesic from it."""
    params, _, _ = load_golden("stop_riemann2_any_all")
    p = dict(params)
    p.pop("stopWhenAllAccepted")
    tgt = np.asarray(p["stopWhenAnyAccepted"])[:1]
    p["stopWhenAnyAccepted"] = tgt
    p["tips"] = tgt
    out = hfm.run(p)
    pts = out["geodesicPoints"]
    assert len(pts) > 2
    np.testing.assert_allclose(pts[0], tgt[0])
