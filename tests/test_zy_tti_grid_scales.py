"""TTI3 on the GPU with seeds spread by seedRadius and with distinct grid scales per axis: values
within 1e-10 (relative) of the reference's, and of the oracle's at a larger size, same nAccepted."""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as hfm
from conftest import load_golden
from hamiltonfastmarching_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _rel(a, b):
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    return float(np.max(np.abs(a[fin] - b[fin])) / np.max(np.abs(b[fin])))


@pytest.mark.parametrize("name", ["spread_tti3", "spread_tti3_scales"])
def test_tti_spread_seeds_solve_matches_reference(name):
    params, ref, _ = load_golden(name)
    out = hfm.run(dict(params, verbosity=0.0))
    np.testing.assert_array_equal(out["spreadedSeedValues"], ref["spreadedSeedValues"])
    assert _rel(out["values"], ref["values"]) <= RTOL
    assert int(out["nAccepted"]) == int(ref["nAccepted"])


def test_tti_distinct_grid_scales_match_oracle():
    p = {k: v for k, v in W.tti3_case(24, h=0.01, seed=8).items() if k not in ("_vp", "gridScale")}
    p["gridScales"] = np.array([0.01, 0.013, 0.008])
    ref = O.tti_solve(p)
    out = hfm.run(dict(p, verbosity=0.0))
    assert _rel(out["values"], ref["values"]) <= RTOL
    assert int(out["nAccepted"]) == ref["nAccepted"]
