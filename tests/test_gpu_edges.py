"""Edge cases of the drop-in, on the GPU against the oracle or the reference's behaviour: seeds
outside the domain, colliding seeds, no seeds, single-row grids, invalid (NaN) metrics, and
full-size instances of the benchmark configurations (Riemann2 1024^2, ReedsShepp2 128^2 x 60)."""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as hfm
from hamiltonfastmarching_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _rel(a, b):
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    if not fin.any():
        return 0.0
    return float(np.max(np.abs(a[fin] - b[fin])) / max(np.max(np.abs(b[fin])), 1e-300))


def test_seed_outside_domain_is_ignored_and_colliding_seeds_keep_the_first():
    p = W.riemann2_case(40, seed=3)
    q = dict(p, seeds=np.array([[0.5, 0.5], [1.7, 0.2], [0.5, 0.5001]]),
             seedValues=np.array([0.0, 1.0, 0.3]))
    out, ref = hfm.run(q)["values"], O.solve(q)["values"]
    assert _rel(out, ref) <= RTOL
    assert _rel(out, hfm.run(dict(p, seeds=np.array([[0.5, 0.5]])))["values"]) <= 1e-12


def test_no_seed_returns_no_values():
    p = W.riemann2_case(16)
    p["seeds"] = np.zeros((0, 2))
    out = hfm.run(p)
    assert "values" not in out


def test_single_row_and_single_cell_grids():
    for dims in ((1, 50), (50, 1), (1, 1)):
        n = max(dims)
        p = W.riemann2_case(n, seed=4)
        p["metric"] = np.ascontiguousarray(p["metric"][:dims[0], :dims[1]])
        p["dims"] = np.array(dims, float)
        p["seeds"] = np.array([[0.5 / n, 0.5 / n]])
        assert _rel(hfm.run(p)["values"], O.solve(p)["values"]) <= RTOL


def test_nan_metric_is_an_error():
    p = W.riemann2_case(16)
    p["metric"] = p["metric"].copy()
    p["metric"][2, 3, 0] = np.nan
    with pytest.raises(hfm.PyExp) as e:
        hfm.run(p)
    assert e.value.code == 2


def test_full_size_riemann2_1024_matches_oracle():
    p = W.riemann2_case(1024, aniso=5.0, seed=0)
    assert _rel(hfm.run(p)["values"], O.solve(p, with_active=False)["values"]) <= RTOL


def test_full_size_reedsshepp2_128x60_matches_oracle():
    p = W.curvature2_case(128, 60, "ReedsShepp2", seed=2)
    assert _rel(hfm.run(p)["values"], O.solve(p, with_active=False)["values"]) <= RTOL


@pytest.mark.parametrize("name", ["spread_riemann2_dual", "spread_riemann3_walls", "spread_isotropic2",
                                  "spread_diagonal3"])
def test_spread_seeds_solve_matches_reference(name):
    """Solve from seeds spread by seedRadius: values within 1e-10 of the reference's."""
    from conftest import load_golden
    params, ref, _ = load_golden(name)
    out = hfm.run(dict(params))
    a, b = out["values"], ref["values"]
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    assert np.max(np.abs(a[fin] - b[fin])) <= 1e-10 * np.max(np.abs(b[fin]))
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
