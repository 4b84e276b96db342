"""Isotropic2/3 and Diagonal2/3 on the GPU against the reference's golden fixtures: values within 1e-10
(relative), activeNeighs on > 99 % of cells, nAccepted and MaxStencilWidth exactly, the reverse
and forward first variations within 1e-8 of their largest entry, geodesics with the same lengths
and points within 1e-7 of the domain size."""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as hfm
from conftest import load_golden
from hamiltonfastmarching_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["iso2_40x36_walls", "iso3_14x12x10_walls", "diag2_40x36_walls",
                                  "diag3_14x12x10_walls"])
@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_isotropic_golden(name, precision):
    params, ref, _ = load_golden(name)
    out = hfm.run(dict(params, solverPrecision=precision))
    a, b = out["values"], ref["values"]
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    tol = 1e-10 if precision == "float64" else 1e-5
    assert np.max(np.abs(a[fin] - b[fin])) <= tol * np.max(np.abs(b[fin]))
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    assert int(out["MaxStencilWidth"]) == int(ref["MaxStencilWidth"])
    if precision == "float32":
        return
    assert np.mean(out["activeNeighs"] == ref["activeNeighs"]) > 0.99
    for key in ("costSensitivity_0", "valueVariation"):
        if key in ref:
            assert np.max(np.abs(out[key] - ref[key])) <= 1e-8 * np.max(np.abs(ref[key])), key
    np.testing.assert_array_equal(out["geodesicLengths"], ref["geodesicLengths"])
    assert np.max(np.abs(out["geodesicPoints"] - ref["geodesicPoints"])) <= 1e-7
    f, g = out["geodesicFlow"], ref["geodesicFlow"]
    ok = np.isfinite(g)
    assert np.max(np.abs(f[ok] - g[ok])) <= 1e-8 * np.max(np.abs(g[ok]))


def test_isotropic3_matches_oracle_at_64():
    rng = np.random.default_rng(9)
    n = 64
    p = {"model": "Isotropic3", "arrayOrdering": "RowMajor", "dims": np.array([n, n, n], float),
         "gridScale": 1.0 / n, "speed": 0.5 + rng.random((n, n, n)), "seeds": rng.uniform(0.1, 0.9, (3, 3)),
         "exportValues": 1.0, "verbosity": 0.0}
    ref = O.solve(p)
    out = hfm.run(p)
    assert np.max(np.abs(out["values"] - ref["values"])) <= 1e-10 * np.max(ref["values"])
    assert int(out["nAccepted"]) == ref["nAccepted"]


@pytest.mark.parametrize("name", ["fv_diag2_30x26", "fv_diag3_12x10x8"])
def test_diagonal_first_variations_match_reference(name):
    """Diagonal models: costSensitivity (one component per axis) and valueVariation (a cost
    variation with one component per axis) within 1e-8 of the reference's largest entry."""
    params, ref, _ = load_golden(name)
    out = hfm.run(dict(params))
    for key in ("costSensitivity_0", "valueVariation"):
        a, b = out[key], ref[key]
        assert a.shape == b.shape, key
        assert np.max(np.abs(a - b)) <= 1e-8 * np.max(np.abs(b)), key
