"""Static factoring of TTI3 (Headers/ExtraAlgorithms/Implementation/StaticFactoring.hxx) on the CPU.

* The oracle's fast marching with the order-1 factoring correction, fed the reference's own factor
  (exported with exportFactoring, or the imported arrays) and spread seeds, reproduces the
  reference's arrival times.
* The library's factor, computed on the host while the store is read (the TTI norm at the seed and
  its gradient), equals the reference's exported factoringValues / factoringGradients /
  factoringIndexShift bit for bit, and the seeds it spreads (seedRadius defaults to 2 with
  factoring) equal the reference's spreadedSeeds. On a machine without a GPU the run fails after
  these host steps, which is all this file needs.
"""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as H
from conftest import load_golden
from oracle import oracle as O

COMPUTED = ["fac_tti3_16_r4", "fac_tti3_14_scales_r5", "fac_tti3_10_whole"]


def oracle_inputs(name):
    params, ref, _ = load_golden(name)
    q = {k: v for k, v in params.items() if not k.startswith("factoring") and k not in ("exportFactoring",)}
    q["seeds"] = ref["spreadedSeeds"]
    q["seedValues"] = ref["spreadedSeedValues"]
    if "factoringValues" in params:  # imported: gradients given in physical units, adimensionized
        hs = np.asarray(params.get("gridScales", [params.get("gridScale")] * 3), float)
        fg = params["factoringGradients"] * hs
        q["_factor"] = (params["factoringValues"], fg, params.get("factoringIndexShift"))
        mask = params.get("factoringMask")
        if mask is not None:
            q["_factor_mask"] = mask
    else:
        q["_factor"] = (ref["factoringValues"], ref["factoringGradients"], ref.get("factoringIndexShift"))
    return q, ref


@pytest.mark.parametrize("name", COMPUTED + ["fac_tti3_16_import"])
def test_oracle_factored_fast_marching_matches_reference(name):
    q, ref = oracle_inputs(name)
    out = O.tti_solve(q)
    a, b = ref["values"], out["values"]
    assert np.array_equal(np.isinf(a), np.isinf(b))
    fin = np.isfinite(a)
    assert np.max(np.abs(a[fin] - b[fin])) <= 1e-14 * np.max(np.abs(a[fin]))
    assert out["nAccepted"] == int(ref["nAccepted"])


def _host_outputs(params):
    io = H.HFMIO("RowMajor")
    io.set_dict(dict(params, verbosity=0.0))
    try:
        io.run()  # without a GPU the solve fails after the factor and the seeds were set up
    except H.PyExp:
        pass
    return io


@pytest.mark.parametrize("name", COMPUTED)
def test_host_factor_matches_reference_export(name):
    params, ref, _ = load_golden(name)
    io = _host_outputs(params)
    np.testing.assert_array_equal(io.get_array("factoringValues"), ref["factoringValues"])
    np.testing.assert_array_equal(io.get_array("factoringGradients"), ref["factoringGradients"])
    if "factoringIndexShift" in ref:
        np.testing.assert_array_equal(io.get_array("factoringIndexShift"), ref["factoringIndexShift"])
    np.testing.assert_array_equal(io.get_array("spreadedSeeds"), ref["spreadedSeeds"])
    np.testing.assert_array_equal(io.get_array("spreadedSeedValues"), ref["spreadedSeedValues"])


def test_factoring_argument_errors():
    params, _, _ = load_golden("fac_tti3_16_r4")
    with pytest.raises(H.PyExp) as e:  # two seeds for a computed factor
        H.run(dict(params, seeds=np.array([[0.05, 0.05, 0.005], [0.1, 0.1, 0.005]]), verbosity=0.0))
    assert e.value.code == 2
    with pytest.raises(H.PyExp) as e:  # both import and compute
        H.run(dict(params, factoringValues=np.zeros((2, 2, 2)), verbosity=0.0))
    assert e.value.code == 2
    p = {"model": "Riemann2", "dims": np.array([8.0, 8.0]), "gridScale": 0.125, "metric": np.array([1.0, 0.0, 1.0]),
         "seeds": np.array([[0.5, 0.5]]), "factoringRadius": 3.0, "verbosity": 0.0}
    with pytest.raises(H.PyExp) as e:  # Eulerian models: refused before any device work
        H.run(p)
    assert e.value.code == 3


@pytest.mark.parametrize("name", COMPUTED + ["fac_tti3_16_import"])
def test_factored_fast_marching_is_order_dependent(name):
    """The corrected update is not causal: fast marching's factored result is not a fixed point of
    the order-independent update at a few cells (the unfactored result is one everywhere), and the
    Jacobi fixed point of that update stays within 3e-2 of the reference (relative max-norm)."""
    q, ref = oracle_inputs(name)
    res = O.tti_solve(q)
    v = res["values"]
    fin = np.isfinite(v)
    again = O.tti_prefix_solve(res)
    moved = int(np.sum(again[fin] != v[fin]))
    assert 0 < moved <= 16
    plain = dict(q)
    plain.pop("_factor", None)
    plain.pop("_factor_mask", None)
    r0 = O.tti_solve(plain)
    assert np.array_equal(O.tti_prefix_solve(r0), r0["values"])
    fp = O.tti_prefix_fixed_point(res)
    a = ref["values"]
    assert np.max(np.abs(fp[fin] - a[fin])) / np.max(np.abs(a[fin])) <= 3e-2
