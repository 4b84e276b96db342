"""Dubins2 on the GPU (two groups of 6 forward differences per angle, the value the smaller of the
two groups' solutions, Headers/Specializations/Curvature2.h:113-140) against the reference's
fixtures: arrival times within 1e-10, nAccepted and MaxStencilWidth exact, activeNeighs equal
(the group bit included) except at exact ties; on the fixture with first variations and
geodesics, costSensitivity and valueVariation within 1e-10 of their largest entries, seed
sensitivities within 1e-10, geodesics of the same lengths with points within 1e-7 of the domain
size and the flow within 1e-7 (the arrival times differ from the reference's at the 1e-10 level).
"""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as H
from conftest import load_golden
from test_gpu_parity import rel_err, untied_active_differences

pytestmark = pytest.mark.gpu

CASES = ["dubins2_32x24", "dubins2_24x16_walls", "dubins2_24x16_geo"]


@pytest.mark.parametrize("name", CASES)
def test_dubins2_values_and_active_neighbours(name):
    params, ref, _ = load_golden(name)
    out = H.run(dict(params, verbosity=0.0))
    assert rel_err(ref["values"], out["values"]) <= 1e-10
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    assert int(out["MaxStencilWidth"]) == int(ref["MaxStencilWidth"])
    act_ref = ref["activeNeighs"].astype(np.uint64)
    act = out["activeNeighs"].astype(np.uint64)
    untied = untied_active_differences(params, ref["values"], act_ref, act)
    assert not untied, f"activeNeighs differ away from exact ties at cells {untied[:10]}"


def test_dubins2_variations_and_geodesics():
    params, ref, _ = load_golden("dubins2_24x16_geo")
    out = H.run(dict(params, verbosity=0.0))
    for key in ("costSensitivity_0", "valueVariation"):
        a, b = ref[key], out[key]
        assert a.shape == b.shape
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(a)), key
    np.testing.assert_allclose(out["seedSensitivity_0"], ref["seedSensitivity_0"], rtol=1e-10, atol=0)
    for suffix in ("", "_Unoriented"):
        np.testing.assert_array_equal(out["geodesicLengths" + suffix], ref["geodesicLengths" + suffix])
        a, b = out["geodesicPoints" + suffix], ref["geodesicPoints" + suffix]
        assert a.shape == b.shape
        assert np.max(np.abs(a - b)) <= 1e-7 * max(1.0, np.max(np.abs(b)))
    f, g = out["geodesicFlow"], ref["geodesicFlow"]
    fin = np.isfinite(g)
    assert np.array_equal(np.isfinite(f), fin)
    assert np.max(np.abs(f[fin] - g[fin])) <= 1e-7 * np.max(np.abs(g[fin]))


def test_dubins2_fp32_close_to_fp64():
    params, _, _ = load_golden("dubins2_32x24")
    o64 = H.run(dict(params, verbosity=0.0))
    o32 = H.run(dict(params, verbosity=0.0, solverPrecision="float32"))
    assert rel_err(o64["values"], o32["values"]) <= 1e-5
