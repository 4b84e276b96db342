"""Dubins2 on the GPU (two groups of 6 forward differences per angle, the value the smaller of the
two groups' solutions, Headers/Specializations/Curvature2.h:113-140) against the reference's
fixtures: arrival times within 1e-10, nAccepted and MaxStencilWidth exact, activeNeighs equal
(the group bit included) except at exact ties. First variations and geodesics of Dubins2 are
refused (HFM_ERR_UNSUPPORTED): an illegal memory access was met twice on the fixture that has
them, and its cause is not found.
"""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as H
from conftest import load_golden
from test_gpu_parity import rel_err, untied_active_differences

pytestmark = pytest.mark.gpu

CASES = ["dubins2_32x24", "dubins2_24x16_walls", "dubins2_24x16_geo"]
# inputs of the geodesic/variation fixture that the GPU path refuses for Dubins2
GEO_KEYS = ("tips", "tips_Unoriented", "exportGeodesicFlow", "costVariation", "seedValueVariation",
            "inspectSensitivity", "inspectSensitivityWeights", "inspectSensitivityLengths")


@pytest.mark.parametrize("name", CASES)
def test_dubins2_values_and_active_neighbours(name):
    params, ref, _ = load_golden(name)
    params = {k: v for k, v in params.items() if k not in GEO_KEYS}
    out = H.run(dict(params, verbosity=0.0))
    assert rel_err(ref["values"], out["values"]) <= 1e-10
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    assert int(out["MaxStencilWidth"]) == int(ref["MaxStencilWidth"])
    act_ref = ref["activeNeighs"].astype(np.uint64)
    act = out["activeNeighs"].astype(np.uint64)
    untied = untied_active_differences(params, ref["values"], act_ref, act)
    assert not untied, f"activeNeighs differ away from exact ties at cells {untied[:10]}"


def test_dubins2_variations_and_geodesics_are_refused():
    """First variations and geodesics of Dubins2 are refused before any GPU work (an illegal memory
    access was met on this fixture and its cause is not found)."""
    params, _, _ = load_golden("dubins2_24x16_geo")
    for key in ("inspectSensitivity", "costVariation", "tips", "tips_Unoriented", "exportGeodesicFlow"):
        q = {k: v for k, v in params.items() if k not in GEO_KEYS or k == key or
             (key == "inspectSensitivity" and k.startswith("inspectSensitivity"))}
        with pytest.raises(H.PyExp) as e:
            H.run(dict(q, verbosity=0.0))
        assert e.value.code == 3


def test_dubins2_fp32_close_to_fp64():
    params, _, _ = load_golden("dubins2_32x24")
    o64 = H.run(dict(params, verbosity=0.0))
    o32 = H.run(dict(params, verbosity=0.0, solverPrecision="float32"))
    assert rel_err(o64["values"], o32["values"]) <= 1e-5
