"""TTI3 on the GPU against the reference (golden fixture) and the C oracle.

Values within 1e-10 relative max-norm of the reference's FP64 values, the reverse first variation
(costSensitivity) within 1e-10 of its max norm.
"""
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


def test_tti_golden_values_and_sensitivity():
    params, ref, _ = load_golden("tti3_16")
    params = dict(params)
    params.pop("exportActiveNeighs", None)
    out = hfm.run(params)
    assert _rel(out["values"], ref["values"]) <= RTOL
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    sens, rs = out["costSensitivity_0"], ref["costSensitivity_0"]
    assert np.max(np.abs(sens - rs)) <= RTOL * np.max(np.abs(rs))
    seeds = ref["seedSensitivity_0"]
    np.testing.assert_allclose(out["seedSensitivity_0"], seeds, rtol=RTOL)


@pytest.mark.parametrize("n,seed", [(40, 5), (28, 6)])
def test_tti_matches_oracle(n, seed):
    p = W.tti3_case(n, h=0.01, seed=seed)
    p.pop("_vp")
    ref = O.tti_solve(p)
    out = hfm.run(p)
    assert _rel(out["values"], ref["values"]) <= RTOL
    assert int(out["nAccepted"]) == ref["nAccepted"]


def test_tti_active_neighs_encoding():
    """activeNeighs of TTI3: the extremum t (negative at an interval endpoint), as the reference
    exports it; flat extrema make the endpoint/interior label and t agree only to rounding on a
    few cells."""
    params, ref, _ = load_golden("tti3_16")
    out = hfm.run(dict(params, exportActiveNeighs=1.0))
    a, b = out["activeNeighs"], ref["activeNeighs"]
    assert np.array_equal(np.isinf(a), np.isinf(b))
    fin = np.isfinite(b)
    assert np.mean(np.abs(np.abs(a[fin]) - np.abs(b[fin])) < 1e-6) > 0.95
    assert np.mean(np.abs(a[fin] - b[fin]) < 1e-6) > 0.9


def test_tti_rejects_what_the_gpu_path_does_not_do():
    p = W.tti3_case(8, h=0.01, seed=1)
    p.pop("_vp")
    for extra, code in (({"nmix": 2.0}, 3), ({"solverPrecision": "float32"}, 3),
                        ({"walls": np.zeros((8, 8, 8))}, 3)):
        with pytest.raises(hfm.PyExp) as e:
            hfm.run(dict(p, **extra))
        assert e.value.code == code
