"""TTI3 with static factoring on the GPU (StaticFactoring.hxx with TTI.hpp:160-276): arrival times
within 1e-10 of the reference on the factoring fixtures (a computed factor over a subdomain box, with
distinct grid scales, over the whole domain, and an imported factor with a mask), nAccepted exact;
and, at 32^3 with a radius-8 box, within 1e-10 of the oracle's factored fast marching fed the
factor and spread seeds the library exported."""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as H
from hamiltonfastmarching_b200 import workloads as W
from conftest import load_golden
from oracle import oracle as O
from test_gpu_parity import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["fac_tti3_16_r4", "fac_tti3_14_scales_r5", "fac_tti3_10_whole", "fac_tti3_16_import"])
def test_factored_tti3_matches_reference(name):
    params, ref, _ = load_golden(name)
    out = H.run(dict(params, verbosity=0.0))
    assert rel_err(ref["values"], out["values"]) <= 1e-10
    assert int(out["nAccepted"]) == int(ref["nAccepted"])


def test_factored_tti3_matches_oracle_at_32():
    p = W.tti3_case(32, h=0.01, seed=12)
    p.pop("_vp")
    p.update(factoringRadius=8.0, exportFactoring=1.0, verbosity=0.0)
    out = H.run(p)
    q = {k: v for k, v in p.items() if not k.startswith("factoring") and k != "exportFactoring"}
    q.update(seeds=out["spreadedSeeds"], seedValues=out["spreadedSeedValues"],
             _factor=(out["factoringValues"], out["factoringGradients"], out["factoringIndexShift"]))
    ora = O.tti_solve(q)
    assert rel_err(ora["values"], out["values"]) <= 1e-10
