"""seedRadius > 0 (StaticFactoring.hxx:242-346): the library spreads each seed to the cells whose
centre lies within seedRadius cells of it, with values from the model's norm at the seed
(interpolated) and at the cell. The spreading is host work done while the store is read, before
any device work, so it is checked here on the CPU against the reference's spreadedSeeds and
spreadedSeedValues, bit for bit; the GPU solve from the spread seeds is in test_gpu_edges.py."""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as H
from conftest import load_golden

SPREAD = ["spread_riemann2_dual", "spread_riemann3_walls", "spread_isotropic2", "spread_diagonal3", "spread_tti3",
          "spread_tti3_scales", "spread_riemann2_step", "spread_riemann3_step", "spread_isotropic2_step",
          "spread_diagonal3_step"]


@pytest.mark.parametrize("name", SPREAD)
def test_spread_seeds_match_reference(name):
    params, ref, _ = load_golden(name)
    io = H.HFMIO("RowMajor")
    io.set_dict(dict(params, verbosity=0.0))
    try:
        io.run()  # on a machine without a GPU the solve fails after the seeds were spread
    except H.PyExp:
        pass
    np.testing.assert_array_equal(io.get_array("spreadedSeeds"), ref["spreadedSeeds"])
    np.testing.assert_array_equal(io.get_array("spreadedSeedValues"), ref["spreadedSeedValues"])


def test_negative_radius_and_lifted_models_refused():
    params, _, _ = load_golden("spread_tti3")  # seedRadius < 0 on TTI3 (Lag2 reversed offsets)
    with pytest.raises(H.PyExp) as e:
        H.run(dict(params, seedRadius=-2.0, verbosity=0.0))
    assert e.value.code == 3
    p = {"model": "ReedsShepp2", "dims": np.array([8., 8., 8.]), "gridScale": 0.125, "cost": 1.0,
         "seeds": np.array([[0.5, 0.5, 0.0]]), "seedRadius": 2.0, "verbosity": 0.0}
    with pytest.raises(H.PyExp) as e:
        H.run(p)
    assert e.value.code == 3


def test_stencil_step_refusals():
    """seedRadius < 0 on a Riemann model is refused (HFM_ERR_UNSUPPORTED, before any device work)
    with walls, and for a seed whose spread cells reach outside the domain."""
    params, _, _ = load_golden("spread_riemann2_step")
    n = int(params["dims"][0])
    with pytest.raises(H.PyExp) as e:
        H.run(dict(params, walls=np.zeros((n, n)), verbosity=0.0))
    assert e.value.code == 3
    with pytest.raises(H.PyExp) as e:
        H.run(dict(params, seeds=np.array([[0.01, 0.5]]), verbosity=0.0))
    assert e.value.code == 3
