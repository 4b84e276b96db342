"""The C oracle against the reference's golden vectors (CPU only).

The fixtures were produced by the reference's own FileHFM executables
(tests/golden/make_golden.py); the oracle must reproduce them bit for bit.
"""
import numpy as np
import pytest

from conftest import GOLDEN_SOLVES, GOLDEN_STENCILS, load_golden
from oracle import oracle as O


@pytest.mark.parametrize("name", GOLDEN_SOLVES + GOLDEN_STENCILS)
def test_oracle_values_bit_exact(name):
    params, ref, _ = load_golden(name)
    res = O.solve(params)
    a, b = ref["values"], res["values"]
    assert np.array_equal(np.isinf(a), np.isinf(b))
    fin = np.isfinite(a)
    assert np.array_equal(a[fin], b[fin]), "oracle values differ from the reference"
    assert int(ref["nAccepted"]) == res["nAccepted"]
    assert int(ref["MaxStencilWidth"]) == res["MaxStencilWidth"]
    assert np.array_equal(ref["activeNeighs"].ravel().astype(np.uint64), res["activeNeighs"])


@pytest.mark.parametrize("name", [n for n in GOLDEN_SOLVES])
def test_oracle_sensitivity_bit_exact(name):
    params, ref, _ = load_golden(name)
    if "costSensitivity_0" not in ref:
        pytest.skip("fixture has no inspectSensitivity group")
    res = O.solve(params)
    sens, si, sw = O.backward_variation(res, params["inspectSensitivity"], params["inspectSensitivityWeights"])
    assert np.array_equal(ref["costSensitivity_0"], sens)
    seeds = ref["seedSensitivity_0"]
    assert len(seeds) == len(si)
    np.testing.assert_array_equal(seeds[:, -1], sw)


@pytest.mark.parametrize("name", GOLDEN_STENCILS)
def test_oracle_stencils_match_reference(name):
    """Offsets bit-exact against the reference's getStencils export; weights to its 6 printed digits."""
    params, _, extra = load_golden(name)
    ndim = len(params["dims"])
    dual = "dualMetric" in params
    metric = params["dualMetric" if dual else "metric"]
    h = params["gridScale"]
    off, w = O.riemann_stencils(metric, h, dual)
    ref_off = extra["stencil_offsets"].astype(np.int64)
    ref_w = extra["stencil_weights_6digits"]
    np.testing.assert_array_equal(off[..., :ndim].astype(np.int64), ref_off)
    np.testing.assert_allclose(w, ref_w, rtol=5e-6, atol=0)


def test_tti_oracle_matches_reference():
    """TTI3 (semi-Lagrangian, interval-wise Newton over the Selling path): values within 1e-14 and
    the reverse first variation within 1e-12 of the reference executable (the extremum over t is
    found by an iterative search whose last digits depend on the order of operations)."""
    params, ref, _ = load_golden("tti3_16")
    res = O.tti_solve(params)
    a, b = ref["values"], res["values"]
    assert np.array_equal(np.isinf(a), np.isinf(b))
    fin = np.isfinite(a)
    assert np.max(np.abs(a[fin] - b[fin])) <= 1e-14 * np.max(np.abs(a[fin]))
    assert np.mean(a[fin] == b[fin]) > 0.3
    assert int(ref["nAccepted"]) == res["nAccepted"]
    sens, si, sw = O.tti_backward_variation(res, params["inspectSensitivity"], params["inspectSensitivityWeights"])
    rs = ref["costSensitivity_0"]
    assert np.max(np.abs(sens - rs)) <= 1e-12 * np.max(np.abs(rs))
    seeds = ref["seedSensitivity_0"]
    assert len(seeds) == len(si)
    np.testing.assert_allclose(seeds[:, -1], sw, rtol=1e-12)


GOLDEN_GEODESICS = ["geo_riemann2_48_walls", "geo_riemann3_16_walls", "geo_reedsshepp2_24x16", "geo_elastica2_24x16",
                    "geo_tti3_12", "ode_riemann2_48_walls", "ode_riemann3_16_walls", "ode_reedsshepp2_24x16",
                    "ode_elastica2_24x16", "ode_tti3_12", "rsf2_24x16_walls", "dubins2_24x16_geo"]


@pytest.mark.parametrize("name", GOLDEN_GEODESICS)
def test_geodesic_oracle_matches_reference(name):
    """Geodesics (discrete and ODE solvers; tips, tips_Unoriented) and the geodesic flow of the
    oracle against the reference executable: same lengths, points bit for bit (TTI3 within 1e-14 of
    the domain size), flow within 1e-12 of its largest entry."""
    params, ref, _ = load_golden(name)
    res = O.tti_solve(params) if params["model"] == "TTI3" else O.solve(params)
    geo = O.geodesics(res, params)
    for suffix in ("", "_Unoriented"):
        if "geodesicPoints" + suffix not in ref:
            continue
        np.testing.assert_array_equal(geo["geodesicLengths" + suffix], ref["geodesicLengths" + suffix])
        if params["model"] == "TTI3":  # the extremum over t comes from an iterative search
            scale = np.max(np.abs(ref["geodesicPoints" + suffix]))
            assert np.max(np.abs(geo["geodesicPoints" + suffix] - ref["geodesicPoints" + suffix])) <= 1e-14 * scale
        else:
            np.testing.assert_array_equal(geo["geodesicPoints" + suffix], ref["geodesicPoints" + suffix])
        if name != "ode_riemann3_16_walls":  # its last tip stalls, for the reference too
            assert not geo["geodesicFailed" + suffix].any()
    if "geodesicFlow" not in ref:
        return
    flow, rflow = O.geodesic_flow(res), ref["geodesicFlow"]
    fin = np.isfinite(rflow)
    assert np.array_equal(fin, np.isfinite(flow))
    assert np.max(np.abs(flow[fin] - rflow[fin])) <= 1e-12 * np.max(np.abs(rflow[fin]))


GOLDEN_VARIATIONS = ["fwd_riemann2_40_seeds", "fwd_riemann3_16_walls", "fwd_reedsshepp2_20x12", "fwd_elastica2_20x12",
                     "fwd_tti3_12", "rsf2_24x16_walls", "dubins2_24x16_geo"]


@pytest.mark.parametrize("name", GOLDEN_VARIATIONS)
def test_forward_variation_oracle_matches_reference(name):
    """valueVariation (costVariation, seedValueVariation): bit for bit on the Eulerian models,
    within 1e-14 of its max on TTI3."""
    params, ref, _ = load_golden(name)
    res = O.tti_solve(params) if params["model"] == "TTI3" else O.solve(params)
    v, r = O.forward_variation(res, params), ref["valueVariation"]
    assert v.shape == r.shape
    if params["model"] == "TTI3":
        assert np.max(np.abs(v - r)) <= 1e-14 * np.max(np.abs(r))
    else:
        np.testing.assert_array_equal(v, r)


@pytest.mark.parametrize("name", ["iso2_40x36_walls", "iso3_14x12x10_walls", "diag2_40x36_walls",
                                  "diag3_14x12x10_walls"])
def test_isotropic_oracle_matches_reference(name):
    """Isotropic2/3 (one difference per axis, speed multiplier) and Diagonal2/3 (a speed per axis):
    values, activeNeighs, costSensitivity, valueVariation, geodesics and flow bit for bit (points
    within 1e-15)."""
    params, ref, _ = load_golden(name)
    if params["model"] == "TTI3":  # values within 1e-13 (iterative extremum over t)
        res = O.tti_solve(params)
        a, b = res["values"], ref["values"]
        fin = np.isfinite(b)
        assert np.array_equal(np.isfinite(a), fin)
        assert np.max(np.abs(a[fin] - b[fin])) <= 1e-13 * np.max(np.abs(b[fin]))
        assert res["nAccepted"] == int(ref["nAccepted"])
        return
    res = O.solve(params)
    np.testing.assert_array_equal(res["values"], ref["values"])
    np.testing.assert_array_equal(res["activeNeighs"].reshape(res["values"].shape).astype(float), ref["activeNeighs"])
    assert res["nAccepted"] == int(ref["nAccepted"])
    assert res["MaxStencilWidth"] == int(ref["MaxStencilWidth"])
    if "inspectSensitivity" in params:
        sens, _, _ = O.backward_variation(res, params["inspectSensitivity"], params["inspectSensitivityWeights"])
        np.testing.assert_array_equal(sens, ref["costSensitivity_0"])
    np.testing.assert_array_equal(O.forward_variation(res, params), ref["valueVariation"])
    geo = O.geodesics(res, params)
    np.testing.assert_array_equal(geo["geodesicLengths"], ref["geodesicLengths"])
    assert np.max(np.abs(geo["geodesicPoints"] - ref["geodesicPoints"])) <= 1e-15
    fin = np.isfinite(ref["geodesicFlow"])
    np.testing.assert_array_equal(O.geodesic_flow(res)[fin], ref["geodesicFlow"][fin])


GOLDEN_STOPPING = ["stop_riemann2_distance", "stop_riemann2_nmax", "stop_riemann2_any_all", "stop_riemann3_walls_nmax",
                   "stop_reedsshepp2_unoriented", "stop_tti3_distance", "stop_tti3_all"]


@pytest.mark.parametrize("name", GOLDEN_STOPPING)
def test_stopping_criteria_oracle_matches_reference(name):
    """stopAtDistance, nMaxAccepted, stopWhenAny/AllAccepted (and _Unoriented): values (accepted
    and tentative), activeNeighs and nAccepted bit for bit."""
    params, ref, _ = load_golden(name)
    if params["model"] == "TTI3":  # values within 1e-13 (iterative extremum over t)
        res = O.tti_solve(params)
        a, b = res["values"], ref["values"]
        fin = np.isfinite(b)
        assert np.array_equal(np.isfinite(a), fin)
        assert np.max(np.abs(a[fin] - b[fin])) <= 1e-13 * np.max(np.abs(b[fin]))
        assert res["nAccepted"] == int(ref["nAccepted"])
        return
    res = O.solve(params)
    np.testing.assert_array_equal(res["values"], ref["values"])
    np.testing.assert_array_equal(res["activeNeighs"].reshape(res["values"].shape).astype(float), ref["activeNeighs"])
    assert res["nAccepted"] == int(ref["nAccepted"])


@pytest.mark.parametrize("name", ["fv_diag2_30x26", "fv_diag3_12x10x8"])
def test_diagonal_first_variations_oracle_matches_reference(name):
    """Diagonal models: the reverse (costSensitivity, one component per axis) and forward
    (costVariation with one component per axis) first variations bit for bit."""
    params, ref, _ = load_golden(name)
    res = O.solve(params)
    sens, _, _ = O.backward_variation(res, params["inspectSensitivity"], params["inspectSensitivityWeights"])
    np.testing.assert_array_equal(sens, ref["costSensitivity_0"])
    np.testing.assert_array_equal(O.forward_variation(res, params), ref["valueVariation"])


def test_rsf2_exact_angular_tie_moves_one_cell():
    """ReedsSheppForward2 fixture: the cells whose angular neighbours (offset (0,0,-1) and its
    opposite) hold exactly equal values. The reference took the -e side on one of them; with that
    tie moved to the +e side (the GPU solver's rule) the forward variation of the oracle differs
    from the reference's on that one cell, and with the reference's activeNeighs on none."""
    params, ref, _ = load_golden("rsf2_24x16_walls")
    u = ref["values"]
    act = ref["activeNeighs"].astype(np.uint64)
    plus, minus = np.roll(u, 1, axis=2), np.roll(u, -1, axis=2)
    tie = np.isfinite(u) & np.isfinite(plus) & (plus == minus)
    took_minus = tie & (((act >> np.uint64(4)) & np.uint64(1)) == 1)
    assert int(took_minus.sum()) == 1
    moved = act.copy()
    moved[took_minus] = (moved[took_minus] & ~np.uint64(1 << 4)) | np.uint64(1 << 3)
    res = {"values": np.ascontiguousarray(u), "activeNeighs": np.ascontiguousarray(moved.ravel()),
           "problem": O.Problem(params)}
    r = ref["valueVariation"]
    far = np.abs(O.forward_variation(res, params) - r) > 1e-8 * np.max(np.abs(r))
    assert int(far.sum()) == 1
    res["activeNeighs"] = np.ascontiguousarray(act.ravel())
    np.testing.assert_array_equal(O.forward_variation(res, params), r)


@pytest.mark.parametrize("name", ["spread_tti3", "spread_tti3_scales"])
def test_tti_oracle_from_spread_seeds_matches_reference(name):
    """TTI3 solved from the reference's spreadedSeeds / spreadedSeedValues: the reference's values
    within 1e-14 (relative) and its nAccepted, also with distinct grid scales per axis, where the
    transform's scaling axis matters."""
    params, ref, _ = load_golden(name)
    q = {k: v for k, v in params.items() if k != "seedRadius"}
    q["seeds"], q["seedValues"] = ref["spreadedSeeds"], ref["spreadedSeedValues"]
    res = O.tti_solve(q)
    a, b = res["values"], ref["values"]
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    assert np.max(np.abs(a[fin] - b[fin])) <= 1e-14 * np.max(np.abs(b[fin]))
    assert res["nAccepted"] == int(ref["nAccepted"])


@pytest.mark.parametrize("name", ["dubins2_32x24", "dubins2_24x16_walls", "dubins2_24x16_geo"])
def test_dubins2_oracle_bit_exact(name):
    """Dubins2 (two stencils of 6 forward differences, the value the smaller of their solutions):
    values, activeNeighs with the bit naming the stencil, nAccepted, MaxStencilWidth and the
    reverse first variation (Recompute on the named stencil) as the reference's, bit for bit."""
    params, ref, _ = load_golden(name)
    res = O.solve(params)
    a, b = ref["values"], res["values"]
    assert np.array_equal(np.isinf(a), np.isinf(b))
    fin = np.isfinite(a)
    assert np.array_equal(a[fin], b[fin])
    assert int(ref["nAccepted"]) == res["nAccepted"]
    assert int(ref["MaxStencilWidth"]) == res["MaxStencilWidth"]
    assert np.array_equal(ref["activeNeighs"].ravel().astype(np.uint64), res["activeNeighs"])
    if "costSensitivity_0" in ref:
        sens, _, sw = O.backward_variation(res, params["inspectSensitivity"], params["inspectSensitivityWeights"])
        assert np.array_equal(ref["costSensitivity_0"], sens)
        np.testing.assert_array_equal(ref["seedSensitivity_0"][:, -1], sw)
