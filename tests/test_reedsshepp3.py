"""ReedsShepp3 and ReedsSheppForward3 on R^3 x S^2 (Headers/Specializations/Curvature3.h:29-107):
the oracle against the reference's own FileHFM_ReedsShepp3 / FileHFM_ReedsSheppForward3 outputs
(CPU only).

The fixtures (tests/golden/make_golden.py rs3) cover the primal and dual models, the projective
bundle (nphi = 4 ntheta), and a cost field over (x, y, z), over (theta, phi), over the whole grid
and constant; ReedsSheppForward3 with a full and an angular cost; seeds given beyond the poles
with an origin. The oracle reproduces values, activeNeighs, nAccepted and MaxStencilWidth bit for
bit: the shared stencils (one per (theta, phi)), the Sphere2 periodization of theta and phi
(PeriodicGrid.hxx:120-160) and the reversed offsets taken from each class's centre point
(HFM_StencilShare.hxx:132-181).
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O

RS3_FIXTURES = ["rs3_10x6", "rs3_8x4_dual", "rs3_8x4_projective", "rs3_12x6_xi1", "rsf3_10x6", "rsf3_8x4_angular",
                "rs3_8x4_pole_seeds"]


@pytest.mark.parametrize("name", RS3_FIXTURES)
def test_rs3_oracle_bit_exact(name):
    params, ref, _ = load_golden(name)
    res = O.rs3_solve(params)
    a, b = ref["values"], res["values"]
    assert np.array_equal(np.isinf(a), np.isinf(b))
    fin = np.isfinite(a)
    assert np.array_equal(a[fin], b[fin]), "oracle values differ from the reference"
    assert int(ref["nAccepted"]) == res["nAccepted"]
    assert int(ref["MaxStencilWidth"]) == res["MaxStencilWidth"]
    assert np.array_equal(ref["activeNeighs"].ravel().astype(np.uint64), res["activeNeighs"])


def test_rs3_stencil_classes():
    """Six Selling differences of the direction's matrix, then the theta and phi steps of weights
    1 / (xi ds)^2 and 1 / (sin(theta) xi ds)^2, ds = 2 pi / nphi."""
    nt, nph, h, xi, eps = 4, 8, 0.125, 0.3, 0.1
    off, w = O.rs3_stencil(nt, nph, h, xi, eps)
    ds = 2 * np.pi / nph
    for it in range(nt):
        for ip in range(nph):
            c = it * nph + ip
            assert np.array_equal(off[c, 6], [0, 0, 0, 1, 0])
            assert np.array_equal(off[c, 7], [0, 0, 0, 0, 1])
            assert not off[c, :6, 3:].any()
            th, ph = (it + 0.5) * ds, ip * ds
            assert w[c, 6] == pytest.approx(1 / (xi * ds) ** 2)
            assert w[c, 7] == pytest.approx(1 / (np.sin(th) * xi * ds) ** 2)
            v = np.array([np.cos(th), np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph)])
            m = ((1 - eps ** 2) * np.outer(v, v) + eps ** 2 * np.eye(3)) / h ** 2
            rec = sum(w[c, k] * np.outer(off[c, k, :3], off[c, k, :3]) for k in range(6))
            np.testing.assert_allclose(rec, m, rtol=1e-12, atol=1e-9 * np.trace(m))


def test_rs3_bundle_dimensions_checked():
    params, _, _ = load_golden("rs3_8x4_dual")
    bad = dict(params, dims=np.array([8, 8, 8, 4, 12], float))
    with pytest.raises(ValueError):
        O.rs3_solve(bad)


def test_rs3_host_refusals_before_device_work():
    """The setup checks and the refused keys of the GPU solve path answer before any device work:
    HFM_ERR_VALUE (2) for inconsistent bundle dimensions (Curvature3.h:63-67, 97-98), and
    HFM_ERR_UNSUPPORTED (3) for the outputs this path does not build on the sphere bundle."""
    import hamiltonfastmarching_b200 as H
    from hamiltonfastmarching_b200 import workloads as W
    p = W.reedsshepp3_case(8, 4, seed=45)
    cases = [(dict(dims=np.array([8, 8, 8, 4, 12.0])), 2, "inconsistent bundle dimensions"),
             (dict(model="ReedsSheppForward3", projective=1.0, dims=np.array([8, 8, 8, 4, 16.0])), 2,
              "ReedsSheppForward3 setup error"),
             (dict(walls=np.zeros((8, 8, 8, 4, 8))), 3, "walls"),
             (dict(inspectSensitivity=p["seeds"]), 3, "inspectSensitivity"),
             (dict(seedRadius=1.0), 3, "seedRadius"),
             (dict(tips=p["seeds"]), 3, "tips")]
    for extra, code, text in cases:
        with pytest.raises(H.PyExp) as e:
            H.run(dict(p, verbosity=0.0, **extra))
        assert e.value.code == code and text in str(e.value), (extra, e.value.code, str(e.value))
