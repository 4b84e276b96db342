"""Stencils on the GPU against the reference: getStencils (HFMInterface.hxx:360-375) and the
exportStencils arrays.

* The GPU Selling offsets of every cell equal the reference's getStencils offsets exactly on the
  three stencil fixtures (random SPD metrics, anisotropy 1-100, diagonal and exact-tie metrics,
  one of them dual); the printed weights equal the reference's 6-digit prints.
* The whole `stencils` string equals the one the reference executable prints for the same input
  (Riemann2/3, ReedsShepp2, Elastica2, Isotropic2, Diagonal2), out-of-range points included.
* A random-SPD sweep (2D and 3D, anisotropy 1-100, with diagonal, grid-aligned and exact-tie
  metrics) gives offsets and FP64 weights equal bit for bit to the oracle's Selling
  decomposition (fmo_riemann_stencils, itself bit-exact with the reference on the fixtures).
"""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN_STENCILS, ROOT, load_golden
import hamiltonfastmarching_b200 as H
from hamiltonfastmarching_b200 import workloads as W
from oracle import oracle as O
from oracle.refrun import have_reference, run_reference

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from make_golden import parse_stencils, random_spd  # noqa: E402

pytestmark = pytest.mark.gpu


def cell_centres(dims, h):
    axes = [(np.arange(n) + 0.5) * h for n in dims]
    return np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, len(dims))


@pytest.mark.parametrize("name", GOLDEN_STENCILS)
def test_gpu_offsets_equal_reference_fixture(name):
    params, _, extra = load_golden(name)
    ndim = len(params["dims"])
    dims = [int(d) for d in params["dims"]]
    p = dict(params, getStencils=cell_centres(dims, params["gridScale"]), verbosity=0.0)
    out = H.run(p)
    st = parse_stencils(out["stencils"], ndim)
    assert len(st) == int(np.prod(dims))
    offs = np.stack([o for o, _ in st])
    ws = np.stack([w for _, w in st])
    ref_off = extra["stencil_offsets"].astype(np.int64)
    assert np.array_equal(offs, ref_off), f"{np.sum(np.any(offs != ref_off, axis=(1, 2)))} cells differ"
    np.testing.assert_array_equal(ws, extra["stencil_weights_6digits"])


def _reference_string_cases():
    r2 = W.riemann2_case(12, aniso=20.0, seed=7)
    r3 = W.riemann3_case(8, seed=2, n_spheres=0, n_seeds=1)
    rs = W.curvature2_case(16, 12, "ReedsShepp2", seed=3)
    el = W.curvature2_case(12, 8, "Elastica2", seed=4)
    iso = {"model": "Isotropic2", "arrayOrdering": "RowMajor", "dims": np.array([6.0, 5.0]), "gridScale": 0.2,
           "cost": np.linspace(1.0, 2.0, 30).reshape(6, 5), "seeds": np.array([[0.5, 0.5]])}
    diag = {"model": "Diagonal2", "arrayOrdering": "RowMajor", "dims": np.array([6.0, 5.0]),
            "gridScales": np.array([0.2, 0.3]), "seeds": np.array([[0.5, 0.5]]),
            "speed": np.stack([np.linspace(1.0, 2.0, 30).reshape(6, 5), np.full((6, 5), 3.0)], -1)}
    rng = np.random.default_rng(9)
    cases = {}
    for name, p, pts in (
            ("riemann2", r2, np.vstack([rng.uniform(0, 1, (9, 2)), [[1.5, 0.2]]])),
            ("riemann3", r3, rng.uniform(0, 1, (6, 3))),
            ("reedsshepp2", rs, np.column_stack([rng.uniform(0, 1, (7, 2)), rng.uniform(-7, 13, 7)])),
            ("elastica2", el, np.column_stack([rng.uniform(0, 1, (3, 2)), rng.uniform(0, 6.3, 3)])),
            ("isotropic2", iso, np.array([[0.1, 0.1], [0.7, 0.3], [5.0, 5.0]])),
            ("diagonal2", diag, np.array([[0.1, 0.1], [0.7, 0.3]]))):
        q = {k: v for k, v in p.items() if not k.startswith("_")}
        q.update(getStencils=pts, exportValues=0.0)
        cases[name] = q
    return cases


@pytest.mark.parametrize("name", ["riemann2", "riemann3", "reedsshepp2", "elastica2", "isotropic2", "diagonal2"])
def test_gpu_stencils_string_equals_reference_executable(name):
    p = _reference_string_cases()[name]
    if not have_reference(p["model"]):
        pytest.skip("reference executables not built (make -C oracle ref)")
    ref = run_reference(dict(p, verbosity=0.0))
    assert ref["retcode"] == 0, ref["log"]
    out = H.run(dict(p, verbosity=0.0))
    assert out["stencils"] == ref["stencils"]


@pytest.mark.parametrize("ndim,dual", [(2, False), (2, True), (3, False), (3, True)])
def test_gpu_selling_sweep_bit_exact_with_oracle(ndim, dual):
    side = 48 if ndim == 2 else 14
    rng = np.random.default_rng(100 + 10 * ndim + int(dual))
    dims = (side,) * ndim
    mats = random_spd(rng, side ** ndim, ndim)
    # grid-aligned anisotropic metrics (weights of zero and exact ties among superbase updates)
    for i in range(0, len(mats), 29):
        d = rng.choice([1.0, 4.0, 100.0], ndim)
        mats[i] = [d[0], 0.0, d[1]] if ndim == 2 else [d[0], 0.0, d[1], 0.0, 0.0, d[2]]
    mats = mats.reshape(dims + (-1,))
    h = 1.0 / side
    p = {"model": f"Riemann{ndim}", "arrayOrdering": "RowMajor", "dims": np.array(dims, float), "gridScale": h,
         "dualMetric" if dual else "metric": mats, "seeds": np.full((1, ndim), 0.5), "exportStencils": 1.0,
         "exportValues": 0.0, "verbosity": 0.0}
    out = H.run(p)
    nk = 3 if ndim == 2 else 6
    off = out["stencilOffsets"].reshape(-1, nk, ndim)
    w = out["stencilWeights"].reshape(-1, nk)
    ooff, ow = O.riemann_stencils(mats.reshape(-1, mats.shape[-1]), h, dual)
    assert np.array_equal(off, ooff[:, :, :ndim].astype(np.float64))
    np.testing.assert_array_equal(w, ow)
