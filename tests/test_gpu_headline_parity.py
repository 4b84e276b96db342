"""Parity at the configurations the benchmark numbers are quoted on, against the reference's own
executables run at test time (oracle/_ref, compiled from the reference sources).

* Riemann3 192^3 FP64, the benchmark instance (40 spherical walls, 16 seeds, generator seed 1):
  arrival times within 1e-10 relative max-norm of FileHFM_Riemann3, nAccepted exact; the FP32
  path within 1e-5 of FP64.
* TTI3 128^3 (10 m spacing, Thomsen media, one top-face source), the differentiation workload:
  costSensitivity_0 of the 64-receiver loss gradient within 1e-10 of its max-norm of
  FileHFM_TTI3's backward differentiation, arrival times within 1e-10.
* The lifted models at the batch and serving sizes: ReedsShepp2 256x256x60 and Elastica2
  128x128x60 (tubular-image cost, xi = 0.1) FP64 within 1e-10 of the reference, FP32 within 1e-5
  of FP64.

Each reference run takes 10-70 s of one CPU core.
"""
import numpy as np
import pytest

import hamiltonfastmarching_b200 as H
from hamiltonfastmarching_b200 import workloads as W
from oracle.refrun import have_reference, run_reference

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10
FP32_RTOL = 1e-5


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert np.array_equal(np.isinf(a), np.isinf(b)), "reached sets differ"
    fin = np.isfinite(a)
    return float(np.max(np.abs(a[fin] - b[fin])) / np.max(np.abs(a[fin])))


def need(model):
    if not have_reference(model):
        pytest.skip("reference executables not built (make -C oracle ref)")


def test_riemann3_192_fp64_equals_reference():
    need("Riemann3")
    p = W.riemann3_case(192, seed=1)
    ref = run_reference(dict(p, verbosity=0.0))
    assert ref["retcode"] == 0, ref["log"][-2000:]
    out = H.run(dict(p, verbosity=0.0))
    assert rel_err(ref["values"], out["values"]) <= FP64_RTOL
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    assert int(out["MaxStencilWidth"]) == int(ref["MaxStencilWidth"])
    o32 = H.run(dict(p, verbosity=0.0, solverPrecision="float32"))
    assert rel_err(out["values"], o32["values"]) <= FP32_RTOL


def tti3_loss_gradient_case(n=128):
    """The differentiation workload: one source at the top-face centre, 64 receivers on the top face
    and the loss gradient 2 (T - T_obs) as their inspection weights (T_obs from vp with a +5%
    Gaussian blob)."""
    h = 0.01
    p = W.tti3_case(n, h=h, seed=4)
    p.pop("_vp")
    L = n * h
    obs = W.tti3_case(n, h=h, seed=4, blob=((0.5 * L, 0.5 * L, 0.35 * L), 0.12 * L, 0.05))
    obs.pop("_vp")
    rng = np.random.default_rng(7)
    rx = rng.integers(0, n, (64, 2))
    T = H.run(dict(p, verbosity=0.0))["values"]
    T_obs = H.run(dict(obs, verbosity=0.0))["values"]
    t, t_obs = T[rx[:, 0], rx[:, 1], 0], T_obs[rx[:, 0], rx[:, 1], 0]
    pts = np.column_stack([(rx + 0.5) * h, np.full(64, 0.5 * h)])
    p.update(inspectSensitivity=pts, inspectSensitivityWeights=2.0 * (t - t_obs),
             inspectSensitivityLengths=np.array([64.0]))
    return p


def test_tti3_128_sensitivity_equals_reference_backward_differentiation():
    need("TTI3")
    p = tti3_loss_gradient_case(128)
    ref = run_reference(dict(p, verbosity=0.0))
    assert ref["retcode"] == 0, ref["log"][-2000:]
    out = H.run(dict(p, verbosity=0.0))
    assert rel_err(ref["values"], out["values"]) <= FP64_RTOL
    a, b = ref["costSensitivity_0"], out["costSensitivity_0"]
    assert np.max(np.abs(a)) > 0
    assert np.max(np.abs(a - b)) <= FP64_RTOL * np.max(np.abs(a))


@pytest.mark.parametrize("model,n", [("ReedsShepp2", 256), ("Elastica2", 128)])
def test_lifted_models_at_batch_sizes(model, n):
    need(model)
    p = W.curvature2_case(n, 60, model, seed=2)
    ref = run_reference(dict(p, verbosity=0.0))
    assert ref["retcode"] == 0, ref["log"][-2000:]
    out = H.run(dict(p, verbosity=0.0))
    assert rel_err(ref["values"], out["values"]) <= FP64_RTOL
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    o32 = H.run(dict(p, verbosity=0.0, solverPrecision="float32"))
    assert rel_err(out["values"], o32["values"]) <= FP32_RTOL
