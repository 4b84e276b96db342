"""The entry point that allocates nothing (hfm_solve_riemann2_static_scratch), through the C ABI.

It serves callers that cannot let the library allocate device memory. Its output must equal the
existing device entry point (hfm_solve_riemann_device, FP64) within the FP64 parity tolerance of
these tests, on consecutive calls that share its fixed scratch buffer: the second call is a
smaller problem than the first, so stale contents of the buffer would show up. It is also held to
the reference's own values on the `riemann2_64` fixture, on a dual metric, on repeated seeds
(the first value is kept) and on a metric that is not positive definite (an error, not a result).
Collected last on purpose; it passes alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from hamiltonfastmarching_b200 import _lib
from hamiltonfastmarching_b200 import workloads as W

from conftest import load_golden

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10


def _seeds(p, values=None):
    n0, n1 = (int(d) for d in p["dims"])
    ij = np.floor(np.atleast_2d(p["seeds"]) / p["gridScale"]).astype(np.int64)
    sidx = np.ascontiguousarray(np.ravel_multi_index(ij.T, (n0, n1)).astype(np.int64))
    sval = np.ascontiguousarray(np.zeros(len(sidx)) if values is None else np.asarray(values, float))
    return sidx, sval


def _metric(p):
    import torch
    key = "dualMetric" if "dualMetric" in p else "metric"
    return torch.from_numpy(np.ascontiguousarray(p[key].reshape(-1, 3))).cuda(), key == "dualMetric"


def _existing_entry(p, sidx, sval):
    import torch
    L = _lib.load()
    n0, n1 = (int(d) for d in p["dims"])
    metric, dual = _metric(p)
    values = torch.empty(n0 * n1, dtype=torch.float64, device="cuda")
    a = _lib.RiemannDeviceArgs()
    a.ndim = 2
    a.dims[0], a.dims[1] = n0, n1
    a.grid_scale[0] = a.grid_scale[1] = p["gridScale"]
    a.dual = 1 if dual else 0
    a.precision = 64
    a.metric, a.values = metric.data_ptr(), values.data_ptr()
    a.nseeds, a.seed_index, a.seed_value = len(sidx), sidx.ctypes.data, sval.ctypes.data
    a.stream = torch.cuda.current_stream().cuda_stream
    err = ctypes.create_string_buffer(256)
    rc = L.hfm_solve_riemann_device(ctypes.byref(a), None, err, 256)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    return values.cpu().numpy()


def _static_entry(p, sidx, sval, expect=0):
    import torch
    L = _lib.load()
    n0, n1 = (int(d) for d in p["dims"])
    metric, dual = _metric(p)
    values = torch.empty(n0 * n1, dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    rc = L.hfm_solve_riemann2_static_scratch(n0, n1, p["gridScale"], metric.data_ptr(), 1 if dual else 0, len(sidx),
                                             sidx.ctypes.data, sval.ctypes.data, values.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream, err, 256)
    assert rc == expect, (rc, err.value)
    torch.cuda.synchronize()
    return values.cpu().numpy(), err.value


def _rel(got, ref):
    assert np.array_equal(np.isinf(got), np.isinf(ref))
    fin = np.isfinite(ref)
    return np.max(np.abs(got[fin] - ref[fin])) / np.max(np.abs(ref[fin]))


def test_static_scratch_matches_existing_entry_on_two_consecutive_calls():
    cases = [W.riemann2_case(256, aniso=5.0, seed=0), W.riemann2_case(96, aniso=10.0, seed=3, n_seeds=3)]
    for p in cases:
        sidx, sval = _seeds(p)
        got, _ = _static_entry(p, sidx, sval)
        ref = _existing_entry(p, sidx, sval)
        assert _rel(got, ref) <= FP64_RTOL


def test_static_scratch_matches_reference_fixture():
    params, out, _ = load_golden("riemann2_64")
    sidx, sval = _seeds(params)
    got, _ = _static_entry(params, sidx, sval)
    assert _rel(got, out["values"].reshape(-1)) <= FP64_RTOL


def test_static_scratch_dual_metric_and_repeated_seeds():
    p = W.riemann2_case(80, aniso=6.0, seed=5, n_seeds=3)
    m = p.pop("metric").reshape(-1, 3)
    det = m[:, 0] * m[:, 2] - m[:, 1] ** 2
    p["dualMetric"] = np.stack([m[:, 2] / det, -m[:, 1] / det, m[:, 0] / det], -1).reshape(80, 80, 3)
    sidx, _ = _seeds(p)
    # the first seed repeated with another value: the first value is kept, as the main entry does
    sidx = np.ascontiguousarray(np.concatenate([sidx, sidx[:1]]))
    sval = np.ascontiguousarray(np.concatenate([np.arange(len(sidx) - 1) * 0.01, [5.0]]))
    got, _ = _static_entry(p, sidx, sval)
    ref = _existing_entry(p, sidx, sval)
    assert _rel(got, ref) <= FP64_RTOL
    assert got[sidx[0]] == sval[0]


def test_static_scratch_rejects_a_metric_that_is_not_positive_definite():
    p = W.riemann2_case(32, aniso=3.0, seed=2)
    p["metric"] = p["metric"].copy()
    p["metric"][7, 9] = [1.0, 2.0, 1.0]  # determinant -3
    sidx, sval = _seeds(p)
    _, err = _static_entry(p, sidx, sval, expect=2)
    assert b"positive definite" in err
    # the shared buffer holds that call's failed state; the next call starts clean
    q = W.riemann2_case(32, aniso=3.0, seed=2)
    sidx, sval = _seeds(q)
    got, _ = _static_entry(q, sidx, sval)
    assert _rel(got, _existing_entry(q, sidx, sval)) <= FP64_RTOL


def test_static_scratch_rejects_grids_above_its_limit():
    L = _lib.load()
    err = ctypes.create_string_buffer(256)
    idx = np.zeros(1, np.int64)
    val = np.zeros(1)
    rc = L.hfm_solve_riemann2_static_scratch(600, 600, 1.0 / 600, 1, 0, 1, idx.ctypes.data, val.ctypes.data, 1,
                                             None, err, 256)
    assert rc == 2
    assert b"262144-cell limit" in err.value
