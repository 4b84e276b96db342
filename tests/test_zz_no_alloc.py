"""The entry point that allocates nothing (hfm_solve_riemann2_static_scratch), through the C ABI.

It serves callers that cannot let the library allocate device memory. Its output must equal the
existing device entry point (hfm_solve_riemann_device, FP64) within the FP64 parity tolerance of
these tests, on consecutive calls that share its fixed scratch buffer: the second call is a
smaller problem than the first, so stale contents of the buffer would show up.
Collected last on purpose; it passes alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from hamiltonfastmarching_b200 import _lib
from hamiltonfastmarching_b200 import workloads as W

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10


def _inputs(p):
    import torch
    n0, n1 = (int(d) for d in p["dims"])
    metric = torch.from_numpy(np.ascontiguousarray(p["metric"].reshape(-1, 3))).cuda()
    ij = np.floor(np.atleast_2d(p["seeds"]) / p["gridScale"]).astype(np.int64)
    sidx = np.ascontiguousarray(np.unique(np.ravel_multi_index(ij.T, (n0, n1))).astype(np.int64))
    sval = np.zeros(len(sidx))
    return n0, n1, metric, sidx, sval


def _existing_entry(p):
    import torch
    L = _lib.load()
    n0, n1, metric, sidx, sval = _inputs(p)
    values = torch.empty(n0 * n1, dtype=torch.float64, device="cuda")
    a = _lib.RiemannDeviceArgs()
    a.ndim = 2
    a.dims[0], a.dims[1] = n0, n1
    a.grid_scale[0] = a.grid_scale[1] = p["gridScale"]
    a.precision = 64
    a.metric, a.values = metric.data_ptr(), values.data_ptr()
    a.nseeds, a.seed_index, a.seed_value = len(sidx), sidx.ctypes.data, sval.ctypes.data
    a.stream = torch.cuda.current_stream().cuda_stream
    err = ctypes.create_string_buffer(256)
    rc = L.hfm_solve_riemann_device(ctypes.byref(a), None, err, 256)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    return values.cpu().numpy()


def _static_entry(p):
    import torch
    L = _lib.load()
    n0, n1, metric, sidx, sval = _inputs(p)
    values = torch.empty(n0 * n1, dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    rc = L.hfm_solve_riemann2_static_scratch(n0, n1, p["gridScale"], metric.data_ptr(), 0, len(sidx),
                                             sidx.ctypes.data, sval.ctypes.data, values.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream, err, 256)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    return values.cpu().numpy()


def test_static_scratch_matches_existing_entry_on_two_consecutive_calls():
    cases = [W.riemann2_case(256, aniso=5.0, seed=0), W.riemann2_case(96, aniso=10.0, seed=3, n_seeds=3)]
    for p in cases:
        got = _static_entry(p)
        ref = _existing_entry(p)
        assert np.array_equal(np.isinf(got), np.isinf(ref))
        fin = np.isfinite(ref)
        rel = np.max(np.abs(got[fin] - ref[fin])) / np.max(np.abs(ref[fin]))
        assert rel <= FP64_RTOL, rel


def test_static_scratch_rejects_grids_above_its_limit():
    L = _lib.load()
    err = ctypes.create_string_buffer(256)
    idx = np.zeros(1, np.int64)
    val = np.zeros(1)
    rc = L.hfm_solve_riemann2_static_scratch(600, 600, 1.0 / 600, 1, 0, 1, idx.ctypes.data, val.ctypes.data, 1,
                                             None, err, 256)
    assert rc == 2
    assert b"262144-cell limit" in err.value
