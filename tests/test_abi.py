"""The C ABI library without a GPU: it loads, exports every symbol include/hfm_b200.h declares,
and its key-value store follows the reference IO semantics. No compute call is made."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
import hamiltonfastmarching_b200 as H
from hamiltonfastmarching_b200 import _lib


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hfm_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hfm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 16
    lib = _lib.load()
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES)
    nm = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    for s in syms:
        assert re.search(rf"\bT {s}\b", nm), f"{s} not exported"


def test_version_and_device_count_without_gpu():
    assert "sm_100a" in H.version()
    n = _lib.load()
    import ctypes
    c = ctypes.c_int(-1)
    assert n.hfm_device_count(ctypes.byref(c)) in (0, 4)
    assert c.value >= 0


def test_store_roundtrip_and_bookkeeping():
    io = H.HFMIO("RowMajor")
    io.set_string("model", "Riemann2")
    io.set_scalar("gridScale", 0.25)
    a = np.arange(24, dtype=float).reshape(2, 4, 3)
    io.set_array("metric", a)
    assert io.get_string("model") == "Riemann2"
    assert io.get_scalar("gridScale") == 0.25
    np.testing.assert_array_equal(io.get_array("metric"), a)
    assert io.has_field("metric") and not io.has_field("nothing")
    assert io.erase_field("metric") and not io.has_field("metric")
    assert io.computed_keys() == "[]"   # nothing computed yet


def test_store_errors_raise_not_crash():
    io = H.HFMIO()
    with pytest.raises(H.PyExp) as e:
        io.get_scalar("missing")
    assert e.value.code == 1
    io.set_array("v", np.zeros(3))
    with pytest.raises(H.PyExp):
        io.get_scalar("v")     # array field read as scalar
    io.set_scalar("s", 1.0)
    with pytest.raises(H.PyExp):
        io.get_array("s")      # scalar read as array
    with pytest.raises(H.PyExp):
        io.run()               # no model key: reported, not a segfault


@pytest.mark.parametrize("key,val", [("exportActiveOffsets", 1.0), ("order", 2.0), ("factoringRadius", 5.0),
                                     ("speed_times", np.zeros(3))])
def test_unsupported_options_rejected_before_gpu_work(key, val):
    p = {"model": "Riemann2", "arrayOrdering": "RowMajor", "dims": np.array([8., 8.]), "gridScale": 0.125,
         "metric": np.array([1., 0., 1.]), "seeds": np.array([[0.5, 0.5]]), "verbosity": 0.0, key: val}
    with pytest.raises(H.PyExp) as e:
        H.run(p)
    assert e.value.code == 3, str(e.value)


@pytest.mark.parametrize("solver,code", [("Runge", 2)])
def test_geodesic_solver_choice_checked_before_gpu_work(solver, code):
    p = {"model": "Riemann2", "arrayOrdering": "RowMajor", "dims": np.array([8., 8.]), "gridScale": 0.125,
         "metric": np.array([1., 0., 1.]), "seeds": np.array([[0.5, 0.5]]), "verbosity": 0.0,
         "tips": np.array([[0.1, 0.1]]), "geodesicSolver": solver}
    with pytest.raises(H.PyExp) as e:
        H.run(p)
    assert e.value.code == code, str(e.value)


def test_model_mismatch_is_reported():
    p = {"model": "Riemann3", "dims": np.array([8., 8.]), "verbosity": 0.0}
    io = H.HFMIO("RowMajor")
    io.set_dict(p)
    with pytest.raises(H.PyExp) as e:
        io.run("Riemann2")
    assert "Executable applies to Riemann2" in str(e.value)


def test_cli_reports_missing_input(tmp_path):
    exe = os.path.join(ROOT, "hamiltonfastmarching_b200", "bin", "FileHFM_b200")
    if not os.path.exists(exe):
        pytest.skip("CLI not built")
    r = subprocess.run([exe, str(tmp_path / "nope"), str(tmp_path / "out")], capture_output=True, text=True)
    assert r.returncode != 0
    assert "could not be opened" in r.stdout


def test_no_host_path_exits_the_process():
    """Only host stubs of __device__ functions may contain a call to exit: a host launch path that
    reaches one (a device-only helper called from host code) would end the caller's process."""
    out = subprocess.run(["objdump", "-d", "--no-show-raw-insn", "-C", _lib.LIB_PATH],
                         capture_output=True, text=True).stdout
    fn, callers = None, set()
    for line in out.splitlines():
        m = re.match(r"^[0-9a-f]+ <(.*)>:$", line)
        if m:
            fn = m.group(1)
        elif "<exit@plt>" in line and "call" in line:
            callers.add(fn)
    allowed = {"wall_visible"}
    bad = [c for c in callers if not any(a in c for a in allowed)]
    assert not bad, bad


def test_server_without_device_fails_cleanly():
    import ctypes
    c = ctypes.c_int(0)
    _lib.load().hfm_device_count(ctypes.byref(c))
    if c.value > 0:
        pytest.skip("a CUDA device is present")
    from hamiltonfastmarching_b200.serving import Server
    with pytest.raises(RuntimeError):
        Server(lanes=2)


def test_array_view_is_read_in_place():
    io = H.HFMIO("RowMajor")
    a = np.arange(12, dtype=np.float64).reshape(3, 4)
    io.set_array_view("metric", a)
    assert np.array_equal(io.get_array("metric"), a)
    a[1, 2] = -7.0  # the store reads the caller's memory
    assert io.get_array("metric")[1, 2] == -7.0
    io.set_array("metric", np.zeros((2, 2)))  # replacing the key drops the view
    assert np.array_equal(io.get_array("metric"), np.zeros((2, 2)))
    io.set_array_view("empty", np.zeros((0, 3)))
    assert io.get_array("empty").shape == (0, 3)


def test_static_scratch_entry_rejects_bad_arguments_before_any_device_work():
    """The allocation-free entry validates its arguments on the host: no CUDA call is reached."""
    import ctypes
    L = _lib.load()
    err = ctypes.create_string_buffer(256)
    idx = np.zeros(2, np.int64)
    val = np.zeros(2)

    def call(nx, ny, h=0.1, metric=1, nseeds=1, sidx=idx, values=1):
        return L.hfm_solve_riemann2_static_scratch(nx, ny, h, metric, 0, nseeds, sidx.ctypes.data,
                                                   val.ctypes.data, values, None, err, 256)

    assert call(8, 8, metric=0) == 7                      # null metric
    assert call(8, 8, values=0) == 7                      # null output
    assert call(0, 8) == 2 and call(8, 8, h=0.0) == 2     # empty grid, bad scale
    assert call(1 << 40, 1 << 40) == 2 and b"limit" in err.value   # no overflow of nx * ny
    assert call(600, 600) == 2 and b"262144-cell limit" in err.value
    assert call(8, 8, nseeds=0) == 2 and call(8, 8, nseeds=1025) == 2
    bad = np.array([64, 0], np.int64)
    assert call(8, 8, nseeds=2, sidx=bad) == 2 and b"out of range" in err.value
