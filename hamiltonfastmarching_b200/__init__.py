"""hamiltonfastmarching_b200 — B200-native drop-in for the HamiltonFastMarching solve path.

:class:`HFMIO` mirrors the reference's pybind11 class of the same name
(``Interfaces/PythonHFM/src/main.cpp:11-47``): ``run``, ``get_string``/``set_string``,
``get_scalar``/``set_scalar``, ``get_array``/``set_array``, ``computed_keys``, ``has_field``,
``erase_field``; errors raise :class:`PyExp` (the reference registers ``JMMCppException`` as
``PyExp``, ``main.cpp:31``). As in the reference Python binding the default array ordering is
``YXZ_RowMajor`` (``Output/PythonIO.h:20``); the key ``arrayOrdering`` overrides it.

:func:`run` is the dictionary-in / dictionary-out convenience of the file-based interface
(``JMM_CPPLibs/FileIO/FileIO.py:54-73``), with the file interface's default ordering ``RowMajor``.
:func:`run_batch` solves many such dictionaries in one batched launch sequence
(``hfm_run_batch``); each gets what :func:`run` would return for it alone.

Everything runs through the C ABI of ``include/hfm_b200.h`` on the GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ast
import ctypes
from typing import Dict

import numpy as np

from . import _lib

__all__ = ["HFMIO", "PyExp", "run", "run_batch", "run_ios", "version"]


class PyExp(RuntimeError):
    """Error raised by the solver library; ``code`` is the HFM_ERR_* status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{_lib.ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


def version() -> str:
    return _lib.load().hfm_version().decode()


class HFMIO:
    def __init__(self, arrayOrdering: str = "YXZ_RowMajor"):
        self._L = _lib.load()
        if arrayOrdering not in _lib.ORDERINGS:
            raise ValueError(f"unknown array ordering {arrayOrdering}")
        self._views = {}
        self._h = self._L.hfm_io_create(_lib.ORDERINGS[arrayOrdering])
        if not self._h:
            raise MemoryError("hfm_io_create failed")

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._L.hfm_io_destroy(h)

    def _check(self, rc: int):
        if rc != _lib.HFM_OK:
            raise PyExp(rc, self._L.hfm_io_last_error(self._h).decode())

    # ---- reference HFMIO surface
    def run(self, expected_model: str = None):
        self._check(self._L.hfm_run(self._h, expected_model.encode() if expected_model else None))

    def run_sensitivity(self):
        """Reverse first variation for the inspectSensitivity keys now set, from the device state
        of the last ``run`` with ``retainState = 1`` (no new solve); fills costSensitivity_i."""
        self._check(self._L.hfm_run_sensitivity(self._h))

    def set_scalar(self, key: str, value: float):
        self._check(self._L.hfm_io_set_scalar(self._h, key.encode(), float(value)))

    def get_scalar(self, key: str) -> float:
        v = ctypes.c_double()
        self._check(self._L.hfm_io_get_scalar(self._h, key.encode(), ctypes.byref(v)))
        return v.value

    def set_string(self, key: str, value: str):
        self._check(self._L.hfm_io_set_string(self._h, key.encode(), value.encode()))

    def get_string(self, key: str) -> str:
        n = ctypes.c_size_t()
        self._check(self._L.hfm_io_get_string(self._h, key.encode(), None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        self._check(self._L.hfm_io_get_string(self._h, key.encode(), buf, n.value + 1, ctypes.byref(n)))
        return buf.value.decode()

    def set_array(self, key: str, value):
        a = np.ascontiguousarray(value, dtype=np.float64)
        shape = (ctypes.c_int64 * max(a.ndim, 1))(*a.shape)
        self._check(self._L.hfm_io_set_array(self._h, key.encode(), a.ctypes.data_as(ctypes.c_void_p), a.ndim,
                                             shape))

    def set_array_view(self, key: str, value):
        """Zero-copy ``set_array``: the store reads ``value`` in place (a reference is kept here)."""
        a = np.ascontiguousarray(value, dtype=np.float64)
        shape = (ctypes.c_int64 * max(a.ndim, 1))(*a.shape)
        self._check(self._L.hfm_io_set_array_view(self._h, key.encode(), a.ctypes.data_as(ctypes.c_void_p), a.ndim,
                                                  shape))
        self._views[key] = a

    def get_array(self, key: str, copy: bool = True) -> np.ndarray:
        """The array `key`; with ``copy=False`` a read-only view of the store's memory, which keeps
        this store alive (valid while the key is not replaced or erased)."""
        if not copy:
            ptr, nd = ctypes.c_void_p(), ctypes.c_int()
            shape = (ctypes.c_int64 * 16)()
            self._check(self._L.hfm_io_get_array_ptr(self._h, key.encode(), ctypes.byref(ptr), ctypes.byref(nd),
                                                     shape, 16))
            if nd.value == 0:
                raise PyExp(1, f"PythonIO error : field {key} is a scalar, not an array")
            dims = tuple(shape[i] for i in range(nd.value))
            n = int(np.prod(dims))
            if n == 0:
                return np.empty(dims, np.float64)
            buf = (ctypes.c_double * n).from_address(ptr.value)
            buf.owner = self  # the store outlives the view
            a = np.frombuffer(buf, dtype=np.float64).reshape(dims)
            a.flags.writeable = False
            return a
        nd = ctypes.c_int()
        shape = (ctypes.c_int64 * 16)()
        self._check(self._L.hfm_io_get_array_info(self._h, key.encode(), ctypes.byref(nd), shape, 16))
        if nd.value == 0:
            raise PyExp(1, f"PythonIO error : field {key} is a scalar, not an array")
        dims = tuple(shape[i] for i in range(nd.value))
        out = np.empty(dims, np.float64)
        self._check(self._L.hfm_io_get_array(self._h, key.encode(), out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def computed_keys(self) -> str:
        n = ctypes.c_size_t()
        self._check(self._L.hfm_io_computed_keys(self._h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        self._check(self._L.hfm_io_computed_keys(self._h, buf, n.value + 1, ctypes.byref(n)))
        return buf.value.decode()

    def has_field(self, key: str) -> bool:
        r = self._L.hfm_io_has_field(self._h, key.encode())
        if r < 0:
            raise PyExp(-r, "invalid argument")
        return bool(r)

    def erase_field(self, key: str) -> bool:
        return self._L.hfm_io_erase_field(self._h, key.encode()) == _lib.HFM_OK

    # ---- helpers
    def set_dict(self, params: Dict, views: bool = False):
        """Sets every entry; with ``views`` arrays are referenced in place (set_array_view)."""
        for k, v in params.items():
            if isinstance(v, str):
                self.set_string(k, v)
            elif np.isscalar(v) or (isinstance(v, np.ndarray) and v.ndim == 0):
                self.set_scalar(k, float(v))
            elif views:
                self.set_array_view(k, v)
            else:
                self.set_array(k, np.asarray(v, dtype=np.float64))

    def get_computed(self, copy: bool = True) -> Dict:
        out = {}
        for key, kind in ast.literal_eval(self.computed_keys()):
            out[key] = (self.get_string(key) if kind == "string" else
                        self.get_scalar(key) if kind == "float" else self.get_array(key, copy))
        return out


def run(params: Dict, arrayOrdering: str = "RowMajor", expected_model: str = None) -> Dict:
    """Solve an ``hfmIn`` dictionary on the GPU and return the computed ``hfmOut`` dictionary."""
    io = HFMIO(arrayOrdering)
    io.set_dict(params, views=True)  # the call is synchronous: the caller's arrays are read in place
    io.run(expected_model)
    return io.get_computed(copy=False)  # read-only views of the result store


def run_ios(ios, expected_model: str = None):
    """Run several :class:`HFMIO` stores as one batch (``hfm_run_batch``).

    Returns the list of per-store status codes (0 = success); the message of a failed store is
    ``hfm_io_last_error`` of that store.
    """
    L = _lib.load()
    n = len(ios)
    handles = (ctypes.c_void_p * max(n, 1))(*[io._h for io in ios])
    codes = (ctypes.c_int * max(n, 1))()
    L.hfm_run_batch(handles, n, expected_model.encode() if expected_model else None, codes)
    return [codes[i] for i in range(n)]


def run_batch(params_list, arrayOrdering: str = "RowMajor", expected_model: str = None, raise_errors: bool = True):
    """Solve a list of ``hfmIn`` dictionaries as one batch; returns the list of ``hfmOut``.

    With ``raise_errors`` False a failed instance yields a :class:`PyExp` in its slot instead of
    raising.
    """
    ios = []
    for params in params_list:
        io = HFMIO(arrayOrdering)
        io.set_dict(params)
        ios.append(io)
    codes = run_ios(ios, expected_model)
    out = []
    for io, rc in zip(ios, codes):
        if rc != _lib.HFM_OK:
            e = PyExp(rc, io._L.hfm_io_last_error(io._h).decode())
            if raise_errors:
                raise e
            out.append(e)
        else:
            out.append(io.get_computed())
    return out
