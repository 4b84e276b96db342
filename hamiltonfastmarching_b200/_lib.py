"""ctypes binding of the in-tree C ABI library ``libhfm_b200.so`` (include/hfm_b200.h).

The library is loaded from this package directory only; if it is missing the import fails loudly
(run ``python -m hamiltonfastmarching_b200.build``). There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhfm_b200.so")

HFM_OK = 0
ERROR_NAMES = {1: "HFM_ERR_KEY", 2: "HFM_ERR_VALUE", 3: "HFM_ERR_UNSUPPORTED", 4: "HFM_ERR_CUDA",
               5: "HFM_ERR_NOT_CONVERGED", 6: "HFM_ERR_NOMEM", 7: "HFM_ERR_ARG"}
ORDERINGS = {"RowMajor": 0, "ColumnMajor": 1, "YXZ_RowMajor": 2, "YXZ_ColumnMajor": 3}

# Every symbol include/hfm_b200.h declares, with its ctypes signature.
_P, _I, _D, _S, _SZ, _I64P = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p, ctypes.c_size_t, \
    ctypes.POINTER(ctypes.c_int64)
SIGNATURES = {
    "hfm_io_create": ([_I], _P),
    "hfm_io_destroy": ([_P], None),
    "hfm_io_set_scalar": ([_P, _S, _D], _I),
    "hfm_io_set_string": ([_P, _S, _S], _I),
    "hfm_io_set_array": ([_P, _S, _P, _I, _I64P], _I),
    "hfm_io_set_array_view": ([_P, _S, _P, _I, _I64P], _I),
    "hfm_io_get_scalar": ([_P, _S, ctypes.POINTER(_D)], _I),
    "hfm_io_get_string": ([_P, _S, _P, _SZ, ctypes.POINTER(_SZ)], _I),
    "hfm_io_get_array_info": ([_P, _S, ctypes.POINTER(_I), _I64P, _I], _I),
    "hfm_io_get_array": ([_P, _S, _P, _SZ], _I),
    "hfm_io_get_array_ptr": ([_P, _S, ctypes.POINTER(_P), ctypes.POINTER(_I), _I64P, _I], _I),
    "hfm_io_has_field": ([_P, _S], _I),
    "hfm_io_erase_field": ([_P, _S], _I),
    "hfm_io_computed_keys": ([_P, _P, _SZ, ctypes.POINTER(_SZ)], _I),
    "hfm_run": ([_P, _S], _I),
    "hfm_run_batch": ([_P, _I, _S, ctypes.POINTER(_I)], _I),
    "hfm_run_sensitivity": ([_P], _I),
    "hfm_io_last_error": ([_P], _S),
    "hfm_version": ([], _S),
    "hfm_device_count": ([ctypes.POINTER(_I)], _I),
}

class RiemannDeviceArgs(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("dims", ctypes.c_int64 * 3), ("grid_scale", ctypes.c_double * 3),
                ("dual", ctypes.c_int), ("precision", ctypes.c_int), ("sweeps_per_tile", ctypes.c_int),
                ("metric", ctypes.c_void_p), ("walls", ctypes.c_void_p), ("nseeds", ctypes.c_int64),
                ("seed_index", ctypes.c_void_p), ("seed_value", ctypes.c_void_p), ("values", ctypes.c_void_p),
                ("stream", ctypes.c_void_p)]


class SolveStats(ctypes.Structure):
    _fields_ = [("n_accepted", ctypes.c_int64), ("max_stencil_width", ctypes.c_int),
                ("stencil_ms", ctypes.c_double), ("solve_ms", ctypes.c_double), ("rounds", ctypes.c_int64),
                ("tile_activations", ctypes.c_int64), ("local_solves", ctypes.c_int64)]


SIGNATURES["hfm_solve_riemann_device"] = ([ctypes.POINTER(RiemannDeviceArgs), ctypes.POINTER(SolveStats),
                                           ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int)
SIGNATURES["hfm_solve_riemann2_static_scratch"] = ([ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                                    ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int)
SIGNATURES["hfm_kernel_launches"] = ([ctypes.POINTER(ctypes.c_ulonglong)], ctypes.c_int)


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("lanes", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("hbm_budget_bytes", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_ulonglong), ("completed", ctypes.c_ulonglong),
                ("batches", ctypes.c_ulonglong), ("max_batch", ctypes.c_ulonglong),
                ("queued", ctypes.c_ulonglong), ("running_batches", ctypes.c_ulonglong),
                ("budget_bytes", ctypes.c_double), ("bytes_in_use", ctypes.c_double),
                ("peak_bytes", ctypes.c_double)]


SIGNATURES["hfm_server_create"] = ([ctypes.POINTER(ServerConfig)], ctypes.c_void_p)
SIGNATURES["hfm_server_submit"] = ([ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int)
SIGNATURES["hfm_server_wait"] = ([ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(ctypes.c_int)],
                                 ctypes.c_int)
SIGNATURES["hfm_server_release"] = ([ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)], ctypes.c_int)
SIGNATURES["hfm_server_get_stats"] = ([ctypes.c_void_p, ctypes.POINTER(ServerStats)], ctypes.c_int)
SIGNATURES["hfm_server_destroy"] = ([ctypes.c_void_p], None)

_lib = None


def load():
    """Load the library and declare every exported symbol; raises ImportError if absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m hamiltonfastmarching_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib
