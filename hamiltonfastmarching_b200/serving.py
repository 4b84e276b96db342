"""Serving loop: continuous batching of solve requests on one GPU (``hfm_server_*`` of the C ABI).

``Server(max_batch=64)`` starts the native request loop: one scheduler thread and, per model
family (Riemann2, Riemann3, ReedsShepp2, per precision), a resident persistent solver.
``submit(params)`` queues an ``hfmIn`` dictionary and returns a :class:`Ticket`. A plain solve
is admitted, in arrival order, while its device footprint fits in the memory budget and fewer
than ``max_batch`` instances are resident; it joins the running solver at its next slice and is
released as soon as its own tiles have converged, so requests that arrive while others run share
the GPU with them and none waits for a larger one. Requests with other outputs (geodesics,
sensitivities, activeNeighs ...) or other models run through ``hamiltonfastmarching_b200.run``
between slices. ``max_batch=1`` serves every request that way, one at a time (the plain loop).
``Ticket.result()`` returns the ``hfmOut`` dictionary that ``hamiltonfastmarching_b200.run``
returns for the same request alone; ``Ticket.times`` gives the submit, start and completion times
(seconds) used for latency statistics.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional

from . import HFMIO, PyExp, _lib

__all__ = ["Server", "Ticket"]


class Ticket:
    def __init__(self, server: "Server", io: HFMIO, ticket: int):
        self._server, self._io, self.id = server, io, ticket
        self.status: Optional[int] = None
        self.times = None

    def wait(self, timeout: float = -1.0) -> bool:
        """Waits for completion (timeout < 0: no limit); False if the timeout expired."""
        if self.status is not None:
            return True
        st = ctypes.c_int()
        rc = self._server._L.hfm_server_wait(self._server._h, self.id, float(timeout), ctypes.byref(st))
        if rc == 5:
            return False
        if rc != 0:
            raise PyExp(rc, "hfm_server_wait failed")
        times = (ctypes.c_double * 3)()
        self._server._L.hfm_server_release(self._server._h, self.id, times)
        self.status, self.times = st.value, tuple(times)
        self._server._pending.pop(self.id, None)
        return True

    def result(self, timeout: float = -1.0) -> Dict:
        if not self.wait(timeout):
            raise TimeoutError(f"request {self.id} still running")
        if self.status != _lib.HFM_OK:
            raise PyExp(self.status, self._io._L.hfm_io_last_error(self._io._h).decode())
        return self._io.get_computed()

    @property
    def latency(self) -> float:
        return self.times[2] - self.times[0]


class Server:
    def __init__(self, lanes: int = 1, max_batch: int = 64, hbm_budget_bytes: float = 0.0, device: int = 0):
        """``lanes`` is accepted for compatibility and not used."""
        self._L = _lib.load()
        cfg = _lib.ServerConfig(device, lanes, max_batch, float(hbm_budget_bytes))
        self._h = self._L.hfm_server_create(ctypes.byref(cfg))
        # stores of the requests not yet completed: the scheduler reads them until completion, so
        # they live here even when the caller drops its tickets
        self._pending: Dict[int, HFMIO] = {}
        if not self._h:
            raise RuntimeError("hfm_server_create failed (no CUDA device or no memory)")

    def submit(self, params: Dict, arrayOrdering: str = "RowMajor", views: bool = True) -> Ticket:
        """Queues a request. With ``views`` the arrays of ``params`` are referenced, not copied: keep
        them unmodified until the ticket completes (the ticket holds references to them)."""
        io = HFMIO(arrayOrdering)
        io.set_dict(params, views=views)
        return self.submit_io(io)

    def submit_io(self, io: HFMIO) -> Ticket:
        t = ctypes.c_uint64()
        rc = self._L.hfm_server_submit(self._h, io._h, ctypes.byref(t))
        if rc != 0:
            raise PyExp(rc, self._L.hfm_io_last_error(io._h).decode())
        self._pending[t.value] = io
        return Ticket(self, io, t.value)

    def stats(self) -> Dict:
        st = _lib.ServerStats()
        self._L.hfm_server_get_stats(self._h, ctypes.byref(st))
        return {name: getattr(st, name) for name, _ in _lib.ServerStats._fields_}

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._L.hfm_server_destroy(h)  # returns once every submitted request has completed
        self._pending = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()
