"""Request server: single propagations submitted at any time, batched and
overlapped on the GPU by the library's scheduler (mgpu_server_* and
mgpu_submit / mgpu_poll / mgpu_wait in include/molscat_gpu.h).

    srv = Server("LDMD", hbm_budget=8 << 30, streams=4)
    sid = srv.add_system(coupling, segment)      # device-resident from now on
    req = srv.submit(sid, ered, y0)              # returns at once
    y = req.wait()                               # Y(RSTOP); req.nodes, req.times()

The reference's drivers call MDPROP/LDPROP once per (JTOT, block, energy)
(mol.driver.f:1181-1855); a result here is the same as that single call,
whatever else runs beside it.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .propagators import Coupling, PropagatorError, Segment

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class Request:
    """One submitted propagation; owns the host buffers the library fills."""

    def __init__(self, server: "Server", ticket: int, sys_id: int, n: int, y: np.ndarray, out: np.ndarray):
        self._srv = server
        self.ticket = ticket
        self.sys_id = sys_id
        self.n = n
        self._y = y        # column-major N x N, filled on completion
        self._out = out    # nodes, status, kfail
        self._rc = None

    def done(self) -> bool:
        r = self._srv._L.mgpu_poll(self._srv._h, ctypes.c_longlong(self.ticket))
        if r < 0:
            raise PropagatorError("unknown request", -r)
        return r == 1

    def wait(self) -> np.ndarray:
        """Y(RSTOP) as an N x N array; raises PropagatorError if the request
        failed or its propagation hit a zero / non-finite pivot."""
        if self._rc is None:
            self._rc = int(self._srv._L.mgpu_wait(self._srv._h, ctypes.c_longlong(self.ticket)))
        if self._rc != 0:
            raise PropagatorError(f"request {self.ticket}: {_lib.status_string(self._rc)}", self._rc)
        if self.status != 0:
            raise PropagatorError(f"request {self.ticket}: {_lib.status_string(self.status)} at step {self.kfail}",
                                  self.status, self.kfail)
        return self._y.reshape((self.n, self.n), order="F")

    @property
    def nodes(self) -> int:
        return int(self._out[0])

    @property
    def status(self) -> int:
        return int(self._out[1])

    @property
    def kfail(self) -> int:
        return int(self._out[2])

    def times(self) -> tuple:
        """(submitted, launched, completed) on the host's steady clock, seconds."""
        t = np.zeros(3)
        self._srv._L.mgpu_request_times(self._srv._h, ctypes.c_longlong(self.ticket), t.ctypes.data_as(_dp))
        return float(t[0]), float(t[1]), float(t[2])

    def latency(self) -> float:
        t = self.times()
        return t[2] - t[0]


class Server:
    def __init__(self, prop: str = "LDMD", hbm_budget: int = 8 << 30, streams: int = 4, max_batch: int = 4096,
                 max_systems: int = 4096):
        if prop not in ("LDMD", "LDJ"):
            raise ValueError(prop)
        self._L = _lib.load()
        self.prop = prop
        h = ctypes.c_void_p()
        iprop = _lib.MGPU_PROP_LDMD if prop == "LDMD" else _lib.MGPU_PROP_LDJ
        rc = self._L.mgpu_server_create(ctypes.byref(h), iprop, int(hbm_budget), int(streams), int(max_batch),
                                        int(max_systems))
        if rc != 0:
            raise PropagatorError(f"server: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        self._h = h
        self._sys_n = []
        self._keep = []  # the coupling / segment objects stay alive with the server

    def add_system(self, c: Coupling, seg: Segment) -> int:
        sid = ctypes.c_int(-1)
        cs, gs = c.c_struct(), seg.c_struct()
        rc = self._L.mgpu_server_add_system(self._h, ctypes.byref(cs), ctypes.byref(gs), ctypes.byref(sid))
        if rc != 0:
            raise PropagatorError(f"add_system: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        self._sys_n.append(c.n)
        self._keep.append((c, seg))
        return sid.value

    def submit(self, sys_id: int, ered: float, y0: np.ndarray) -> Request:
        n = self._sys_n[sys_id]
        y0 = np.asfortranarray(y0, dtype=np.float64)
        if y0.shape != (n, n):
            raise ValueError(f"Y0 must be {n} x {n}")
        y = np.empty(n * n)
        out = np.zeros(3, dtype=np.int32)
        tk = ctypes.c_longlong(0)
        op = out.ctypes.data_as(_ip)
        rc = self._L.mgpu_submit(self._h, int(sys_id), float(ered), y0.ravel(order="F").ctypes.data_as(_dp),
                                 y.ctypes.data_as(_dp), op, ctypes.cast(ctypes.addressof(op.contents) + 4, _ip),
                                 ctypes.cast(ctypes.addressof(op.contents) + 8, _ip), ctypes.byref(tk))
        if rc != 0:
            raise PropagatorError(f"submit: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        return Request(self, tk.value, sys_id, n, y, out)

    def in_flight(self) -> tuple:
        b, q = ctypes.c_int(0), ctypes.c_int(0)
        nb = ctypes.c_size_t(0)
        self._L.mgpu_server_in_flight(self._h, ctypes.byref(b), ctypes.byref(q), ctypes.byref(nb))
        return b.value, q.value, nb.value

    def release(self, req: Request) -> None:
        self._L.mgpu_release(self._h, ctypes.c_longlong(req.ticket))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.mgpu_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def latency_percentiles(reqs, qs=(50, 99)) -> dict:
    lat = np.array([r.latency() for r in reqs])
    return {f"p{q}": float(np.percentile(lat, q)) for q in qs}
