"""MAPROP (source_code/maprop.f, IPROP = 7): the quasi-adiabatic
log-derivative propagator of Manolopoulos, for many energies of one system.

Every quantity that does not depend on the energy is built here on the host,
once per system, in the order maprop.f:33-290 forms it:

* W(R) with ERED = 0 at the sector ends and midpoints (the half-step radii
  of the segment: R += DR/2 twice a sector, maprop.f:86,251);
* per sector k, the midpoint W's eigenvalues EIVAL_k and eigenvectors U_k
  (DIAGVC: ascending), the basis change Q_k = T_{k-1}^T U_k (T_0 = I,
  T_k = U_k), and the correction added to Y in the old basis,
  C_k = T_{k-1}^T [(W(R_start) - W(R_mid)) DR/6 + Q_end(k-1)] T_{k-1}, with
  Q_end(k) = (W(R_end) - W(R_mid)) DR/6;
* the last basis T and end correction Q_end.

The energy-dependent sweep (the basis change of Y, the half-angle sector
propagators of EIVAL - ERED, the inversion and its node count, the last
back-transformation) runs on the device (`mgpu_ldma_run_host`, one CTA per
energy, N <= 100).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import _dp, _ip
from .propagators import Coupling, PropagatorError, Segment


def hammat_host(c: Coupling, r: float, p: np.ndarray, ered: float = 0.0) -> np.ndarray:
    """W(R) (HAMMAT + SUMLAM, hammat.f:85-113) as a full n x n matrix:
    sum_l VL_l P_l (IV indexing where IVLFL > 0), then on the diagonal
    CENT min(1/R^2, 1e16) (NRSQ = 0), EINT (NCONST = 0), the confinement
    term and -ERED."""
    n, nb = c.n, c.nvlblk
    npair = n * (n + 1) // 2
    v = c.vl[: nb * npair].reshape(npair, nb)[:, : c.nham]
    p = np.asarray(p, dtype=np.float64)
    if c.ivlfl > 0:
        ix = c.iv[: nb * npair].reshape(npair, nb)[:, : c.nham] - 1
        w = np.sum(np.where(v != 0.0, v * p[ix], 0.0), axis=1)
    else:
        w = v @ p[: c.nham]
    j = np.repeat(np.arange(n), np.arange(1, n + 1))
    i = np.arange(npair) - j * (j + 1) // 2
    out = np.zeros((n, n))
    out[i, j] = w
    out[j, i] = w
    d = np.zeros(n)
    if c.nrsq == 0:
        d += min(1.0 / (r * r), 1.0e16) * c.cent[:n]
    if c.nconst == 0:
        d += c.eint[:n]
    if c.conlen > 0.0:
        d += r * r / c.conlen ** 4
    out[np.arange(n), np.arange(n)] += d - ered
    return out


@dataclass
class LDMATables:
    n: int
    nstep: int
    dr: float
    eival: np.ndarray  # (nstep, n)
    q: np.ndarray      # (nstep, n, n)
    corr: np.ndarray   # (nstep, n, n)
    tfin: np.ndarray   # (n, n)
    qfin: np.ndarray   # (n, n)


def ldma_tables(c: Coupling, seg: Segment) -> LDMATables:
    """The energy-independent half of MAPROP over one segment (its P table
    at the 2*NSTEP+1 half-step radii)."""
    n, ns, dr = c.n, seg.nstep, seg.dr
    eival = np.empty((ns, n))
    q = np.empty((ns, n, n))
    corr = np.empty((ns, n, n))
    t = np.eye(n)
    qend = np.zeros((n, n))
    u = hammat_host(c, float(seg.rtab[0]), seg.ptab[0])
    cr = dr / 6.0
    for k in range(ns):
        w = hammat_host(c, float(seg.rtab[2 * k + 1]), seg.ptab[2 * k + 1])
        corr[k] = t.T @ ((u - w) * cr + qend) @ t
        ev, vec = np.linalg.eigh(w)
        q[k] = t.T @ vec
        eival[k] = ev
        t = vec
        u = hammat_host(c, float(seg.rtab[2 * k + 2]), seg.ptab[2 * k + 2])
        qend = (u - w) * cr
    return LDMATables(n, ns, dr, eival, q, corr, t, qend)


class LDMAPlan:
    """MAPROP for many energies of one system: the tables built once,
    ``run_host`` propagating every energy on the device."""

    def __init__(self, coupling: Coupling, seg: Segment, tables: LDMATables | None = None):
        if seg.kind != "LD":
            raise ValueError("MAPROP uses the half-step radii of an LD segment")
        self.coupling = coupling
        self.tables = tables if tables is not None else ldma_tables(coupling, seg)
        t = self.tables
        L = _lib.load()
        self._arrays = [np.ascontiguousarray(t.eival, dtype=np.float64),
                        np.ascontiguousarray(np.transpose(t.q, (0, 2, 1)), dtype=np.float64),    # column-major
                        np.ascontiguousarray(np.transpose(t.corr, (0, 2, 1)), dtype=np.float64),
                        np.asfortranarray(t.tfin, dtype=np.float64).ravel(order="F"),
                        np.asfortranarray(t.qfin, dtype=np.float64).ravel(order="F")]
        h = ctypes.c_void_p()
        rc = L.mgpu_ldma_create(ctypes.byref(h), t.n, t.nstep, float(t.dr), 1 if t.dr < 0 else 0,
                                *[a.ctypes.data_as(_dp) for a in self._arrays])
        if rc != 0:
            raise PropagatorError(f"LDMA: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        self._handle = h

    def run_host(self, y0s, ereds):
        """Returns (list of Y at the end, NODES, status) for the energies."""
        L = _lib.load()
        n = self.tables.n
        nj = len(ereds)
        e = np.ascontiguousarray(ereds, dtype=np.float64)
        y = np.concatenate([np.asfortranarray(y0, dtype=np.float64).ravel(order="F") for y0 in y0s])
        nodes = np.zeros(nj, dtype=np.int32)
        status = np.zeros(nj, dtype=np.int32)
        rc = L.mgpu_ldma_run_host(self._handle, nj, e.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                  nodes.ctypes.data_as(_ip), status.ctypes.data_as(_ip))
        if rc != 0:
            raise PropagatorError(f"LDMA run: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        ys = [y[j * n * n:(j + 1) * n * n].reshape((n, n), order="F") for j in range(nj)]
        return ys, nodes, status

    def close(self):
        if getattr(self, "_handle", None):
            _lib.load().mgpu_ldma_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
