"""AIRY (source_code/aiprop.f with potent.f, corr.f, waveig.f; the
reference's IPROPL = 9): the long-range log-derivative propagator of
Alexander and Manolopoulos, for many energies of one system.

In every sector [R_L, R_L + h] the local wavevector matrix -W is
diagonalised (its average over the two Gauss-Legendre points R_mid +- h/(2
sqrt 3), potent.f:55-110) and each local channel i sees the linear
reference k_i^2(x) = E_i - s_i x (s_i the diagonal of the local dW/dR).  Z
crosses the sector by invariant imbedding, Z <- Y4 - Y2 (Y1 + Z)^-1 Y2, with
the diagonal (Y1, Y2, Y4) of the reference's exact solutions, Airy
functions.

Split as the reference splits it between its first energy and the others
(the ISCRU reuse, aiprop.f:107-113,143-160): the sector geometry -- widths
from the TOLHI step control (or the DRSET series for TOLHI = 0), local
eigenvalues at the first energy, slopes, basis changes -- is built once on
the host (`sector_tables`); per energy the eigenvalues shift by E - E0 and
the host evaluates the Airy sector functions (`sector_y124`, O(N) a
sector); the device runs the O(N^3) sweep: the basis change, the inversion
with its negative-pivot count and the imbedding update
(`mgpu_airy_run_host`, one CTA per energy, N <= 100).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import _dp, _ip
from .ldma import hammat_host
from .propagators import Coupling, PropagatorError

SQ3 = 1.732050807  # the reference's sqrt(3) of the Gauss-Legendre points (potent.f:51)


# ----------------------------------------------------------------- Airy functions
def _airy_scaled(z: np.ndarray):
    """(Ai, Ai', Bi, Bi') with the growth split off: for z > 0 the returned
    values are Ai e^zeta, Ai' e^zeta, Bi e^-zeta, Bi' e^-zeta (zeta = 2/3
    z^1.5), for z <= 0 the functions themselves.  Deep in the decaying
    region (z > 1e4) from the asymptotic series in 1/zeta (Abramowitz and
    Stegun 10.4.58-10.4.67, four terms)."""
    from scipy.special import airy, airye
    z = np.asarray(z, dtype=np.float64)
    a, ap, b, bp = airy(np.minimum(z, 0.0))
    mid = (z > 0.0) & (z <= 1.0e4)
    ea, eap, eb, ebp = airye(np.where(mid, z, 0.0))
    a, ap, b, bp = (np.where(mid, u, v) for u, v in ((ea, a), (eap, ap), (eb, b), (ebp, bp)))
    big = z > 1.0e4
    if np.any(big):
        zb = z[big]
        zeta = 2.0 / 3.0 * zb * np.sqrt(zb)
        u = [1.0]
        v = [1.0]
        for k in range(1, 4):
            uk = math.exp(math.lgamma(3 * k + 0.5) - k * math.log(54.0) - math.lgamma(k + 1) - math.lgamma(k + 0.5))
            u.append(uk)
            v.append(-(6 * k + 1) / (6 * k - 1) * uk)
        sa = sum(((-1) ** k) * u[k] / zeta ** k for k in range(4))
        sva = sum(((-1) ** k) * v[k] / zeta ** k for k in range(4))
        sb = sum(u[k] / zeta ** k for k in range(4))
        svb = sum(v[k] / zeta ** k for k in range(4))
        q = zb ** 0.25
        sp = math.sqrt(math.pi)
        a[big] = sa / (2.0 * sp * q)
        ap[big] = -q * sva / (2.0 * sp)
        b[big] = sb / (sp * q)
        bp[big] = q * svb / sp
    return a, ap, b, bp


def _y124_extended(alpha: float, beta: float, width: float):
    """(Y1, Y2, Y4) of one channel at raised precision, for an oscillatory
    phase too large for a double: z1, z2 formed in mpmath from the double
    inputs, so that their difference alpha*h keeps its digits."""
    import mpmath as mp
    zeta = 2.0 / 3.0 * (abs(alpha) * (abs(beta) + abs(width))) ** 1.5
    with mp.workdps(int(25 + 2 * math.log10(max(zeta, 10.0)))):
        al, be, h = mp.mpf(alpha), mp.mpf(beta), mp.mpf(width)
        z1, z2 = al * (be - h / 2), al * (be + h / 2)
        a1, b1, a1p, b1p = mp.airyai(z1), mp.airybi(z1), mp.airyai(z1, 1), mp.airybi(z1, 1)
        a2, b2, a2p, b2p = mp.airyai(z2), mp.airybi(z2), mp.airyai(z2, 1), mp.airybi(z2, 1)
        d = a1 * b2 - b1 * a2
        return float(al * (b1p * a2 - a1p * b2) / d), float(al / mp.pi / d), float(al * (a1 * b2p - b1 * a2p) / d)


def sector_y124(width: float, eig: np.ndarray, hp: np.ndarray):
    """Diagonal imbedding propagator of one sector for every local channel:
    psi'' = (s x - E) psi on x in [-h/2, h/2] (E = eig, s = hp), written as
    psi'(a) = -Y1 psi(a) + Y2 psi(b), psi'(b) = -Y2 psi(a) + Y4 psi(b)."""
    s = np.where(hp == 0.0, 1.0e-30, hp)
    alpha = np.sign(s) * np.abs(s) ** (1.0 / 3.0)
    beta = -eig / s
    z1 = alpha * (beta - 0.5 * width)
    z2 = alpha * (beta + 0.5 * width)
    a1, a1p, b1, b1p = _airy_scaled(z1)
    a2, a2p, b2, b2p = _airy_scaled(z2)
    pos1, pos2 = np.maximum(z1, 0.0), np.maximum(z2, 0.0)
    zt1 = 2.0 / 3.0 * pos1 * np.sqrt(pos1)
    zt2 = 2.0 / 3.0 * pos2 * np.sqrt(pos2)
    both = (z1 > 0.0) & (z2 > 0.0)
    # zeta(z2) - zeta(z1) without cancellation where both are positive
    za, zb = np.where(both, z1, 1.0), np.where(both, z2, 1.0)
    dz = 2.0 / 3.0 * (alpha * width) * (zb * zb + za * zb + za * za) / (zb * np.sqrt(zb) + za * np.sqrt(za))
    g = np.where(both, dz, zt2 - zt1)
    m = np.abs(g)
    ep, em = np.exp(g - m), np.exp(-g - m)
    d = a1 * b2 * ep - b1 * a2 * em
    y1 = alpha * (b1p * a2 * em - a1p * b2 * ep) / d
    y4 = alpha * (a1 * b2p * ep - b1 * a2p * em) / d
    y2 = alpha / math.pi * np.exp(-m) / d
    osc = np.maximum(np.where(z1 < 0.0, 2.0 / 3.0 * np.abs(z1) ** 1.5, 0.0),
                     np.where(z2 < 0.0, 2.0 / 3.0 * np.abs(z2) ** 1.5, 0.0))
    for i in np.nonzero(osc > 1.0e6)[0]:
        y1[i], y2[i], y4[i] = _y124_extended(float(alpha[i]), float(beta[i]), float(width))
    return y1, y2, y4


# ----------------------------------------------------------------- sector geometry
@dataclass
class AiryTables:
    n: int
    e0: float            # the energy the geometry was built at
    outward: bool
    widths: np.ndarray   # (nsect,)
    eig0: np.ndarray     # (nsect, n) local eigenvalues of -W at e0
    hp: np.ndarray       # (nsect, n) local dW/dR diagonal
    tmat: np.ndarray     # (nsect, n, n): previous local basis -> this one (the first: primitive -> local)
    vfin: np.ndarray     # (n, n) the last local basis in the primitive one


def _drcalc(rstart, rstop, kstep, nstep, pw):
    """Step kstep (0-based) of NSTEP steps equally spaced in R^(1-POW) (drcalc.f:22-38)."""
    pi = 1.0 - pw
    if pi != 0.0:
        z0, z1 = rstart ** pi, rstop ** pi
        dz = (z1 - z0) / float(nstep)
        return (z0 + float(kstep + 1) * dz) ** (1.0 / pi) - (z0 + float(kstep) * dz) ** (1.0 / pi)
    dz = rstart * ((rstop / rstart) ** (1.0 / float(nstep)) - 1.0)
    return dz * (1.0 + dz / rstart) ** kstep


def sector_tables(c: Coupling, potential, rstart: float, rstop: float, drnow: float, e0: float,
                  tolhi: float = 1.0e-4, powr: float = 3.0, nstep: int = 0, maxstp: int = 500000) -> AiryTables:
    """The sector geometry of aiprop.f:120-380 at energy e0 (reduced units):
    per sector the local eigenvalues and eigenvectors of -W averaged over
    the Gauss-Legendre points, the local dW/dR diagonal and its largest
    off-diagonal element, CORR's CDIAG / COFF, and the next width from
    TOLHI (capped at twice the last, times (1 + DR/R)^3 inwards), or with
    TOLHI = 0 the DRCALC series of NSTEP widths.  potential(R) gives the P
    vector at R."""
    if tolhi == 0.0 and nstep < 1:
        raise ValueError("TOLHI = 0 needs NSTEP")
    if rstop == rstart or (rstop > rstart) != (drnow > 0.0):
        raise ValueError("DRNOW must point from RSTART to RSTOP")
    outward = rstop > rstart
    n = c.n
    eigold = np.linalg.eigvalsh(-hammat_host(c, rstart, potential(rstart), e0))
    widths, eigs, hps, tmats = [], [], [], []
    drmid = 0.5 * drnow
    rlast = rstart
    rnow = rlast + drmid
    rnext = rlast + drnow
    last = False
    vecnow = None
    for kstep in range(1, maxstp + 1):
        ra, rb = rnow - 0.5 * drnow / SQ3, rnow + 0.5 * drnow / SQ3
        wa = hammat_host(c, ra, potential(ra), e0)
        wb = hammat_host(c, rb, potential(rb), e0)
        eig, vec = np.linalg.eigh(-0.5 * (wb + wa))
        loc = vec.T @ ((SQ3 / drnow) * (wb - wa)) @ vec
        loc = 0.5 * (loc + loc.T)
        hp = np.diag(loc).copy()
        xlarge = float(np.abs(np.tril(loc, -1)).max()) if n > 1 else 0.0
        tmats.append(vec if vecnow is None else vecnow.T @ vec)
        vecnow = vec
        # CORR (corr.f:43-75)
        w2p = -(2.0 / drmid ** 2) * (eig - eigold + drmid * hp)
        cdiag = abs(drnow ** 3) * float(np.mean(np.abs(w2p))) / 12.0
        coff = float(np.mean(np.sqrt(np.abs(eig)))) * xlarge * abs(drnow ** 3) / 12.0
        eigold = eig
        widths.append(drnow)
        eigs.append(eig)
        hps.append(hp)
        if last:
            break
        if 0.0 < tolhi < 1.0:
            cmax = max(abs(cdiag), abs(coff))
            fac = 2.0 if cmax == 0.0 else (tolhi / cmax) ** (1.0 / powr)
            if drnow < 0.0 and rnext + drnow > 0.0:
                fac = fac * (1.0 + drnow / rnext) ** 3
            drnow = drnow * min(fac, 2.0)
            rlast = rnext
            rnext = rnext + drnow
            last = (rstop - rstart) * (rstop - rnext) < 0.0
        elif tolhi == 0.0:
            drnow = _drcalc(rstart, rstop, kstep, nstep, powr)
            rlast = rnext
            rnext = rnext + drnow
            last = nstep - kstep <= 1
        else:
            raise ValueError("0 <= TOLHI < 1")
        if last:
            rnext = rstop
            drnow = rnext - rlast
        rnew = rlast + 0.5 * drnow
        drmid = rnew - rnow
        rnow = rnew
    return AiryTables(n, float(e0), outward, np.array(widths), np.array(eigs), np.array(hps), np.array(tmats),
                      vecnow)


def energy_y124(t: AiryTables, ered: float) -> np.ndarray:
    """(nsect, n, 3) sector functions at ERED: the eigenvalues shifted by ERED - E0."""
    out = np.empty((t.widths.size, t.n, 3))
    for k, h in enumerate(t.widths):
        y1, y2, y4 = sector_y124(float(h), t.eig0[k] + (ered - t.e0), t.hp[k])
        out[k, :, 0], out[k, :, 1], out[k, :, 2] = y1, y2, y4
    return out


class AiryPlan:
    """AIRY over one system's sector tables: ``run_host`` propagates Z for
    every energy on the device (the sector functions from the host)."""

    def __init__(self, tables: AiryTables):
        self.tables = t = tables
        L = _lib.load()
        self._tm = np.ascontiguousarray(np.transpose(t.tmat, (0, 2, 1)), dtype=np.float64)  # column-major
        self._vf = np.asfortranarray(t.vfin, dtype=np.float64).ravel(order="F")
        h = ctypes.c_void_p()
        rc = L.mgpu_airy_create(ctypes.byref(h), t.n, int(t.widths.size), 0 if t.outward else 1,
                                self._tm.ctypes.data_as(_dp), self._vf.ctypes.data_as(_dp))
        if rc != 0:
            raise PropagatorError(f"AIRY: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        self._handle = h

    def run_host(self, z0s, ereds):
        """Returns (list of Z at RSTOP in the primitive basis, NODES, status)."""
        L = _lib.load()
        t = self.tables
        n, nj = t.n, len(ereds)
        ys = np.ascontiguousarray(np.stack([energy_y124(t, float(e)) for e in ereds]), dtype=np.float64)
        z = np.concatenate([np.asfortranarray(z0, dtype=np.float64).ravel(order="F") for z0 in z0s])
        nodes = np.zeros(nj, dtype=np.int32)
        status = np.zeros(nj, dtype=np.int32)
        rc = L.mgpu_airy_run_host(self._handle, nj, ys.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
                                  nodes.ctypes.data_as(_ip), status.ctypes.data_as(_ip))
        if rc != 0:
            raise PropagatorError(f"AIRY run: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        return [z[j * n * n:(j + 1) * n * n].reshape((n, n), order="F") for j in range(nj)], nodes, status

    def close(self):
        if getattr(self, "_handle", None):
            _lib.load().mgpu_airy_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AiryInward:
    """A long-range AIRY segment as the inward propagator of a BOUND/FIELD
    search (`BoundProblem(inward=...)`): called with ERED it returns (Z at
    RSTOP, NODES).  The sector geometry is built at the first energy it is
    called with and kept for the later ones, as the reference's ISCRU file
    keeps it; z0(ered) gives Z at RSTART (default: the adiabatic WKB start
    for closed channels, bound.adiabatic_wkb_y)."""

    def __init__(self, coupling: Coupling, potential, rstart: float, rstop: float, drnow: float,
                 tolhi: float = 1.0e-4, powr: float = 3.0, nstep: int = 0, z0=None):
        self.c, self.potential = coupling, potential
        self.args = (rstart, rstop, drnow, tolhi, powr, nstep)
        self.z0 = z0
        self.plan = None

    def __call__(self, ered: float):
        rstart, rstop, drnow, tolhi, powr, nstep = self.args
        if self.plan is None:
            t = sector_tables(self.c, self.potential, rstart, rstop, drnow, float(ered), tolhi=tolhi, powr=powr,
                              nstep=nstep)
            self.plan = AiryPlan(t)
        if self.z0 is not None:
            z0 = self.z0(float(ered))
        else:
            from .bound import adiabatic_wkb_y
            z0 = adiabatic_wkb_y(self.c, rstart, self.potential(rstart), float(ered), rstop > rstart)
        zs, nodes, status = self.plan.run_host([z0], [float(ered)])
        if status[0] != 0:
            raise PropagatorError(f"AIRY: {_lib.status_string(int(status[0]))}", int(status[0]))
        return zs[0], int(nodes[0])
