"""Host-side mirror of the MOLSCAT propagator interface over libmolscat_gpu.

``mdprop`` / ``ldprop`` take the arguments of MDPROP (source_code/mdprop.f:1-4)
and LDPROP (source_code/ldprop.f:1-4) with the same meaning and return
``(Y, NODES)``.  Where the reference would ``STOP`` (mdprop.f:282-288,
ldprop.f:151-153) they raise :class:`PropagatorError` carrying the same
message.  The potential enters as a callable ``potenl(r) -> P`` evaluated on
the host at every radius the propagator visits, exactly the values HAMMAT
would compute (hammat.f:37-83); :func:`hammat_pvec` does that processing for
a POTENL-style function.

:class:`Plan` is the batched form: many systems and many (system, ERED) jobs
in one set of device launches, with the energy-independent MDPROP inverses
shared by all jobs of a system.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import _lib
from ._lib import Coupling_C, Grid_C, MGPU_PROP_LDJ, MGPU_PROP_LDMD, MGPU_PROP_LDMG4, MGPU_PROP_LDMG5

# plan propagators: MDPROP, LDPROP and MGPROP with IMGSEL = 4 / 5
PROPS = {"LDMD": MGPU_PROP_LDMD, "LDJ": MGPU_PROP_LDJ, "LDMG4": MGPU_PROP_LDMG4, "LDMG5": MGPU_PROP_LDMG5}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class PropagatorError(RuntimeError):
    def __init__(self, msg: str, status: int = 0, step: int = 0):
        super().__init__(msg)
        self.status = status
        self.step = step


@dataclass
class Coupling:
    """The propagator inputs that do not depend on R: VL(NVLBLK, N(N+1)/2)
    packed upper-by-columns, IV of the same shape (1-based P indices, used
    when IVLFL>0), EINT(N), CENT(N) and the module-potential flags."""
    n: int
    nham: int
    vl: np.ndarray
    eint: np.ndarray
    cent: np.ndarray
    nvlblk: int = 0
    iv: np.ndarray | None = None
    ivlfl: int = 0
    nconst: int = 0
    nrsq: int = 0
    conlen: float = 0.0

    def __post_init__(self):
        if self.nvlblk == 0:
            self.nvlblk = self.nham
        self.vl = np.ascontiguousarray(self.vl, dtype=np.float64).ravel()
        self.eint = np.ascontiguousarray(self.eint, dtype=np.float64).ravel()
        self.cent = np.ascontiguousarray(self.cent, dtype=np.float64).ravel()
        npair = self.n * (self.n + 1) // 2
        if self.vl.size < self.nvlblk * npair:
            raise ValueError(f"VL needs NVLBLK*N(N+1)/2 = {self.nvlblk * npair} values, got {self.vl.size}")
        if self.eint.size < self.n or self.cent.size < self.n:
            raise ValueError("EINT and CENT need N values")
        if self.ivlfl > 0:
            if self.iv is None:
                raise ValueError("IVLFL>0 needs IV")
            self.iv = np.ascontiguousarray(self.iv, dtype=np.int32).ravel()
        else:
            self.iv = np.zeros(1, dtype=np.int32)

    def c_struct(self) -> Coupling_C:
        return Coupling_C(self.n, self.nham, self.nvlblk, self.ivlfl, self.nconst, self.nrsq,
                          float(self.conlen), self.vl.ctypes.data_as(_dp), self.iv.ctypes.data_as(_ip),
                          self.eint.ctypes.data_as(_dp), self.cent.ctypes.data_as(_dp))


def radial_grid(rstart: float, dr: float, nstep: int) -> np.ndarray:
    """Radii R_k, k=0..2*NSTEP, accumulated as R=R+H the way MDPROP/LDPROP
    step (mdprop.f:69,117,203; ldprop.f:30,57,105)."""
    h = dr / 2.0
    r = np.empty(2 * nstep + 1)
    x = float(rstart)
    r[0] = x
    for k in range(1, 2 * nstep + 1):
        x = x + h
        r[k] = x
    return r


def ldmg_radii(prop: str, rstart: float, dr: float, nstep: int) -> np.ndarray:
    """The radii MGPROP's stages visit ("LDMG4": CS4, 4*NSTEP + 1 of them;
    "LDMG5": MA5, 6*NSTEP), from the library's own coefficients."""
    L = _lib.load()
    ip = PROPS[prop]
    cnt = int(L.mgpu_ldmg_radii(ip, float(rstart), float(dr), int(nstep), None))
    if cnt < 0:
        raise ValueError(f"{prop}: not an LDMG propagator, or NSTEP < 1")
    out = np.empty(cnt)
    L.mgpu_ldmg_radii(ip, float(rstart), float(dr), int(nstep), out.ctypes.data_as(_dp))
    return out


@dataclass
class Segment:
    """One propagation segment: NSTEP, DR and the P table at every radius
    (kind "LD": MDPROP/LDPROP's 2*NSTEP+1 half-step radii; "LDMG4"/"LDMG5":
    the MGPROP stages' radii, ldmg_radii)."""
    nstep: int
    dr: float
    rtab: np.ndarray
    ptab: np.ndarray
    kind: str = "LD"

    @classmethod
    def build(cls, rstart: float, dr: float, nstep: int, potential: Callable[[float], np.ndarray],
              nham: int, kind: str = "LD") -> "Segment":
        rtab = radial_grid(rstart, dr, nstep) if kind == "LD" else ldmg_radii(kind, rstart, dr, nstep)
        ptab = np.empty((rtab.size, max(nham, 1)))
        for k, r in enumerate(rtab):
            ptab[k, :nham] = potential(float(r))[:nham]
        return cls(nstep, dr, rtab, ptab, kind)

    def rows(self) -> int:
        if self.kind == "LD":
            return 2 * self.nstep + 1
        if self.kind == "LDMG4":
            return 4 * self.nstep + 1
        if self.kind == "LDMG5":
            return 6 * self.nstep
        raise ValueError(f"segment kind {self.kind!r}")

    def __post_init__(self):
        self.rtab = np.ascontiguousarray(self.rtab, dtype=np.float64)
        self.ptab = np.ascontiguousarray(self.ptab, dtype=np.float64)
        nr = self.rows()
        if self.rtab.shape[0] != nr or self.ptab.shape[0] != nr:
            raise ValueError(f"tables need {nr} rows for a {self.kind} segment of NSTEP = {self.nstep}")

    def c_struct(self) -> Grid_C:
        return Grid_C(int(self.nstep), float(self.dr), self.rtab.ctypes.data_as(_dp),
                      self.ptab.ctypes.data_as(_dp))


def hammat_pvec(potenl: Callable[[float], Sequence[float]], r: float, mxlam: int, ep2ru: float,
                cm2ru: float, rscale: float = 1.0, vconst: Sequence[float] = (), nrsq: int = 0) -> np.ndarray:
    """The P vector SUMLAM multiplies into VL at radius R (hammat.f:37-83):
    POTENL(R*RSCALE) clamped at +-1e60, VCONST/EP2CM appended, scaled by
    EP2RU, then NRSQ copies of min(1/R^2, 1e16).  SCAPOT and PERTRB are the
    default (identity) hooks."""
    p = np.zeros(mxlam + len(vconst) + nrsq)
    p[:mxlam] = np.asarray(potenl(r * rscale), dtype=np.float64)[:mxlam]
    big = np.abs(p[:mxlam]) > 1.0e60
    p[:mxlam][big] = np.sign(p[:mxlam][big]) * 1.0e60
    ep2cm = ep2ru / cm2ru
    for i, v in enumerate(vconst):
        p[mxlam + i] = v / ep2cm
    p[: mxlam + len(vconst)] *= ep2ru
    if nrsq:
        p[mxlam + len(vconst):] = min(1.0 / (r * r), 1.0e16)
    return p


def _raise_for(name: str, status: int, step: int):
    if status == _lib.MGPU_ERR_INVERSION or status == _lib.MGPU_ERR_NONFINITE:
        if name == "MDPROP":
            msg = f" ***** MDPROP: MATRIX INVERSION ERROR AT STEP K = {step:6d}.  RUN HALTED."
        elif name == "MGPROP":
            msg = f" MGPROP: MATRIX INVERSION ERROR IN SECTOR {step:6d}"
        else:
            msg = " *** ERROR IN SYMINV CALLED FROM LDPROP - TERMINATING"
        if status == _lib.MGPU_ERR_NONFINITE:
            msg += " (non-finite pivot)"
        raise PropagatorError(msg, status, step)
    raise PropagatorError(f"{name}: {_lib.status_string(status)}: {_lib.last_error()}", status, step)


def _single(name, iprop, coupling: Coupling, seg: Segment, ered: float, y0: np.ndarray):
    L = _lib.load()
    n = coupling.n
    y = np.array(y0, dtype=np.float64, order="F", copy=True)
    if y.shape != (n, n):
        raise ValueError(f"Y must be {n}x{n}")
    c = coupling.c_struct()
    g = seg.c_struct()
    nodes = ctypes.c_int(0)
    kfail = ctypes.c_int(0)
    if iprop in (MGPU_PROP_LDMG4, MGPU_PROP_LDMG5):
        rc = L.mgpu_mgprop(4 if iprop == MGPU_PROP_LDMG4 else 5, ctypes.byref(c), ctypes.byref(g), float(ered),
                           y.ctypes.data_as(_dp), ctypes.byref(nodes), ctypes.byref(kfail))
    else:
        fn = L.mgpu_mdprop if iprop == MGPU_PROP_LDMD else L.mgpu_ldprop
        rc = fn(ctypes.byref(c), ctypes.byref(g), float(ered), y.ctypes.data_as(_dp),
                ctypes.byref(nodes), ctypes.byref(kfail))
    if rc != 0:
        _raise_for(name, rc, kfail.value)
    return y, nodes.value


def _args_to_inputs(n, mxlam, nham, vl, iv, eint, cent, rstart, rstop, nstep, dr, potential, nvlblk, ivlfl,
                    nconst, nrsq, conlen, kind="LD"):
    coupling = Coupling(n=n, nham=nham, vl=vl, eint=eint, cent=cent, nvlblk=nvlblk or nham, iv=iv,
                        ivlfl=ivlfl, nconst=nconst, nrsq=nrsq, conlen=conlen)
    seg = Segment.build(rstart, dr, nstep, potential, nham, kind=kind)
    return coupling, seg


def mdprop(n, mxlam, nham, y, vl, iv, eint, cent, rstart, rstop, nstep, dr, ered, *, potential,
           nvlblk=0, ivlfl=0, nconst=0, nrsq=0, conlen=0.0):
    """MDPROP (mdprop.f:1-289) on the GPU.  ``potential(r)`` returns the P
    vector HAMMAT would hand to SUMLAM at R (see :func:`hammat_pvec`).
    Returns (Y at RSTOP as an N x N array, NODES)."""
    del mxlam, rstop  # implied by NHAM/NSTEP/DR exactly as in the reference
    coupling, seg = _args_to_inputs(n, 0, nham, vl, iv, eint, cent, rstart, None, nstep, dr, potential, nvlblk,
                                    ivlfl, nconst, nrsq, conlen)
    return _single("MDPROP", MGPU_PROP_LDMD, coupling, seg, ered, y)


def ldprop(n, mxlam, nham, z, vl, iv, eint, cent, rstart, rstop, nstep, dr, ered, *, potential,
           nvlblk=0, ivlfl=0, nconst=0, nrsq=0, conlen=0.0):
    """LDPROP (ldprop.f:1-154) on the GPU.  Returns (Y at RSTOP, NODES)."""
    del mxlam, rstop
    coupling, seg = _args_to_inputs(n, 0, nham, vl, iv, eint, cent, rstart, None, nstep, dr, potential, nvlblk,
                                    ivlfl, nconst, nrsq, conlen)
    return _single("LDPROP", MGPU_PROP_LDJ, coupling, seg, ered, z)


def mgprop(n, mxlam, nham, y, vl, iv, eint, cent, rstart, rstop, nstep, dr, ered, *, potential, imgsel=4,
           nvlblk=0, ivlfl=0, nconst=0, nrsq=0, conlen=0.0):
    """MGPROP (mgprop.f:1-134) on the GPU, IMGSEL = 4 (CS4) or 5 (MA5):
    NSTEP sectors of DR from RSTART; ``potential(r)`` as for :func:`mdprop`,
    evaluated at every stage's radius.  Returns (Y at RSTOP, NODES)."""
    del mxlam, rstop
    if imgsel not in (4, 5):
        raise ValueError("IMGSEL must be 4 (CS4) or 5 (MA5)")
    kind = f"LDMG{imgsel}"
    coupling, seg = _args_to_inputs(n, 0, nham, vl, iv, eint, cent, rstart, None, nstep, dr, potential, nvlblk,
                                    ivlfl, nconst, nrsq, conlen, kind=kind)
    return _single("MGPROP", PROPS[kind], coupling, seg, ered, y)


def propagate(prop: str, coupling: Coupling, seg: Segment, ered: float, y0: np.ndarray):
    """One propagation from prepared inputs: prop is "LDMD", "LDJ", "LDMG4" or
    "LDMG5" (the segment of the matching kind)."""
    if prop == "LDMD":
        return _single("MDPROP", MGPU_PROP_LDMD, coupling, seg, ered, y0)
    if prop == "LDJ":
        return _single("LDPROP", MGPU_PROP_LDJ, coupling, seg, ered, y0)
    if prop in ("LDMG4", "LDMG5"):
        if seg.kind != prop:
            raise ValueError(f"{prop} needs a {prop} segment")
        return _single("MGPROP", PROPS[prop], coupling, seg, ered, y0)
    raise ValueError(prop)


@dataclass
class Plan:
    """Batched propagation: ``systems[s]`` with ``segments[s]``; job j
    propagates system ``job_sys[j]`` at ``job_ered[j]``."""
    prop: str
    systems: list
    segments: list
    job_sys: np.ndarray
    job_ered: np.ndarray
    _handle: ctypes.c_void_p = field(default=None, repr=False)

    def __post_init__(self):
        L = _lib.load()
        if self.prop not in PROPS:
            raise ValueError(self.prop)
        self.iprop = PROPS[self.prop]
        want = self.prop if self.prop.startswith("LDMG") else "LD"
        for g in self.segments:
            if g.kind != want:
                raise ValueError(f"a {self.prop} plan needs {want} segments, got {g.kind}")
        self.job_sys = np.ascontiguousarray(self.job_sys, dtype=np.int32)
        self.job_ered = np.ascontiguousarray(self.job_ered, dtype=np.float64)
        ns = len(self.systems)
        cs = (Coupling_C * ns)(*[c.c_struct() for c in self.systems])
        gs = (Grid_C * ns)(*[g.c_struct() for g in self.segments])
        h = ctypes.c_void_p()
        rc = L.mgpu_plan_create(ctypes.byref(h), self.iprop, ns, cs, gs, len(self.job_sys),
                                self.job_sys.ctypes.data_as(_ip), self.job_ered.ctypes.data_as(_dp))
        if rc != 0:
            raise PropagatorError(f"plan: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        self._handle = h
        self.y_elems = int(L.mgpu_plan_y_elems(h))
        self.offsets = np.array([L.mgpu_plan_y_offset(h, j) for j in range(len(self.job_sys))], dtype=np.int64)
        self.flops = float(L.mgpu_plan_flops(h))
        self.shared_systems = int(L.mgpu_plan_shared_systems(h))
        self.launches = int(L.mgpu_plan_launches(h))
        self.flops_prep = float(L.mgpu_plan_flops_phase(h, 1))
        self.flops_prop = float(L.mgpu_plan_flops_phase(h, 2))

    @property
    def njobs(self) -> int:
        return len(self.job_sys)

    def pack(self, ys: Sequence[np.ndarray]) -> np.ndarray:
        buf = np.empty(self.y_elems)
        for j, y in enumerate(ys):
            n = self.systems[self.job_sys[j]].n
            buf[self.offsets[j]:self.offsets[j] + n * n] = np.asarray(y, dtype=np.float64).ravel(order="F")
        return buf

    def unpack(self, buf: np.ndarray, j: int) -> np.ndarray:
        n = self.systems[self.job_sys[j]].n
        return buf[self.offsets[j]:self.offsets[j] + n * n].reshape((n, n), order="F")

    def nopen(self, j: int) -> int:
        """Open channels of job j (ERED above the threshold)."""
        return int(_lib.load().mgpu_plan_nopen(self._handle, int(j)))

    def run_host_smatrix(self, ybuf: np.ndarray):
        """Host Y in; the propagation, then Y -> K -> S on the device.  Returns
        (SR buffer, SI buffer, NODES, status, kfail); unpack_s gives job j's
        NOPEN x NOPEN matrices in CHNSRT channel order."""
        L = _lib.load()
        nj = self.njobs
        ns = int(L.mgpu_plan_s_elems(self._handle))
        y = np.ascontiguousarray(ybuf, dtype=np.float64)
        sr = np.zeros(max(ns, 1))
        si = np.zeros(max(ns, 1))
        nodes = np.zeros(nj, dtype=np.int32)
        status = np.zeros(nj, dtype=np.int32)
        kfail = np.zeros(nj, dtype=np.int32)
        rc = L.mgpu_plan_run_host_smatrix(self._handle, y.ctypes.data_as(_dp), sr.ctypes.data_as(_dp),
                                          si.ctypes.data_as(_dp), nodes.ctypes.data_as(_ip),
                                          status.ctypes.data_as(_ip), kfail.ctypes.data_as(_ip))
        if rc != 0:
            raise PropagatorError(f"run (S): {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        return sr, si, nodes, status, kfail

    def set_asymptote(self, sys: int, eint, cent, evec=None, rmatch: float | None = None):
        """YTRANS's output for system ``sys`` (molscat_b200.ytrans): the
        asymptotic channels' thresholds EINT and L(L+1) values CENT, the basis
        EVEC (columns; None if Y is already in it) and the matching radius
        (default: the segment's last radius).  Y -> S then transforms Y to
        that basis and matches there; NOPEN and the S layout follow."""
        L = _lib.load()
        n = self.systems[sys].n
        e = np.ascontiguousarray(eint, dtype=np.float64).reshape(n)
        c = np.ascontiguousarray(cent, dtype=np.float64).reshape(n)
        v = None if evec is None else np.asfortranarray(np.asarray(evec, dtype=np.float64).reshape(n, n))
        r = float(self.segments[sys].rtab[-1]) if rmatch is None else float(rmatch)
        rc = L.mgpu_plan_set_asymptote(self._handle, int(sys), e.ctypes.data_as(_dp), c.ctypes.data_as(_dp),
                                       None if v is None else v.ravel(order="F").ctypes.data_as(_dp), r)
        if rc != 0:
            raise PropagatorError(f"asymptote: {_lib.status_string(rc)}: {_lib.last_error()}", rc)

    def smatrix_host(self, ybuf: np.ndarray, status=None):
        """Y -> K -> S on the device from host matrices at the matching radius
        (the plan's Y layout).  Returns (SR buffer, SI buffer, status)."""
        L = _lib.load()
        ns = int(L.mgpu_plan_s_elems(self._handle))
        y = np.ascontiguousarray(ybuf, dtype=np.float64)
        sr = np.zeros(max(ns, 1))
        si = np.zeros(max(ns, 1))
        st = np.zeros(self.njobs, dtype=np.int32) if status is None else np.array(status, dtype=np.int32)
        rc = L.mgpu_plan_smatrix_host(self._handle, y.ctypes.data_as(_dp), sr.ctypes.data_as(_dp),
                                      si.ctypes.data_as(_dp), st.ctypes.data_as(_ip))
        if rc != 0:
            raise PropagatorError(f"S: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        return sr, si, st

    def unpack_s(self, buf: np.ndarray, j: int) -> np.ndarray:
        no = self.nopen(j)
        off = int(_lib.load().mgpu_plan_s_offset(self._handle, int(j)))
        return buf[off:off + no * no].reshape((no, no), order="F")

    def match_counts(self, pairs) -> np.ndarray:
        """After run_host: for each (a, b) job pair, the number of negative
        eigenvalues of Y_a - Y_b from an LDL^T inertia on the device (the
        matching count of bdctrl.f:221-257); -1 where a pivot was exactly zero
        or not finite (count those from the eigenvalues)."""
        L = _lib.load()
        pr = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
        out = np.zeros(pr.shape[0], dtype=np.int32)
        rc = L.mgpu_plan_match_counts(self._handle, pr.shape[0], pr.ctypes.data_as(_ip), out.ctypes.data_as(_ip))
        if rc != 0:
            raise PropagatorError(f"matching: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        return out

    def run_host(self, ybuf: np.ndarray):
        """Host buffers in and out.  Returns (Y buffer, NODES, status, kfail)."""
        L = _lib.load()
        y = np.ascontiguousarray(ybuf, dtype=np.float64).copy()
        nj = self.njobs
        nodes = np.zeros(nj, dtype=np.int32)
        status = np.zeros(nj, dtype=np.int32)
        kfail = np.zeros(nj, dtype=np.int32)
        rc = L.mgpu_plan_run_host(self._handle, y.ctypes.data_as(_dp), nodes.ctypes.data_as(_ip),
                                  status.ctypes.data_as(_ip), kfail.ctypes.data_as(_ip))
        if rc != 0:
            raise PropagatorError(f"run: {_lib.status_string(rc)}: {_lib.last_error()}", rc)
        return y, nodes, status, kfail

    def run_device(self, y_ptr: int, nodes_ptr: int, status_ptr: int, kfail_ptr: int, stream: int = 0,
                   phases: int = 3):
        """Device buffers (raw pointers, e.g. torch ``data_ptr()``), async on
        ``stream``.  phases: 1 = LDMD preparation only, 2 = propagation only."""
        L = _lib.load()
        rc = L.mgpu_plan_run_device_phases(self._handle, ctypes.c_void_p(y_ptr), ctypes.c_void_p(nodes_ptr),
                                           ctypes.c_void_p(status_ptr), ctypes.c_void_p(kfail_ptr),
                                           ctypes.c_void_p(stream), int(phases))
        if rc != 0:
            raise PropagatorError(f"run: {_lib.status_string(rc)}: {_lib.last_error()}", rc)

    def cancel(self, on: bool = True):
        """Stop this plan's runs (in flight or later) with MGPU_ERR_CANCELLED
        at the step kernels' next poll; cancel(False) clears the request.
        Safe from another thread while run_host is waiting."""
        rc = _lib.load().mgpu_plan_cancel(self._handle, 1 if on else 0)
        if rc != 0:
            raise PropagatorError(f"cancel: {_lib.status_string(rc)}", rc)

    def set_time_limit(self, seconds: float):
        """Stop jobs of a step kernel that runs longer than `seconds` with
        MGPU_ERR_DEADLINE (0: no limit)."""
        rc = _lib.load().mgpu_plan_set_time_limit(self._handle, float(seconds))
        if rc != 0:
            raise PropagatorError(f"time limit: {_lib.status_string(rc)}: {_lib.last_error()}", rc)

    def close(self):
        if self._handle:
            _lib.load().mgpu_plan_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
