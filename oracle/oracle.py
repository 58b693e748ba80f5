"""CPU ORACLE -- TEST INFRASTRUCTURE ONLY.

Python side of the oracle: a ctypes binding of the plain-C restatement in
``oracle_core.c`` (SYMINV, HAMMAT/SUMLAM, MDPROP, LDPROP) plus numpy
restatements of the host-side MOLSCAT pieces that surround the propagator,
so that whole S matrices can be compared with the reference's printed
example outputs:

* physical constants ............ source_code/physical_constants_module.f:8-87
* ITYPE=1 channel basis ......... source_code/base.f:276-345 (ordered on L)
* EINT / CENT ................... source_code/base.f:388-410
* Percival-Seaton couplings ..... source_code/couple.f:52-133
* power/exponential P(R) ........ source_code/potenl.f (evaluation case 1)
* HAMMAT scaling of P ........... source_code/hammat.f:31-83
* FINDRM (IRMSET>0) ............. source_code/findrm.f:1-259
* ITYPE=6 basis, couplings ...... oracle/itype6.py (asrot.f, set6c.f, set6.f)
* DRSET fixed step .............. source_code/drset.f:29-84
* CALCK / GTWVEC / CHNSRT ....... calck.f, gtwvec.f, chnsrt.f
* YINIT (adiabatic, WKB) ........ source_code/yinit.f:66-150
* YTOK / YTOKG / KSYM / KTOS .... ytok.f, ytokg.f, ksym.f, ktos.f

Nothing in the product imports this module.  Only the tests, the smoke
check and bench.py's CPU-baseline leg use it, and only as the checker.
"""
from __future__ import annotations

import ctypes
import glob
import math
import os
import subprocess
from dataclasses import dataclass, field
from fractions import Fraction
from functools import lru_cache

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile oracle_core.c into oracle/liboracle.so (plain gcc)."""
    src = os.path.join(_HERE, "oracle_core.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


def _openblas_path() -> str:
    import scipy  # noqa: F401  (locates the wheel's bundled OpenBLAS)
    libs = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libs, "libscipy_openblas*.so*")))
    if not cands:
        raise RuntimeError("scipy-bundled OpenBLAS not found (needed for DSYTRF/DSYTRI)")
    return cands[0]


def lib():
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = ctypes.CDLL(_LIB_PATH)
    blas = ctypes.CDLL(_openblas_path())
    L.oracle_set_lapack.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.oracle_set_lapack(ctypes.cast(blas.scipy_dsytrf_, ctypes.c_void_p),
                        ctypes.cast(blas.scipy_dsytri_, ctypes.c_void_p))
    L._blas = blas
    L.oracle_syminv.argtypes = [_dp, ctypes.c_int, ctypes.c_int]
    L.oracle_syminv.restype = ctypes.c_int
    prop_args = [ctypes.c_int] * 6 + [ctypes.c_double, _dp, _ip, _dp, _dp, _dp, _dp,
                                      ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      _dp, _ip, _ip]
    for name in ("oracle_mdprop", "oracle_ldprop"):
        f = getattr(L, name)
        f.argtypes = prop_args
        f.restype = ctypes.c_int
    L.oracle_hammat.argtypes = [ctypes.c_int] * 6 + [ctypes.c_double, _dp, _ip, _dp, _dp,
                                                     ctypes.c_double, _dp, ctypes.c_double, _dp]
    L.oracle_hammat.restype = None
    _lib = L
    return L


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


# --------------------------------------------------------------------------
# Boundary data: the propagator's inputs, laid out exactly as the reference
# passes them (VL(NVLBLK, N(N+1)/2) packed upper-by-columns, IV the same
# shape, Fortran 1-based P indices).
# --------------------------------------------------------------------------
@dataclass
class Coupling:
    n: int
    nham: int
    vl: np.ndarray            # float64, NVLBLK * N(N+1)/2
    eint: np.ndarray          # float64, N (reduced units)
    cent: np.ndarray          # float64, N (L(L+1))
    nvlblk: int = 0
    iv: np.ndarray | None = None   # int32, same length as vl (IVLFL>0 only)
    ivlfl: int = 0
    nconst: int = 0
    nrsq: int = 0
    conlen: float = 0.0

    def __post_init__(self):
        if self.nvlblk == 0:
            self.nvlblk = self.nham
        self.vl = np.ascontiguousarray(self.vl, dtype=np.float64)
        self.eint = np.ascontiguousarray(self.eint, dtype=np.float64)
        self.cent = np.ascontiguousarray(self.cent, dtype=np.float64)
        if self.iv is None:
            self.iv = np.zeros(1, dtype=np.int32)
        self.iv = np.ascontiguousarray(self.iv, dtype=np.int32)


def syminv(a: np.ndarray):
    """SYMINV on a copy of ``a`` (lower triangle read). Returns (inverse, kount)."""
    L = lib()
    n = a.shape[0]
    f = np.array(a, dtype=np.float64, order="F", copy=True)
    k = L.oracle_syminv(f.ctypes.data_as(_dp), n, n)
    return f, k


def hammat(c: Coupling, r: float, p: np.ndarray, ered: float) -> np.ndarray:
    L = lib()
    w = np.zeros((c.n, c.n), dtype=np.float64, order="F")
    p = np.ascontiguousarray(p, dtype=np.float64)
    L.oracle_hammat(c.n, c.nham, c.nvlblk, c.ivlfl, c.nconst, c.nrsq, c.conlen,
                    _p(c.vl), _p(c.iv, _ip), _p(c.eint), _p(c.cent), r, _p(p), ered, _p(w))
    return w


def _propagate(name: str, c: Coupling, rtab, ptab, nstep: int, dr: float, ered: float, y0):
    L = lib()
    rtab = np.ascontiguousarray(rtab, dtype=np.float64)
    ptab = np.ascontiguousarray(ptab, dtype=np.float64)
    assert rtab.shape[0] == 2 * nstep + 1 and ptab.shape == (2 * nstep + 1, c.nham)
    y = np.array(y0, dtype=np.float64, order="F", copy=True)
    nodes = ctypes.c_int(0)
    kfail = ctypes.c_int(0)
    st = getattr(L, name)(c.n, c.nham, c.nvlblk, c.ivlfl, c.nconst, c.nrsq, c.conlen,
                          _p(c.vl), _p(c.iv, _ip), _p(c.eint), _p(c.cent), _p(rtab), _p(ptab),
                          nstep, dr, ered, _p(y), ctypes.byref(nodes), ctypes.byref(kfail))
    return y, nodes.value, st, kfail.value


def mdprop(c: Coupling, rtab, ptab, nstep, dr, ered, y0):
    """MDPROP restatement. Returns (Y, NODES, status, failing KSTEP)."""
    return _propagate("oracle_mdprop", c, rtab, ptab, nstep, dr, ered, y0)


def ldprop(c: Coupling, rtab, ptab, nstep, dr, ered, y0):
    """LDPROP restatement. Returns (Z->Y, NODES, status, failing ISTEP)."""
    return _propagate("oracle_ldprop", c, rtab, ptab, nstep, dr, ered, y0)


# Symplectic integrator coefficients a_k (R advances by a_k h) and b_k (the
# W kick), Table I of D. E. Manolopoulos and S. K. Gray, J. Chem. Phys. 102,
# 9214 (1995): CS4 (five stages, a_5 = 0) and McLachlan-Atela's MA5 (six).
MG_COEFFS = {
    4: ((0.20517766154229, 0.40302128160421, -0.12092087633891, 0.51272193319241, 0.0),
        (0.061758858135626, 0.33897802655364, 0.61479130717558, -0.14054801465937, 0.12501982279453)),
    5: ((0.33983962583911, -0.088601336903027, 0.58585647682596, -0.60303935653649, 0.32358079655470,
         0.44236379421975),
        (0.11939002928757, 0.69892737038248, -0.17131235827160, 0.40126950225135, 0.010705081848236,
         -0.058979625498031)),
}


def mgprop(c: Coupling, sysm, rstart: float, dr: float, nstep: int, ered: float, y0, imgsel: int = 4):
    """MGPROP (mgprop.f:63-134) restated: per sector, stage k forms
    X = Y + b_k h W(R) and, where a_k != 0, Y = [I - (I + a_k h X)^-1]/(a_k h),
    adding the negative pivots of I + a_k h X to NODES (subtracting them for
    a_k < 0); R advances by a_k h.  Returns (Y, NODES)."""
    a, b = MG_COEFFS[imgsel]
    m = len(a)
    n = c.n
    y = np.array(y0, dtype=np.float64)
    nodes = 0
    eye = np.eye(n)
    w = None
    for s in range(nstep):
        r = rstart + s * dr
        for k in range(m):
            # with a_M = 0 the last stage's W (at the accumulated end of the
            # previous sector) serves as this sector's first (mgprop.f:82-93)
            if not (k == 0 and s > 0 and a[m - 1] == 0.0):
                w = hammat(c, r, sysm.pvec(r), ered)
            x = y + (b[k] * dr) * w
            if a[k] != 0.0:
                inv, cnt = syminv((a[k] * dr) * x + eye)
                inv = np.tril(inv) + np.tril(inv, -1).T
                nodes += cnt if a[k] >= 0.0 else -cnt
                y = (eye - inv) * (1.0 / (a[k] * dr))
            else:
                y = x
            r = r + a[k] * dr
    return 0.5 * (y + y.T), nodes


def maprop(c: Coupling, sysm, rstart: float, dr: float, nstep: int, ered: float, y0):
    """MAPROP (maprop.f:33-290) restated: the quasi-adiabatic log-derivative
    propagator.  Per sector: W at the midpoint (ERED = 0) diagonalised; the
    first-order corrections (W(R_start) - W(R_mid)) DR/6 at the sector's start
    and (W(R_end) - W(R_mid)) DR/6 carried from the previous end, added to Y
    in the old adiabatic basis; Y turned into the new one (Q = T_old^T U); the
    diagonal half-angle sector propagators of EIVAL - ERED; nodes from the
    inversion unless a channel is deeper than 24/DR^2 (NCHECK).  Returns (Y
    in the primitive basis, NODES)."""
    n = c.n
    eye = np.eye(n)
    y = np.array(y0, dtype=np.float64)
    t = eye.copy()
    q = np.zeros((n, n))
    r = rstart
    u = hammat(c, r, sysm.pvec(r), 0.0)
    nodes = 0
    wmax = 24.0 / (dr * dr)
    for k in range(nstep):
        r = r + 0.5 * dr
        w = hammat(c, r, sysm.pvec(r), 0.0)
        corr = (u - w) * (dr / 6.0) + q
        y = y + t.T @ corr @ t
        ev, vec = np.linalg.eigh(w)
        qm = t.T @ vec
        t = vec
        y = qm.T @ y @ qm
        wref = ev - ered
        flam = 0.5 * np.sqrt(np.abs(wref))
        y1 = np.empty(n)
        y2 = np.empty(n)
        neg = wref < 0.0
        tn = np.tan(flam[neg] * dr)
        y1[neg] = flam[neg] / tn - flam[neg] * tn
        y2[neg] = flam[neg] / tn + flam[neg] * tn
        th = np.tanh(flam[~neg] * dr)
        y1[~neg] = flam[~neg] / th + flam[~neg] * th
        y2[~neg] = flam[~neg] / th - flam[~neg] * th
        ncheck = int(np.sum(wref[~neg] > wmax))
        inv, cnt = syminv(y + np.diag(y1))
        if cnt > n:
            raise RuntimeError(f"MAPROP: matrix inversion error at step {k + 1}")
        inv = np.tril(inv) + np.tril(inv, -1).T
        if rstart > rstart + dr:  # inward
            cnt = n - cnt
        if ncheck == 0:
            nodes += cnt
        y = -(y2[:, None] * inv * y2[None, :]) + np.diag(y1)
        r = r + 0.5 * dr
        u = hammat(c, r, sysm.pvec(r), 0.0)
        q = (u - w) * (dr / 6.0)
    y = t @ y @ t.T + q
    return 0.5 * (y + y.T), nodes


def radial_grid(rstart: float, dr: float, nstep: int) -> np.ndarray:
    """Radii in the order MDPROP/LDPROP visit them: R=RSTART, then R=R+H
    repeated (mdprop.f:69,117,203; ldprop.f:30,57,105)."""
    h = dr / 2.0
    r = np.empty(2 * nstep + 1)
    x = rstart
    r[0] = x
    for k in range(1, 2 * nstep + 1):
        x = x + h
        r[k] = x
    return r


# --------------------------------------------------------------------------
# physical constants (physical_constants_module.f)
# --------------------------------------------------------------------------
PLANCK = 6.62607015e-34
CLIGHT = 2.99792458e8
AMU = 1.66053906892e-27
PI = 3.141592653589793
HBAR = PLANCK / 2.0 / PI
BFCT = HBAR / (4.0 * PI * (CLIGHT * 1.0e2)) / (1.0e-10) ** 2 / AMU
HARTREE_CM = 2.1947463136314e5
BOHR_ANG = 0.529177210544


# --------------------------------------------------------------------------
# angular momentum algebra (exact Racah formulae, own implementation)
# --------------------------------------------------------------------------
@lru_cache(maxsize=None)
def _fact(n: int) -> int:
    return math.factorial(n)


def _delta2(a, b, c) -> Fraction:
    return Fraction(_fact(a + b - c) * _fact(a - b + c) * _fact(-a + b + c), _fact(a + b + c + 1))


def _tri(a, b, c) -> bool:
    return abs(a - b) <= c <= a + b


@lru_cache(maxsize=None)
def threej000(j1: int, j2: int, j3: int) -> float:
    """(j1 j2 j3; 0 0 0) for integer j."""
    J = j1 + j2 + j3
    if J % 2 or not _tri(j1, j2, j3):
        return 0.0
    g = J // 2
    r2 = Fraction(_fact(J - 2 * j1) * _fact(J - 2 * j2) * _fact(J - 2 * j3), _fact(J + 1))
    pre = Fraction(_fact(g), _fact(g - j1) * _fact(g - j2) * _fact(g - j3))
    val = math.sqrt(r2) * float(pre)
    return -val if g % 2 else val


@lru_cache(maxsize=None)
def sixj(a: int, b: int, c: int, d: int, e: int, f: int) -> float:
    """{a b c; d e f} for integer arguments (Racah's single-sum formula)."""
    if not (_tri(a, b, c) and _tri(a, e, f) and _tri(d, b, f) and _tri(d, e, c)):
        return 0.0
    pref2 = _delta2(a, b, c) * _delta2(a, e, f) * _delta2(d, b, f) * _delta2(d, e, c)
    tmin = max(a + b + c, a + e + f, d + b + f, d + e + c)
    tmax = min(a + b + d + e, a + c + d + f, b + c + e + f)
    s = 0
    for t in range(tmin, tmax + 1):
        num = _fact(t + 1)
        den = (_fact(t - a - b - c) * _fact(t - a - e - f) * _fact(t - d - b - f) * _fact(t - d - e - c)
               * _fact(a + b + d + e - t) * _fact(a + c + d + f - t) * _fact(b + c + e + f - t))
        s += Fraction((-1) ** t * num, den)
    if s == 0:
        return 0.0
    # value = sqrt(pref2) * s ; do it as sqrt(pref2 * s^2) with sign to keep precision
    return math.copysign(math.sqrt(pref2 * s * s), float(s))


# --------------------------------------------------------------------------
# ITYPE=1 atom + rigid linear rotor
# --------------------------------------------------------------------------
@dataclass
class Itype1:
    """MOLSCAT ITYPE=1 system: &BASIS (BE, JLEVEL) + &POTL power/exp terms."""
    ured: float
    be: float
    jlevel: list
    lam: list                 # LAMBDA per expansion term
    terms: list               # per term: list of (A, NPOWER, E or None)
    rm: float                 # RM (Angstrom) = RUNIT
    epsil: float              # EPSIL (cm-1)

    @property
    def cm2ru(self) -> float:
        # mol.driver.f:734 CM2RU=URED*MUNIT*RUNIT*RUNIT/BFCT with MUNIT=1
        return self.ured * 1.0 * self.rm * self.rm / BFCT

    @property
    def ep2ru(self) -> float:
        return self.epsil * self.cm2ru

    def elevel(self, j: int) -> float:
        return self.be * j * (j + 1)

    def channels(self, jtot: int, block: int):
        """(jsindx, L) lists, base.f:276-345: L outer, states inner, parity
        IPTY = block mod 2 on L+j+JTOT."""
        ipty = block % 2
        jmax = max(self.jlevel)
        jmin = min(self.jlevel)
        lmax = jtot + jmax
        lmin = jtot - jmax
        if lmin < 0:
            lmin = max(jmin - jtot, 0)
        out = []
        for li in range(lmin, lmax + 1):
            jk = abs(jtot - li)
            jtop = jtot + li
            for i, ji in enumerate(self.jlevel):
                lpj = li + ji + jtot
                if lpj % 2 != ipty:
                    continue
                if ji < jk or ji > jtop:
                    continue
                out.append((i, li))
        return out

    def coupling(self, jtot: int, block: int) -> Coupling:
        ch = self.channels(jtot, block)
        n = len(ch)
        nham = len(self.lam)
        vl = np.zeros(nham * n * (n + 1) // 2)
        idx = 0
        for icol in range(n):
            jc = self.jlevel[ch[icol][0]]
            lc = ch[icol][1]
            for irow in range(icol + 1):
                jr = self.jlevel[ch[irow][0]]
                lr = ch[irow][1]
                for t, lam in enumerate(self.lam):
                    v = (math.sqrt((2 * jc + 1) * (2 * jr + 1) * (2 * lc + 1) * (2 * lr + 1))
                         * threej000(jc, lam, jr) * threej000(lc, lam, lr)
                         * sixj(jr, lr, jtot, lc, jc, lam))
                    if (jc + jr + jtot) % 2:
                        v = -v
                    vl[idx + t] = v
                idx += nham
        eint = np.array([self.cm2ru * self.elevel(self.jlevel[i]) for i, _ in ch])
        cent = np.array([float(l * (l + 1)) for _, l in ch])
        return Coupling(n=n, nham=nham, vl=vl, eint=eint, cent=cent)

    def potenl(self, r: float) -> np.ndarray:
        """POTENL case 1 (R in units of RM, result in units of EPSIL)."""
        p = np.zeros(len(self.lam))
        for t, tl in enumerate(self.terms):
            tot = 0.0
            for a, npw, e in tl:
                if npw != 0:
                    rr = r
                    if npw < 0 and abs(r) < 1.0e-8:
                        rr = 1.0e-8
                    term = rr ** npw
                else:
                    term = math.exp(e * r)
                tot = tot + a * term
            p[t] = tot
        return p

    def pvec(self, r: float) -> np.ndarray:
        """The P vector SUMLAM receives (hammat.f:37-83 with no NCONST/NRSQ)."""
        p = self.potenl(r)
        p = np.where(np.abs(p) > 1.0e60, np.sign(p) * 1.0e60, p)
        return self.ep2ru * p


def ptable(sysm, rtab) -> np.ndarray:
    return np.stack([sysm.pvec(float(r)) for r in rtab])


def lowest_adiabat(sysm, c: Coupling, r: float, ered: float) -> float:
    w = hammat(c, r, sysm.pvec(r), ered)
    return float(np.linalg.eigvalsh(w)[0])


def findrm(sysm, c: Coupling, rstart: float, ered: float, irmset: int = 9, bound: bool = False):
    """FINDRM (findrm.f:43-250).  Returns (RSTART, RTURN).  MOLSCAT starts
    the secant search from the smallest centrifugal turning point of the open
    channels (findrm.f:40-57); BOUND and FIELD (bound=True) start it at the
    input RSTART with one try only (findrm.f:31-38).  Where the reference's
    BOUND branch would fall back to its (unset) RMIN, this returns the input
    RSTART."""
    rmin = rstart
    if bound:
        rturn = rstart
        itry = 1
    else:
        rturn = 1.0e30
        for i in range(c.n):
            dif = ered - c.eint[i]
            if dif < 0.0:
                continue
            rcent = math.sqrt(c.cent[i] / dif)
            rcent = max(rcent, rmin)
            rturn = min(rturn, rcent)
        itry = 0
        if rturn == rmin:
            itry = 1
    while True:  # label 10
        itry += 1
        rstart = rturn
        if itry > 25:
            return rmin, rturn
        diag1 = lowest_adiabat(sysm, c, rstart, ered)
        rturn = 0.999 * rstart
        converged = False
        retry = False
        for _ in range(100):
            diag2 = lowest_adiabat(sysm, c, rturn, ered)
            v2 = diag2
            dv1 = (diag2 - diag1) / (rturn - rstart)
            diag1 = diag2
            if dv1 >= 0.0:
                if itry == 1:
                    rturn = rmin
                    retry = True
                    break
                return rmin, 2.0 * rmin
            rstart = rturn
            v1 = v2
            dr = -v1 / dv1
            if dr < -0.3 * rturn:
                dr = -0.3 * rturn
            rturn = rturn + dr
            if dr > 1.0e3:
                break
            if rturn <= 0.0:
                break
            if abs(dr / rturn) <= 1.0e-3:
                converged = True
                break
        if retry:
            continue
        if not converged:
            return rmin, rturn
        break
    # phase integral inwards (findrm.f:160-245)
    nstep = 3 + irmset // 3
    target = 2.303 * float(irmset)
    dr = (1.5 * target / math.sqrt(abs(dv1)) / float(nstep)) ** (2.0 / 3.0)
    phase = 0.0
    xk2 = 0.0
    while True:  # label 220
        restart = False
        for istep in range(1, nstep + 1):
            rnext = rstart - dr
            if rnext < 0.0:
                return 0.0, rturn
            d = lowest_adiabat(sysm, c, rnext, ered)
            drnext = 0.0
            if d <= 0.0:
                raise RuntimeError("FINDRM: inner classically allowed region (not restated)")
            xk1 = math.sqrt(d)
            if istep == 1:
                phase = (2.0 / 3.0) * xk1 * dr
            else:
                xkavg = 0.5 * (xk1 + xk2)
                phase = phase + dr * xkavg
            drnext = max(drnext, (target - phase) / xk1)
            xk2 = xk1
            rstart = rnext
            if istep < nstep:
                dr = drnext / float(nstep - istep)
            if drnext <= 0.0:
                break
            if istep < nstep and dr > 0.5 * rstart and dr > 0.5 * rmin:
                dr = 0.02 * rstart
                restart = True
                break
        if not restart:
            return rstart, rturn


def nint(x: float) -> int:
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def calck(ep: float, ered: float, eint) -> float:
    k = 0.0
    for e in eint:
        if ep + ered - e <= 0.0:
            continue
        k = max(k, math.sqrt(ep + ered - e))
    return k


def drset_fixed(rstart: float, rstop: float, step: float, cay: float):
    """DRSET for a fixed-step propagator with STEP>0 (drset.f:29-84)."""
    rsmall = min(rstart, rstop)
    rlarge = max(rstart, rstop)
    prange = rlarge - rsmall
    drfit = math.acos(-1.0) / (cay * step)
    nstep = max(nint(prange / drfit), 1)
    dr = prange / float(nstep)
    if rstop < rstart:
        dr = -abs(dr)
    return nstep, dr


def yinit_adiabatic_wkb(sysm, c: Coupling, r: float, ered: float) -> np.ndarray:
    """YINIT with ADIAMN and WKBMN at RMIN (outward), all channels closed."""
    w = hammat(c, r, sysm.pvec(r), ered)
    ev, evec = np.linalg.eigh(w)
    if np.any(ev <= 0.0):
        raise RuntimeError("YINIT restatement: locally open channel at RMIN (BCYOMN path)")
    yl = np.sqrt(np.abs(ev))
    return (evec * yl) @ evec.T


def chnsrt(eint) -> list:
    n = len(eint)
    nb = list(range(n))
    for i in range(n - 1):
        for j in range(i + 1, n):
            if eint[nb[i]] <= eint[nb[j]]:
                continue
            if abs(eint[nb[i]] - eint[nb[j]]) < 1.0e-11:
                continue
            nb[i], nb[j] = nb[j], nb[i]
    return nb


def ricbes(ell: float, x: float):
    """Riccati-Bessel x j_l(x), x y_l(x) and their x-derivatives (integer l)."""
    from scipy.special import spherical_jn, spherical_yn
    l = int(round(ell))
    assert abs(ell - l) < 1e-12
    j = spherical_jn(l, x)
    jp = spherical_jn(l, x, derivative=True)
    yv = spherical_yn(l, x)
    yp = spherical_yn(l, x, derivative=True)
    return x * j, j + x * jp, x * yv, yv + x * yp


def rbessk_ratio(ell: float, x: float) -> float:
    """d/dx ln[sqrt(x) K_{l+1/2}(x)]  (rbessk.f:18-31)."""
    from scipy.special import kve
    v = ell + 0.5
    return -(kve(v - 1.0, x) + kve(v + 1.0, x)) / (2.0 * kve(v, x)) + 0.5 / x


def ytok(nb, wvec, n: int, nopen: int, y: np.ndarray, rval: float, cent) -> np.ndarray:
    """YTOK + YTOKG + KSYM (ytok.f:21-47; ytokg.f:71-126)."""
    sj = np.zeros(n); sjp = np.zeros(n); sn = np.zeros(n); snp = np.zeros(n)
    for i in range(nopen):
        nx = nb[i]
        dw = wvec[nx]
        ell = math.sqrt(cent[nx] + 0.25) - 0.5
        uj, ujp, un, unp = ricbes(ell, dw * rval)
        rd = math.sqrt(dw)
        sj[nx] = uj / rd; sjp[nx] = ujp * rd; sn[nx] = un / rd; snp[nx] = unp * rd
    for i in range(nopen, n):
        nx = nb[i]
        dw = abs(wvec[nx])
        ell = math.sqrt(cent[nx] + 0.25) - 0.5
        sn[nx] = 1.0
        snp[nx] = rbessk_ratio(ell, dw * rval) * dw
    yy = np.array(y)[np.ix_(nb, nb)]
    t = yy[:, :nopen] * sj[nb][None, :nopen]
    for i in range(nopen):
        t[i, i] -= sjp[nb[i]]
    km = yy * sn[nb][None, :]
    for i in range(n):
        km[i, i] -= snp[nb[i]]
    x = np.linalg.solve(km, t)
    k = x[:nopen, :nopen]
    return 0.5 * (k + k.T)


def ktos(k: np.ndarray):
    """KTOS (ktos.f:149-169): returns (SR, SI)."""
    nop = k.shape[0]
    sr = 0.5 * (k @ k) + 0.5 * np.eye(nop)
    srinv, _ = syminv(sr)
    srinv = np.tril(srinv) + np.tril(srinv, -1).T
    si = srinv @ k
    return srinv - np.eye(nop), si


def gtwvec(ered: float, eint):
    w = []
    nopen = 0
    for e in eint:
        dif = ered - e
        w.append(math.copysign(math.sqrt(abs(dif)), dif))
        if dif > 0.0:
            nopen += 1
    return np.array(w), nopen


@dataclass
class ScatteringResult:
    energy: float
    rstart: float
    nstep: int
    nodes: int
    nb: list
    nopen: int
    sr: np.ndarray
    si: np.ndarray
    y: np.ndarray = field(repr=False)


def molscat_smatrix(sysm: Itype1, jtot: int, block: int, energies, rmin: float, rmax: float,
                    steps: float, propagator: str = "LDMD", irmset: int = 9,
                    iscru: bool = True):
    """One (JTOT, block) of a MOLSCAT run with a single LDMD, LDJ or LDMG
    segment ("LDMG4" / "LDMG5": MGPROP with IMGSEL = 4 or 5, the same step
    count as the log-derivative propagators).

    Follows mol.driver.f:1141-1146,1453,1488-1549 (EREDMX = highest energy when
    ISCRU is set, FINDRM at EREDMX, CAYS = CALCK(0, EREDMX)) and scctrl.f
    (YINIT, propagator, YTOK, KTOS)."""
    c = sysm.coupling(jtot, block)
    cm2ru = sysm.cm2ru
    emx = max(energies) * cm2ru
    out = []
    rstart = nstep = dr = None
    for ie, e in enumerate(energies):
        ered = e * cm2ru
        eredmx = emx if iscru else ered
        if ie == 0 or not iscru:
            rstart, _ = findrm(sysm, c, rmin, eredmx, irmset)
            cay = calck(0.0, eredmx, c.eint)
            nstep, dr = drset_fixed(rstart, rmax, steps, cay)
        wvec, nopen = gtwvec(ered, c.eint)
        y0 = yinit_adiabatic_wkb(sysm, c, rstart, ered)
        rtab = radial_grid(rstart, dr, nstep)
        ptab = ptable(sysm, rtab)
        if propagator == "LDMD":
            y, nodes, st, kf = mdprop(c, rtab, ptab, nstep, dr, ered, y0)
        elif propagator == "LDJ":
            y, nodes, st, kf = ldprop(c, rtab, ptab, nstep, dr, ered, y0)
        elif propagator == "LDMA":
            y, nodes = maprop(c, sysm, rstart, dr, nstep, ered, y0)
            st, kf = 0, 0
        elif propagator in ("LDMG4", "LDMG5"):
            y, nodes = mgprop(c, sysm, rstart, dr, nstep, ered, y0, int(propagator[-1]))
            st, kf = 0, 0
            rtab = np.array([rstart, rstart + nstep * dr])
        else:
            raise ValueError(propagator)
        if st != 0:
            raise RuntimeError(f"{propagator}: inversion error at step {kf}")
        nb = chnsrt(c.eint)
        k = ytok(nb, wvec, c.n, nopen, y, rtab[-1], c.cent)
        sr, si = ktos(k)
        out.append(ScatteringResult(e, rstart, nstep, nodes, nb, nopen, sr, si, y))
    return out
