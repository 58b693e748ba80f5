"""CPU ORACLE -- TEST INFRASTRUCTURE ONLY.

MOLSCAT ITYPE=6 (atom + rigid asymmetric top) host-side pieces, restated in
numpy so that the propagator's inputs for the large-N workload come from the
reference's own basis and coupling algebra:

* rotor levels and functions .... source_code/asrot.f:38-66 (H in the |J K>
  basis: diagonal alpha J(J+1) + beta K^2 - DJ, DJK, DK distortion, plus the
  tetrahedral DT terms of a spherical top; K, K+-2 gamma terms; K, K+-4 DT
  terms), the symmetry code of ipasym.f:5-12 and the selection of
  set6c.f:57-220 (ISYM(1) bits, degeneracy, EMAX, level bookkeeping)
* channel basis ................. source_code/base.f:276-345 (ITP = 6 branch,
  ordered on L, parity on IPLEV + IPLEV/2 + J + L + JTOT)
* EINT / CENT ................... source_code/base.f:388-410
* couplings ..................... source_code/set6.f:117-263 (CPL6: the
  pair-state factor from the rotor coefficients and 3j symbols, then the
  channel VL from 3j(L L' lambda; 000) and 6j{J' L' JTOT; L J lambda})
* Buck MSV Ar-CH4 potential ..... source_code/vstar-Rg_CH4_Buck.f:14-108
  (the VSTAR/VINIT plug-in of the bound-Ar_CH4 example)

Diagonalisation: H conserves the parity of K and the symmetry under
K -> -K, so each J is diagonalised in the four Wang blocks (even/odd K,
symmetric/antisymmetric in K -> -K).  Every rotor function then has a
definite IPASYM code by construction, which is what the reference's DMSYM
enforces on degenerate sets after a full diagonalisation; the energies and
the space each symmetry selection keeps are the same.  Where the signs or
the order of degenerate functions differ from the reference's choice, only
the labels (TAU) and the signs of some couplings change, not the propagated
physics (node counts, bound-state energies, |S|).

Bits 8 and 9 of ISYM(1) (K a multiple of 3) have no effect in the
reference (their CYCLE statements sit inside an inner loop over K,
set6c.f:160-170), and none here.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction
from functools import lru_cache

import numpy as np

from . import oracle as O


# ---------------------------------------------------------------------------
# 3j symbols with projections (own implementation of Racah's formula)
# ---------------------------------------------------------------------------
@lru_cache(maxsize=None)
def threej(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """(j1 j2 j3; m1 m2 m3), integer arguments."""
    if m1 + m2 + m3 != 0 or abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    if not (abs(j1 - j2) <= j3 <= j1 + j2):
        return 0.0
    f = O._fact
    pre2 = Fraction(f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3), f(j1 + j2 + j3 + 1))
    pre2 *= (f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3))
    kmin = max(0, j2 - j3 - m1, j1 - j3 + m2)
    kmax = min(j1 + j2 - j3, j1 - m1, j2 + m2)
    s = Fraction(0)
    for k in range(kmin, kmax + 1):
        den = (f(k) * f(j1 + j2 - j3 - k) * f(j1 - m1 - k) * f(j2 + m2 - k) * f(j3 - j2 + m1 + k)
               * f(j3 - j1 - m2 + k))
        s += Fraction(-1 if k % 2 else 1, den)
    if s == 0:
        return 0.0
    val = math.sqrt(pre2 * s * s)
    if s < 0:
        val = -val
    return -val if (j1 - j2 - m3) % 2 else val


# ---------------------------------------------------------------------------
# rotor functions
# ---------------------------------------------------------------------------
def rotor_hamiltonian(j: int, roti) -> np.ndarray:
    """H(K, K') for K, K' = -J..J (asrot.f:38-63).  roti = (A, 0, B, 0, C,
    0, DJ, DJK, DK, DT) as &BASIS ROTI."""
    a, b, c = roti[0], roti[2], roti[4]
    dj, djk, dk, dt = roti[6], roti[7], roti[8], roti[9]
    alpha = 0.5 * (a + b)
    beta = c - alpha
    gamma = 0.25 * (a - b)
    td = (a == b) and (b == c)
    jj = j * (j + 1)
    nk = 2 * j + 1
    h = np.zeros((nk, nk))
    for ir in range(nk):
        kr = ir - j
        for ic in range(ir + 1):
            kc = ic - j
            t = 0.0
            if kr == kc:
                t = (alpha * jj + beta * kc * kc - dj * float(jj * jj) - djk * float(jj * kc * kc)
                     - dk * float(kc ** 4))
                if td:
                    t += 0.5 * dt * float(-3 * jj * (jj - 2) + 30 * (jj - 2) * kc * kc - 35 * kc * kc * (kc * kc - 1))
            elif kr - kc == 2:
                kmid = (kr + kc) // 2
                t = gamma * math.sqrt(float((jj - kr * kmid) * (jj - kc * kmid)))
            elif kr - kc == 4 and td:
                t = 1.25 * dt * math.sqrt(float((jj - kc * (kc + 1)) * (jj - (kc + 1) * (kc + 2)))
                                          * float((jj - (kc + 2) * (kc + 3)) * (jj - (kc + 3) * (kc + 4))))
            h[ir, ic] = t
            h[ic, ir] = t
    return h


def rotor_functions(j: int, roti):
    """Eigenpairs of H for one J, each with its symmetry code IPLEV =
    2*KPAR + IPAR (ipasym.f:5-12: KPAR 0/1 for even/odd K, IPAR 0/1 for
    coefficients symmetric/antisymmetric under K -> -K).  Returns a list of
    (energy, iplev, coefficients over K = -J..J) in ascending energy."""
    h = rotor_hamiltonian(j, roti)
    nk = 2 * j + 1
    out = []
    for kpar in (0, 1):
        for ipar in (0, 1):
            cols = []
            for k in range(0, j + 1):
                if k % 2 != kpar:
                    continue
                v = np.zeros(nk)
                if k == 0:
                    if ipar == 1:
                        continue
                    v[j] = 1.0
                else:
                    s = 1.0 if ipar == 0 else -1.0
                    v[j + k] = 1.0 / math.sqrt(2.0)
                    v[j - k] = s / math.sqrt(2.0)
                cols.append(v)
            if not cols:
                continue
            t = np.stack(cols, axis=1)
            hb = t.T @ h @ t
            ev, w = np.linalg.eigh(hb)
            vec = t @ w
            for i in range(ev.size):
                out.append((float(ev[i]), 2 * kpar + ipar, vec[:, i]))
    out.sort(key=lambda x: (x[0], x[1]))
    return out


@dataclass
class RotorState:
    j: int
    tau: int
    iplev: int
    level: int           # 0-based index into Itype6.elevel
    coef: np.ndarray     # coefficients over K = -J..J


@dataclass
class Itype6:
    """&BASIS ITYPE=6 with rotational constants (SET6C path) + a potential
    given as a list of (lambda, mu) terms and a radial function per term.

    pfunc(r) returns the MXLAM radial coefficients in units of EPSIL for R in
    units of RM (what POTENL returns before HAMMAT scales it by EP2RU)."""
    ured: float
    roti: tuple
    jmax: int
    lam: list            # [(lambda, mu), ...] of the MXLAM terms
    pfunc: object
    rm: float
    epsil: float
    jmin: int = 0
    emax: float = 0.0    # cm-1; <= 0 keeps every level
    isym: int = -1
    states: list = field(default_factory=list, init=False)
    elevel: list = field(default_factory=list, init=False)

    def __post_init__(self):
        self._select()
        self._pair = {}

    @property
    def cm2ru(self) -> float:
        return self.ured * 1.0 * self.rm * self.rm / O.BFCT

    @property
    def ep2ru(self) -> float:
        return self.epsil * self.cm2ru

    def _select(self):
        """Rotor functions kept in the basis (set6c.f:110-215)."""
        ip = [(self.isym >> b) & 1 if self.isym > 0 else 0 for b in range(10)]
        if ip[0] + ip[1] == 2 or ip[2] + ip[3] == 2 or ip[8] + ip[9] == 2 or sum(ip[4:8]) == 4:
            raise ValueError("ISYM combination leaves no basis functions")
        tol = 1.0e-8
        esave = -999.0
        nlvl = 0
        spherical_level_merge = self.roti[0] == self.roti[4]
        for j in range(self.jmin, self.jmax + 1):
            funcs = rotor_functions(j, self.roti)
            evals = np.array([f[0] for f in funcs])
            for ik, (elev, iplev, vec) in enumerate(funcs, start=1):
                if self.emax > 0.0 and elev > self.emax:
                    continue
                if self.isym > 0:
                    ideg = int(np.sum(np.abs(evals - elev) < tol))
                    if ip[0] and iplev >= 2:
                        continue
                    if ip[1] and iplev <= 1:
                        continue
                    if ip[2] and (iplev + j) % 2 == 1:
                        continue
                    if ip[3] and (iplev + j) % 2 == 0:
                        continue
                    if ip[4] and ideg == 1:
                        continue
                    if ip[5] and ideg == 2:
                        continue
                    if ip[6] and ideg == 3:
                        continue
                    if ip[7] and ideg > 3:
                        continue
                prev, esave = esave, elev
                if abs(esave - prev) > tol or not spherical_level_merge:
                    nlvl += 1
                    self.elevel.append(elev)
                self.states.append(RotorState(j, ik - 1 - j, iplev, nlvl - 1, vec))

    # -- channels ------------------------------------------------------------
    def channels(self, jtot: int, block: int):
        """[(state index, L)] for (JTOT, symmetry block): base.f:276-345 with
        ITP = 6, L outer and states inner."""
        ipty = block % 2
        lmax = jtot + self.jmax
        lmin = jtot - self.jmax
        if lmin < 0:
            lmin = max(self.jmin - jtot, 0)
        out = []
        for li in range(lmin, lmax + 1):
            jk, jtop = abs(jtot - li), jtot + li
            for i, s in enumerate(self.states):
                lpj = s.iplev + s.iplev // 2 + s.j + li + jtot
                if lpj % 2 != ipty:
                    continue
                if s.j < jk or s.j > jtop:
                    continue
                out.append((i, li))
        return out

    # -- couplings -------------------------------------------------------------
    def _kmatrix(self, jc: int, jr: int, lm: int, mu: int) -> np.ndarray:
        """M[KC, KR] with CPL(ic, ir) = a_c . M . a_r before the constant
        factor (set6.f:134-158): (-1)^KR times 3j(JC JR LM; KC -KR MU) where
        KR - KC = MU, plus (-1)^(KR+MU) 3j(JC JR LM; KC -KR -MU) where
        KC - KR = MU (once only for MU = 0)."""
        m = np.zeros((2 * jc + 1, 2 * jr + 1))
        for kc in range(-jc, jc + 1):
            for kr in range(-jr, jr + 1):
                sgn = -1.0 if kr % 2 else 1.0
                v = 0.0
                if kr - kc == mu:
                    v += sgn * threej(jc, jr, lm, kc, -kr, mu)
                    if mu == 0:
                        m[kc + jc, kr + jr] = v
                        continue
                if kc - kr == mu:
                    s2 = -sgn if mu % 2 else sgn
                    v += s2 * threej(jc, jr, lm, kc, -kr, -mu)
                m[kc + jc, kr + jr] = v
        return m

    def pair_coupling(self, t: int, ic: int, ir: int) -> float:
        """The pair-state factor CPL of term t between rotor states ic, ir."""
        key = (t, ic, ir) if ic >= ir else (t, ir, ic)
        if key in self._pair:
            return self._pair[key]
        lm, mu = self.lam[t]
        sc, sr = self.states[key[1]], self.states[key[2]]
        ac = np.where(np.abs(sc.coef) <= 1.0e-9, 0.0, sc.coef)
        ar = np.where(np.abs(sr.coef) <= 1.0e-9, 0.0, sr.coef)
        x = float(ac @ self._kmatrix(sc.j, sr.j, lm, mu) @ ar)
        fct = math.sqrt((2 * sc.j + 1) * (2 * sr.j + 1) * (2 * lm + 1) / (4.0 * math.pi))
        if (sc.j + sr.j) % 2:
            fct = -fct
        self._pair[key] = x * fct
        return self._pair[key]

    def coupling(self, jtot: int, block: int, nmax: int | None = None) -> O.Coupling:
        """VL(MXLAM, N(N+1)/2) (set6.f:186-260), EINT and CENT (base.f:388-410).

        VL of term (lambda, mu) between channels (c, L_c) and (r, L_r) is
        (-1)^JTOT sqrt((2L_c+1)(2L_r+1)) CPL(c, r) 3j(L_c lambda L_r; 000)
        6j{J_r L_r JTOT; L_c J_c lambda}.  The angular factor depends on the
        channels only through (J, L), so it is tabulated over the distinct
        (J, L) pairs and gathered.  nmax keeps the first nmax channels of the
        channel order (a truncation in L, not a reference option)."""
        ch = self.channels(jtot, block)
        if nmax is not None:
            ch = ch[:nmax]
        n = len(ch)
        nham = len(self.lam)
        st = np.array([c[0] for c in ch])
        ls = np.array([c[1] for c in ch])
        js = np.array([self.states[i].j for i in st])
        jl = sorted(set(zip(js.tolist(), ls.tolist())))
        q = {p: k for k, p in enumerate(jl)}
        qi = np.array([q[(int(j), int(l))] for j, l in zip(js, ls)])
        nst = len(self.states)
        used = sorted(set(st.tolist()))
        pjt = -1.0 if jtot % 2 else 1.0
        col = np.repeat(np.arange(n), np.arange(1, n + 1))      # SUMLAM pair order
        row = np.arange(n * (n + 1) // 2) - col * (col + 1) // 2
        sqrtl = np.sqrt(2.0 * ls + 1.0)
        vl = np.zeros((n * (n + 1) // 2, nham))
        for t, (lm, mu) in enumerate(self.lam):
            cpl = np.zeros((nst, nst))
            for a_ in used:
                for b_ in used:
                    if b_ <= a_:
                        cpl[a_, b_] = cpl[b_, a_] = self.pair_coupling(t, a_, b_)
            g = np.zeros((len(jl), len(jl)))
            for kc, (jc, lc) in enumerate(jl):
                for kr, (jr, lr) in enumerate(jl):
                    if (lr + lc + lm) % 2 or not (abs(lc - lm) <= lr <= lc + lm) or abs(jc - jr) > lm:
                        continue
                    g[kc, kr] = O.threej000(lc, lm, lr) * O.sixj(jr, lr, jtot, lc, jc, lm)
            vl[:, t] = (pjt * sqrtl[col] * sqrtl[row] * cpl[st[col], st[row]] * g[qi[col], qi[row]])
        eint = np.array([self.cm2ru * self.elevel[self.states[s_].level] for s_ in st])
        cent = (ls * (ls + 1)).astype(np.float64)
        return O.Coupling(n=n, nham=nham, vl=np.ascontiguousarray(vl.ravel()), eint=eint, cent=cent)

    def pvec(self, r: float) -> np.ndarray:
        """The P vector SUMLAM receives (hammat.f:37-83, no NCONST/NRSQ)."""
        p = np.asarray(self.pfunc(r), dtype=np.float64)[:len(self.lam)]
        p = np.where(np.abs(p) > 1.0e60, np.sign(p) * 1.0e60, p)
        return self.ep2ru * p


# ---------------------------------------------------------------------------
# the Buck MSV Ar-CH4 potential (VSTAR plug-in)
# ---------------------------------------------------------------------------
class BuckMSV:
    """Morse-spline-van der Waals isotropic term and the anisotropic
    exp/R^-n terms of Buck et al. (vstar-Rg_CH4_Buck.f): X is R in units
    of RM; term 1 is multiplied by sqrt(4 pi), term i > 1 has the order
    lambda_i of its (lambda, mu) pair."""

    def __init__(self, beta1, beta2, c6, c8, x1, x2, x3, x4, alphas, lams):
        self.beta1, self.beta2, self.c6, self.c8 = beta1, beta2, c6, c8
        self.x1, self.x2, self.x3, self.x4 = x1, x2, x3, x4
        self.alphas = alphas   # [(ALPHAR, ALPHAA)] for terms 2.. (already scaled)
        self.lams = lams       # lambda of terms 2..
        self.a = self._spline(x1, beta1, x2, beta2, lambda z: self._morse(z, beta2),
                              lambda z: self._dmorse(z, beta2))
        self.b = self._spline(x3, beta2, x4, None, self._disp, self._ddisp)
        self.ycfac = math.sqrt(4.0 * math.pi)

    @staticmethod
    def _morse(z, beta):
        return math.exp(2.0 * beta * (1.0 - z)) - 2.0 * math.exp(beta * (1.0 - z))

    @staticmethod
    def _dmorse(z, beta):
        return 2.0 * beta * (math.exp(beta * (1.0 - z)) - math.exp(2.0 * beta * (1.0 - z)))

    def _disp(self, x):
        y = 1.0 / (x * x)
        return -(self.c6 + self.c8 * y) * y ** 3

    def _ddisp(self, x):
        y = 1.0 / (x * x)
        return (6.0 * self.c6 + 8.0 * self.c8 * y) * y ** 3 / x

    def _spline(self, xl, betal, xr, _betar, fr, dfr):
        """Cubic a0 + a1 y + a2 y^2 + a3 y^3 (y = x - xl) matching value and
        slope of the Morse curve (beta of the left end) at xl and of fr at xr."""
        vl, vlp = self._morse(xl, betal), self._dmorse(xl, betal)
        vr, vrp = fr(xr), dfr(xr)
        y = xr - xl
        a2 = 3.0 * (vr - vl) / y ** 2 - (2.0 * vlp + vrp) / y
        a3 = 2.0 * (vl - vr) / y ** 3 + (vlp + vrp) / y ** 2
        return (vl, vlp, a2, a3)

    def iso(self, x: float) -> float:
        if x <= self.x1:
            s = self._morse(x, self.beta1)
        elif x < self.x2:
            y = x - self.x1
            a0, a1, a2, a3 = self.a
            s = a0 + y * (a1 + y * (a2 + y * a3))
        elif x <= self.x3:
            s = self._morse(x, self.beta2)
        elif x < self.x4:
            y = x - self.x3
            b0, b1, b2, b3 = self.b
            s = b0 + y * (b1 + y * (b2 + y * b3))
        else:
            s = self._disp(x)
        return s * self.ycfac

    def aniso(self, i: int, x: float) -> float:
        lam = self.lams[i]
        ipow = {0: 6, 3: 7, 4: 8, 6: 10}[lam]
        ar, aa = self.alphas[i]
        return ar * math.exp(2.0 * self.beta1 * (1.0 - x)) - aa * self.c6 / x ** ipow

    def __call__(self, x: float) -> np.ndarray:
        return np.array([self.iso(x)] + [self.aniso(i, x) for i in range(len(self.lams))])
