"""CPU ORACLE -- TEST INFRASTRUCTURE ONLY.

MOLSCAT ITYPE=9 with the alkali + alkali plug-in in the fully uncoupled
basis |m_sa m_ia m_sb m_ib> |L M_L> (all projections doubled, as the
reference keeps them), in a magnetic field, restated in numpy:

* pair states ................. source_code/base9-alk_alk_ucpld.f:204-240
  (SET9: m_sa, m_ia, m_sb, m_ib loops; identical atoms keep one ordering of
  each exchanged pair)
* channel basis ............... base9-alk_alk_ucpld.f:258-353 (BASE9:
  MTOT = JTOT (doubled), L of one parity per IBLOCK, identical-particle
  exclusions, then the reference's own exchange sort on L)
* couplings ................... base9-alk_alk_ucpld.f:375-514 (CPL9: the
  singlet/triplet projections CENTPT, the spin-spin dipolar term SPINSP,
  the S.I hyperfine term SDOTI2, the electron + nuclear Zeeman term, with
  the identical-particle symmetrisation factors)
* hyperfine constants ......... base9-alk_alk_ucpld.f:142-164
* threshold of MONQN .......... base9-alk_alk_ucpld.f:516-603 (THRSH9:
  Breit-Rabi for each atom)
* Hannover-form potential ..... source_code/vstar-Hannover.f:1-325 (VSTAR
  short-range / power-series / long-range branches, the matching of PMATCH
  and GAMBET) with the parameter set of a data module such as
  source_code/Hdata-Rb2-2010.f (read by the fixture generator)
* physical constants .......... source_code/physical_constants_module.f

Half-integer 3j symbols are evaluated from Racah's formula on doubled
arguments (threej2).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction
from functools import lru_cache

import numpy as np

from . import oracle as O

# physical_constants_module.f (CODATA 2022)
G_E = -2.00231930436092
BOHR_MAGNETON_CM_PER_G = 0.46686447719 / 1.0e4
INV_FINE_STRUCTURE = 137.035999177
HARTREE_CM = 2.1947463136314e5
GHZ_CM = 2.99792458e8 * 1.0e2 / 1.0e9   # speed_of_light_in_cm / Giga
MHZ_IN_CM = 3.335640951e-11 * 1.0e6
BOHR_ANG = 0.529177210544


@lru_cache(maxsize=None)
def threej2(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """(j1/2 j2/2 j3/2; m1/2 m2/2 m3/2) from doubled arguments (Racah)."""
    if m1 + m2 + m3 != 0 or abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    if (j1 + m1) % 2 or (j2 + m2) % 2 or (j3 + m3) % 2 or (j1 + j2 + j3) % 2:
        return 0.0
    if not (abs(j1 - j2) <= j3 <= j1 + j2):
        return 0.0
    f = O._fact
    a = (j1 + j2 - j3) // 2
    b = (j1 - j2 + j3) // 2
    c = (-j1 + j2 + j3) // 2
    big = (j1 + j2 + j3) // 2 + 1
    pre2 = Fraction(f(a) * f(b) * f(c), f(big))
    pre2 *= (f((j1 + m1) // 2) * f((j1 - m1) // 2) * f((j2 + m2) // 2) * f((j2 - m2) // 2)
             * f((j3 + m3) // 2) * f((j3 - m3) // 2))
    kmin = max(0, (j2 - j3 - m1) // 2, (j1 - j3 + m2) // 2)
    kmax = min(a, (j1 - m1) // 2, (j2 + m2) // 2)
    s = Fraction(0)
    for k in range(kmin, kmax + 1):
        den = (f(k) * f(a - k) * f((j1 - m1) // 2 - k) * f((j2 + m2) // 2 - k)
               * f((j3 - j2 + m1) // 2 + k) * f((j3 - j1 - m2) // 2 + k))
        s += Fraction(-1 if k % 2 else 1, den)
    if s == 0:
        return 0.0
    val = math.sqrt(pre2 * s * s)
    if s < 0:
        val = -val
    return -val if ((j1 - j2 - m3) // 2) % 2 else val


def _sgn(k: int) -> float:
    """PARSGN (parsgn.f)."""
    return -1.0 if k % 2 else 1.0


def sdoti2(is_: int, ms1: int, ms2: int, ii: int, mi1: int, mi2: int) -> float:
    """<ms1 mi1| s.i |ms2 mi2> in the uncoupled basis, doubled arguments
    (SDOTI2)."""
    if ms1 + mi1 != ms2 + mi2:
        return 0.0
    if ms1 == ms2:
        return 0.25 * float(mi1 * ms1)
    if abs(ms1 - ms2) == 2:
        return 0.125 * math.sqrt(float(ii * (ii + 2) - mi1 * mi2)) * math.sqrt(float(is_ * (is_ + 2) - ms1 * ms2))
    return 0.0


def centpt(s2: int, isa: int, isb: int, msar: int, msbr: int, msac: int, msbc: int) -> float:
    """Projection on total spin S = s2/2 (CENTPT)."""
    fac1 = threej2(isa, isb, s2, msar, msbr, -msar - msbr)
    fac2 = threej2(isa, isb, s2, msac, msbc, -msac - msbc)
    fac3 = (s2 / 2.0 + s2 / 2.0 + 1.0) * _sgn(isa - isb + (msar + msbr + msac + msbc) // 2)
    return fac1 * fac2 * fac3


def spinsp(isa, isb, msar, msbr, lr, mlr, msac, msbc, lc, mlc) -> float:
    """sqrt(6) sum_q (-1)^q T2_q(s_a, s_b) T2_-q(C) between uncoupled states
    (SPINSP; L undoubled, the rest doubled)."""
    if msar + msbr + mlr != msac + msbc + mlc:
        return 0.0
    if abs(lc - lr) > 2 or abs(mlr - mlc) > 4:
        return 0.0
    iqa = (msar - msac) // 2
    iqb = (msbr - msbc) // 2
    iq = iqa + iqb
    if (mlc - mlr) // 2 != iq:
        return 0.0
    xsa = 0.5 * float(isa)
    xsb = 0.5 * float(isb)
    fac1 = O.threej000(lr, 2, lc)
    fac2 = (math.sqrt(xsa * (xsa + 1.0) * (xsa + xsa + 1.0) * xsb * (xsb + 1.0) * (xsb + xsb + 1.0)
                      * float((2 * lr + 1) * (2 * lc + 1)))
            * _sgn((isa + isb - msar - msbr - mlr) // 2))
    fac3 = fac1 * fac2 * threej2(2 * lr, 4, 2 * lc, -mlr, -2 * iq, mlc)
    fac4 = threej2(2, 2, 4, 2 * iqa, 2 * iqb, -2 * iq)
    fac5 = threej2(isa, 2, isa, -msar, 2 * iqa, msac)
    fac6 = threej2(isb, 2, isb, -msbr, 2 * iqb, msbc)
    return (0.0 + fac3 * fac4 * fac5 * fac6) * math.sqrt(30.0)


# --------------------------------------------------------------------------
# Hannover-form singlet / triplet curves (vstar-Hannover.f)
# --------------------------------------------------------------------------
def _power(x: float, a, n: int) -> float:
    """POWER: Horner on a[0..n-1]."""
    p = 0.0
    for i in range(n - 1, 0, -1):
        p = p + a[i]
        p = p * x
    return p + a[0]


def _dpower(x: float, a, n: int) -> float:
    p = 0.0
    for i in range(n - 1, 1, -1):
        p = p + float(i) * a[i]
        p = p * x
    return p + a[1]


@dataclass
class Hannover:
    """Parameters of a data module (cm-1 and powers of Angstrom); index 0 is
    the singlet X, 1 the triplet a.  runitm: the program's length unit in
    Angstrom (bohr for the Rb2 data)."""
    na: list
    a: list            # a[nv] = coefficients A(0..NA-1)
    rm: list
    b: list
    rsr: list
    rlr: list
    nsr: list
    asr: list
    bsr: list
    alpsr: list
    c6: float
    c8: float
    c10: float
    nex: int
    cex: float
    gambet: int
    exsign: list
    aex: float
    gamma: float
    beta: float
    runitm: float
    matchl: bool = True
    matchv: bool = True
    matchd: bool = True
    vmax: float = 1.0e4

    def __post_init__(self):
        self.a = [list(map(float, x)) for x in self.a]
        self.asr = list(map(float, self.asr))
        self.bsr = list(map(float, self.bsr))
        if self.gambet == 2:
            self.beta = 7.0 / (BOHR_ANG * (self.gamma + 1.0))
        elif self.gambet == 1:
            self.gamma = 7.0 / (self.beta * BOHR_ANG) - 1.0
        for nv in range(2):
            self._pmatch(nv)

    def _pmatch(self, nv: int):
        """PMATCH: A(0) to meet the long-range form at RLR, then ASR and BSR
        to meet the power series' value and slope at RSR."""
        rl = self.rlr[nv]
        rl2 = rl ** 2
        vexch = self.aex * rl ** self.gamma * math.exp(-self.beta * rl)
        vlr = self.exsign[nv] * vexch - (self.c6 + (self.c8 + self.c10 / rl2) / rl2) / rl2 ** 3
        if self.nex > 0:
            vlr = vlr - self.cex / rl ** self.nex
        xi = (rl - self.rm[nv]) / (rl + self.b[nv] * self.rm[nv])
        vmid = _power(xi, self.a[nv], self.na[nv])
        anew = self.a[nv][0] + vlr - vmid
        if self.matchl:
            self.a[nv][0] = anew
        rs = self.rsr[nv]
        xi = (rs - self.rm[nv]) / (rs + self.b[nv] * self.rm[nv])
        vmid = _power(xi, self.a[nv], self.na[nv])
        dxidr = (self.b[nv] + 1.0) * self.rm[nv] / (rs + self.b[nv] * self.rm[nv]) ** 2
        dvdr = dxidr * _dpower(xi, self.a[nv], self.na[nv])
        bsrnew = (-dvdr * rs ** self.nsr[nv] * math.exp(self.alpsr[nv] * rs)
                  / (self.nsr[nv] / rs + self.alpsr[nv]))
        if self.matchd:
            self.bsr[nv] = bsrnew
        asadd = -self.bsr[nv] / rs ** self.nsr[nv] * math.exp(-self.alpsr[nv] * rs)
        if self.matchv:
            self.asr[nv] = vmid + asadd

    def vstar(self, nv: int, r: float) -> float:
        """Curve nv (0 singlet, 1 triplet) at R in program units, cm-1."""
        ra = r * self.runitm
        if ra < self.rsr[nv]:
            v = self.asr[nv] + self.bsr[nv] / ra ** self.nsr[nv] * math.exp(-self.alpsr[nv] * ra)
        elif ra <= self.rlr[nv]:
            xi = (ra - self.rm[nv]) / (ra + self.b[nv] * self.rm[nv])
            v = _power(xi, self.a[nv], self.na[nv])
        else:
            vexch = self.aex * ra ** self.gamma * math.exp(-self.beta * ra)
            v = self.exsign[nv] * vexch - self.c6 / ra ** 6 - self.c8 / ra ** 8 - self.c10 / ra ** 10
            if self.nex > 0:
                v = v - self.cex / ra ** self.nex
        return min(v, self.vmax)


# --------------------------------------------------------------------------
# the basis plug-in (base9-alk_alk_ucpld.f)
# --------------------------------------------------------------------------
@dataclass
class AlkAlk:
    """Two alkali atoms (doubled spins ISA/ISB and nuclear spins INUCA/INUCB;
    INUCB < 0: identical atoms), &BASIS9 constants, LMAX, the radial terms
    and the field.  curves(r) -> (singlet, triplet) in cm-1; ss_terms: the
    spin-spin radial term's (A, NPOWER, E) list (POTENL case 1)."""
    ured: float
    isa: int
    inuca: int
    gsa: float
    ga: float
    hfspla: float
    lmax: int
    curves: object
    ss_terms: list = field(default_factory=list)
    isb: int = 1
    inucb: int = -1
    gsb: float = -1.0
    gb: float = 0.0
    hfsplb: float = 0.0
    ispsp: int = 0
    field_g: float = 0.0
    rm: float = BOHR_ANG     # the program's length unit (Angstrom)
    epsil: float = 1.0

    def __post_init__(self):
        gs = -G_E
        if self.gsa < 0.0:
            self.gsa = gs
        if self.gsb < 0.0:
            self.gsb = gs
        self.ident = self.inucb < 0
        if self.ident:
            self.isb, self.gsb, self.inucb, self.gb, self.hfsplb = self.isa, self.gsa, self.inuca, self.ga, self.hfspla
        self.ansa = self._ans(self.isa, self.inuca, self.hfspla)
        self.ansb = self._ans(self.isb, self.inucb, self.hfsplb)
        self.nspin = 1 + min(self.isa, self.isb)
        self.ibosfr = (self.inuca + self.isa) % 2  # 0: bosons, 1: fermions (identical atoms)

    @staticmethod
    def _ans(is_, inuc, hfspl):
        ifmax = inuc + is_
        ifmin = abs(inuc - is_)
        nsfac = (ifmax * (ifmax + 2) - ifmin * (ifmin + 2)) // 4
        return 2.0 * hfspl / float(nsfac) if nsfac != 0 else 0.0

    @property
    def cm2ru(self) -> float:
        return self.ured * 1.0 * self.rm * self.rm / O.BFCT

    @property
    def ep2ru(self) -> float:
        return self.epsil * self.cm2ru

    @property
    def mxlam(self) -> int:
        return self.nspin + 1

    @property
    def vconst(self) -> list:
        return [1.0 / GHZ_CM, self.field_g]

    def pair_states(self) -> list:
        out = []
        for msa in range(-self.isa, self.isa + 1, 2):
            for mia in range(-self.inuca, self.inuca + 1, 2):
                msbmax = msa if self.ident else self.isb
                for msb in range(-self.isb, msbmax + 1, 2):
                    mibmax = mia if (self.ident and msa == msb) else self.inucb
                    for mib in range(-self.inucb, mibmax + 1, 2):
                        out.append((msa, mia, msb, mib))
        return out

    def channels(self, jtot: int, iblock: int) -> list:
        """[(pair-state index, L)] in the reference's order (BASE9)."""
        if (jtot % 2 == 0) != ((self.isa + self.inuca + self.isb + self.inucb) % 2 == 0):
            raise ValueError("JTOT must have the parity of ISA + INUCA + ISB + INUCB")
        mtot = jtot
        js, ls = [], []
        for i, (msa, mia, msb, mib) in enumerate(self.pair_states()):
            mf = msa + msb + mia + mib
            ml = mtot - mf
            lstart = 4 - 2 * iblock
            if self.ident and msa == msb and mia == mib and self.ibosfr + iblock != 2:
                lstart = 2 * self.lmax + 1
            for ll in range(lstart, 2 * self.lmax + 1, 4):
                if abs(ml) > ll:
                    continue
                js.append(i)
                ls.append(ll // 2)
        n = len(ls)
        for i in range(n):           # the reference's exchange sort on L
            for jj in range(i + 1, n):
                if ls[jj] < ls[i]:
                    ls[i], ls[jj] = ls[jj], ls[i]
                    js[i], js[jj] = js[jj], js[i]
        return list(zip(js, ls))

    def coupling(self, jtot: int, iblock: int) -> O.Coupling:
        """VL(NVLBLK, N(N+1)/2): NSPIN central terms, the spin-spin term,
        hyperfine and Zeeman (CPL9); EINT zero (NCONST > 0), CENT L(L+1)."""
        ps = self.pair_states()
        ch = self.channels(jtot, iblock)
        n = len(ch)
        mtot = jtot
        mxlam = self.mxlam
        nvlblk = mxlam + 2
        spmin = 0.5 * abs(float(self.isa - self.isb))
        vl = np.zeros(nvlblk * n * (n + 1) // 2)
        idx = 0
        for icol in range(n):
            msac, miac, msbc, mibc = ps[ch[icol][0]]
            lc = ch[icol][1]
            mlc = mtot - msac - msbc - miac - mibc
            for irow in range(icol + 1):
                msar, miar, msbr, mibr = ps[ch[irow][0]]
                lr = ch[irow][1]
                mlr = mtot - msar - msbr - miar - mibr
                prefac = 1.0
                if self.ident and msar == msbr and miar == mibr:
                    prefac = prefac / math.sqrt(2.0)
                if self.ident and msac == msbc and miac == mibc:
                    prefac = prefac / math.sqrt(2.0)
                for ll in range(1, nvlblk + 1):
                    v = 0.0
                    if ll <= self.nspin and lr == lc and mlr == mlc:
                        xs = spmin + float(ll - 1)
                        fac = prefac * centpt(int(round(2 * xs)), self.isa, self.isb, msar, msbr, msac, msbc)
                        if miar == miac and mibr == mibc:
                            v = fac
                        if self.ident and miar == mibc and mibr == miac:
                            if (self.isa + int(round(xs)) + self.ibosfr + lr) % 2:
                                fac = -fac
                            v = v + fac
                    elif ll == self.nspin + 1 and self.ispsp >= 0:
                        fac = prefac * spinsp(self.isa, self.isb, msar, msbr, lr, mlr, msac, msbc, lc, mlc)
                        if miar == miac and mibr == mibc:
                            v = v + fac
                        if self.ident and miar == mibc and mibr == miac:
                            fac2 = prefac * spinsp(self.isa, self.isb, msbr, msar, lr, mlr, msac, msbc, lc, mlc)
                            if (self.ibosfr + lr) % 2:
                                fac2 = -fac2
                            v = v + fac2
                        v = v * HARTREE_CM / INV_FINE_STRUCTURE ** 2
                    elif ll == mxlam + 1 and lr == lc and mlr == mlc:
                        faca = self.ansa * sdoti2(self.isa, msar, msac, self.inuca, miar, miac)
                        facb = self.ansb * sdoti2(self.isb, msbr, msbc, self.inucb, mibr, mibc)
                        if msbr == msbc and mibr == mibc:
                            v = prefac * faca
                        if msar == msac and miar == miac:
                            v = v + prefac * facb
                        if self.ident:
                            if msar == msbc and miar == mibc:
                                fac2 = prefac * self.ansa * sdoti2(self.isa, msbr, msac, self.inuca, mibr, miac)
                                if (self.ibosfr + lr) % 2:
                                    fac2 = -fac2
                                v = v + fac2
                            if msbr == msac and mibr == miac:
                                fac2 = prefac * self.ansa * sdoti2(self.isa, msar, msbc, self.inuca, miar, mibc)
                                if (self.ibosfr + lr) % 2:
                                    fac2 = -fac2
                                v = v + fac2
                    elif ll == mxlam + 2 and icol == irow:
                        v = (self.gsa * float(msar) + self.gsb * float(msbr) + self.ga * float(miar)
                             + self.gb * float(mibr))
                        v = v * BOHR_MAGNETON_CM_PER_G * 0.5
                    vl[idx + ll - 1] = v
                idx += nvlblk
        cent = np.array([float(ell * (ell + 1)) for _, ell in ch])
        return O.Coupling(n=n, nham=nvlblk, vl=vl, eint=np.zeros(n), cent=cent, nconst=2)

    def _breit_rabi(self, f2: int, m: int, inuc: int, hfspl: float, gs: float, gn: float, is_: int, b: float):
        bohrm = BOHR_MAGNETON_CM_PER_G * GHZ_CM
        if abs(f2 - inuc) != 1 or abs(m) > f2 or (m + f2) % 2:
            raise ValueError("invalid MONQN pair")
        e1 = -hfspl / (2.0 * float(inuc + 1)) + 0.5 * gn * bohrm * float(m) * b
        bx = bohrm * b * (gs - gn) / hfspl
        e2 = 0.5 * hfspl * math.sqrt(1.0 + float(m + m) * bx / float(inuc + 1) + bx * bx)
        if abs(m) == inuc + 1:
            return (float(inuc) * hfspl / (2.0 * float(inuc + 1))
                    + math.copysign(1.0, float(m)) * bohrm * b * (gs * is_ * 0.5 + gn * inuc * 0.5))
        if f2 == inuc + 1:
            return e1 + e2
        return e1 - e2

    def threshold(self, monqn) -> float:
        """EREF (cm-1) of MONQN = (2F_A, 2M_A, 2F_B, 2M_B) at the field (THRSH9)."""
        b = self.field_g
        ea = self._breit_rabi(monqn[0], monqn[1], self.inuca, self.hfspla, self.gsa, self.ga, self.isa, b)
        eb = self._breit_rabi(monqn[2], monqn[3], self.inucb, self.hfsplb, self.gsb, self.gb, self.isb, b)
        return (ea + eb) / GHZ_CM

    def pvec(self, r: float) -> np.ndarray:
        """P for SUMLAM (hammat.f:37-83): singlet, triplet, the spin-spin
        radial term (POTENL case 1, units of EPSIL), then VCONST."""
        vs, vt = self.curves(r)
        p = [vs, vt]
        tot = 0.0
        for a, npw, e in self.ss_terms:
            if npw != 0:
                rr = r
                if npw < 0 and abs(r) < 1.0e-8:
                    rr = 1.0e-8
                term = rr ** npw
            else:
                term = math.exp(e * r)
            tot = tot + a * term
        p.append(tot)
        p = np.array(p)
        p = np.where(np.abs(p) > 1.0e60, np.sign(p) * 1.0e60, p)
        ep2cm = self.ep2ru / self.cm2ru
        pc = np.array([v / ep2cm for v in self.vconst])
        return self.ep2ru * np.concatenate([p, pc])
