"""Two alkali atoms in a magnetic field (the alkali + alkali plug-in of
source_code/base9-alk_alk_ucpld.f): host-side basis and couplings for the
propagator, the Breit-Rabi thresholds, and the seeded synthetic field sweep
of the BOUND/FIELD workload.

Basis: the fully uncoupled pair states |m_sa m_ia m_sb m_ib> (projections
doubled, as the reference keeps them) with partial waves |L M_L>, M_L fixed by
MTOT = JTOT (doubled), one L parity per symmetry block, sorted on L with the
reference's exchange sort (base9-alk_alk_ucpld.f:258-353).  Identical atoms
keep one ordering of each exchanged pair and carry the reference's
symmetrisation factors.

Coupling terms, in the reference's order (CPL9, base9-alk_alk_ucpld.f:375-514):
the central singlet and triplet projections (total spin S of the electron
pair), the spin-spin dipolar term (a rank-2 spin tensor coupling L to L' =
L, L +- 2), the s.i hyperfine term of each atom, and the electron + nuclear
Zeeman term, which is diagonal in this basis.

A field sweep exploits that diagonality: the Zeeman term becomes a
per-field threshold vector (EINT with NCONST = 0 semantics), so every field
of a block uses one VL array and one P table, and the library shares their
device copies and the energy- and field-independent MDPROP U(C) tables
across all fields (mgpu_plan_shared_systems).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from fractions import Fraction
from functools import lru_cache

import numpy as np

from .propagators import Coupling, Segment

# CODATA 2022 values (source_code/physical_constants_module.f)
_G_E = 2.00231930436092            # |g_e|
_MU_B_CM_PER_G = 0.46686447719e-4   # Bohr magneton, cm-1 per gauss
_ALPHA_INV = 137.035999177
_HARTREE_CM = 2.1947463136314e5
_GHZ_CM = 29.9792458                # cm-1 -> GHz
_MHZ_CM = 3.335640951e-5            # cm-1 per MHz
_BOHR_A = 0.529177210544
_H = 6.62607015e-34
_C = 2.99792458e8
_U = 1.66053906892e-27
_PI = 3.141592653589793
_BFCT = (_H / 2.0 / _PI) / (4.0 * _PI * (_C * 1.0e2)) / (1.0e-10) ** 2 / _U


@lru_cache(maxsize=None)
def _fac(n: int) -> int:
    return math.factorial(n)


@lru_cache(maxsize=None)
def w3j(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """Wigner 3j symbol with every argument doubled (2j, 2m), exact rational
    arithmetic under one square root."""
    if m1 + m2 + m3 or abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    if (j1 + m1) & 1 or (j2 + m2) & 1 or (j3 + m3) & 1 or (j1 + j2 + j3) & 1:
        return 0.0
    if j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    t1, t2, t3 = (j1 + j2 - j3) // 2, (j1 - j2 + j3) // 2, (j2 + j3 - j1) // 2
    a1, a2 = (j1 + m1) // 2, (j1 - m1) // 2
    b1, b2 = (j2 + m2) // 2, (j2 - m2) // 2
    c1, c2 = (j3 + m3) // 2, (j3 - m3) // 2
    norm = Fraction(_fac(t1) * _fac(t2) * _fac(t3) * _fac(a1) * _fac(a2) * _fac(b1) * _fac(b2) * _fac(c1) * _fac(c2),
                    _fac((j1 + j2 + j3) // 2 + 1))
    x1, x2 = (j3 - j2 + m1) // 2, (j3 - j1 - m2) // 2
    tot = Fraction(0)
    for k in range(max(0, -x1, -x2), min(t1, a2, b1) + 1):
        d = _fac(k) * _fac(t1 - k) * _fac(a2 - k) * _fac(b1 - k) * _fac(x1 + k) * _fac(x2 + k)
        tot += Fraction(-1 if k & 1 else 1, d)
    if tot == 0:
        return 0.0
    v = math.copysign(math.sqrt(norm * tot * tot), float(tot))
    return -v if ((j1 - j2 - m3) // 2) & 1 else v


def _par(k: int) -> float:
    return -1.0 if k & 1 else 1.0


def _sdoti(s2: int, ms1: int, ms2: int, i2: int, mi1: int, mi2: int) -> float:
    """<ms1 mi1| s.i |ms2 mi2> (doubled projections)."""
    if ms1 + mi1 != ms2 + mi2:
        return 0.0
    if ms1 == ms2:
        return 0.25 * float(mi1 * ms1)
    if abs(ms1 - ms2) == 2:
        return 0.125 * math.sqrt(float(i2 * (i2 + 2) - mi1 * mi2)) * math.sqrt(float(s2 * (s2 + 2) - ms1 * ms2))
    return 0.0


def _spin_projection(s2: int, sa: int, sb: int, mar: int, mbr: int, mac: int, mbc: int) -> float:
    """<mar mbr| P_S |mac mbc>, the projector on total electron spin S = s2/2."""
    f1 = w3j(sa, sb, s2, mar, mbr, -mar - mbr)
    f2 = w3j(sa, sb, s2, mac, mbc, -mac - mbc)
    return f1 * f2 * (s2 + 1.0) * _par(sa - sb + (mar + mbr + mac + mbc) // 2)


def _spin_spin(sa, sb, mar, mbr, lr, mlr, mac, mbc, lc, mlc) -> float:
    """sqrt(6) sum_q (-1)^q T2_q(s_a, s_b) T2_-q(C) (L undoubled)."""
    if mar + mbr + mlr != mac + mbc + mlc or abs(lc - lr) > 2 or abs(mlr - mlc) > 4:
        return 0.0
    qa, qb = (mar - mac) // 2, (mbr - mbc) // 2
    q = qa + qb
    if (mlc - mlr) // 2 != q:
        return 0.0
    xa, xb = 0.5 * sa, 0.5 * sb
    red = math.sqrt(xa * (xa + 1.0) * (2.0 * xa + 1.0) * xb * (xb + 1.0) * (2.0 * xb + 1.0)
                    * float((2 * lr + 1) * (2 * lc + 1))) * _par((sa + sb - mar - mbr - mlr) // 2)
    v = (w3j(2 * lr, 4, 2 * lc, 0, 0, 0) * red * w3j(2 * lr, 4, 2 * lc, -mlr, -2 * q, mlc)
         * w3j(2, 2, 4, 2 * qa, 2 * qb, -2 * q) * w3j(sa, 2, sa, -mar, 2 * qa, mac) * w3j(sb, 2, sb, -mbr, 2 * qb, mbc))
    return v * math.sqrt(30.0)


@dataclass
class AlkaliPair:
    """Atom constants (doubled spins), LMAX and the length unit (Angstrom per
    program unit).  inucb < 0: identical atoms."""
    ured: float
    sa: int = 1
    ia: int = 3
    gsa: float = _G_E
    ga: float = 0.0
    hfsa: float = 1.0      # GHz
    lmax: int = 4
    sb: int = 1
    ib: int = -1
    gsb: float = _G_E
    gb: float = 0.0
    hfsb: float = 0.0
    rm: float = 1.0

    def __post_init__(self):
        self.ident = self.ib < 0
        if self.ident:
            self.sb, self.ib, self.gsb, self.gb, self.hfsb = self.sa, self.ia, self.gsa, self.ga, self.hfsa
        self.bosons = (self.ia + self.sa) % 2 == 0
        self.nspin = 1 + min(self.sa, self.sb)

    @staticmethod
    def _acoef(s2, i2, hfs):
        fmax, fmin = i2 + s2, abs(i2 - s2)
        nf = (fmax * (fmax + 2) - fmin * (fmin + 2)) // 4
        return 2.0 * hfs / nf if nf else 0.0

    @property
    def cm2ru(self) -> float:
        return self.ured * self.rm * self.rm / _BFCT

    def pair_states(self) -> list:
        out = []
        for msa in range(-self.sa, self.sa + 1, 2):
            for mia in range(-self.ia, self.ia + 1, 2):
                for msb in range(-self.sb, (msa if self.ident else self.sb) + 1, 2):
                    top = mia if (self.ident and msa == msb) else self.ib
                    for mib in range(-self.ib, top + 1, 2):
                        out.append((msa, mia, msb, mib))
        return out

    def channels(self, mtot: int, block: int) -> list:
        """[(pair-state index, L)] for doubled MTOT and symmetry block 1 (odd
        L) or 2 (even L), in the reference's order."""
        if (mtot - self.sa - self.ia - self.sb - self.ib) % 2:
            raise ValueError("MTOT must have the parity of 2(s_a + i_a + s_b + i_b)")
        st, ls = [], []
        for k, (msa, mia, msb, mib) in enumerate(self.pair_states()):
            ml = mtot - (msa + mia + msb + mib)
            l0 = 4 - 2 * block
            if self.ident and msa == msb and mia == mib and (0 if self.bosons else 1) + block != 2:
                continue
            for ll in range(l0, 2 * self.lmax + 1, 4):
                if abs(ml) <= ll:
                    st.append(k)
                    ls.append(ll // 2)
        for i in range(len(ls)):
            for j in range(i + 1, len(ls)):
                if ls[j] < ls[i]:
                    ls[i], ls[j] = ls[j], ls[i]
                    st[i], st[j] = st[j], st[i]
        return list(zip(st, ls))

    def operators(self, mtot: int, block: int):
        """Per channel pair (SUMLAM order, column by column, row <= column):
        the singlet, triplet (NSPIN central terms), spin-spin and hyperfine
        coefficients, and the diagonal Zeeman coefficients (cm-1 per gauss).
        Returns (terms [npair, NSPIN + 2], zeeman [N], L)."""
        ps = self.pair_states()
        ch = self.channels(mtot, block)
        n = len(ch)
        aa = self._acoef(self.sa, self.ia, self.hfsa)
        ab = self._acoef(self.sb, self.ib, self.hfsb)
        smin = abs(self.sa - self.sb)  # doubled
        fsym = 0 if self.bosons else 1
        npair = n * (n + 1) // 2
        terms = np.zeros((npair, self.nspin + 2))
        p = 0
        for c in range(n):
            mac, iac, mbc, ibc = ps[ch[c][0]]
            lc = ch[c][1]
            mlc = mtot - mac - mbc - iac - ibc
            for r in range(c + 1):
                mar, iar, mbr, ibr = ps[ch[r][0]]
                lr = ch[r][1]
                mlr = mtot - mar - mbr - iar - ibr
                pre = 1.0
                if self.ident and mar == mbr and iar == ibr:
                    pre /= math.sqrt(2.0)
                if self.ident and mac == mbc and iac == ibc:
                    pre /= math.sqrt(2.0)
                same_l = lr == lc and mlr == mlc
                for t in range(self.nspin):
                    if not same_l:
                        break
                    s2 = smin + 2 * t
                    f = pre * _spin_projection(s2, self.sa, self.sb, mar, mbr, mac, mbc)
                    v = f if (iar == iac and ibr == ibc) else 0.0
                    if self.ident and iar == ibc and ibr == iac:
                        v += -f if (self.sa + s2 // 2 + fsym + lr) & 1 else f
                    terms[p, t] = v
                f = pre * _spin_spin(self.sa, self.sb, mar, mbr, lr, mlr, mac, mbc, lc, mlc)
                v = f if (iar == iac and ibr == ibc) else 0.0
                if self.ident and iar == ibc and ibr == iac:
                    f2 = pre * _spin_spin(self.sa, self.sb, mbr, mar, lr, mlr, mac, mbc, lc, mlc)
                    v += -f2 if (fsym + lr) & 1 else f2
                terms[p, self.nspin] = v * _HARTREE_CM / _ALPHA_INV ** 2
                if same_l:
                    v = 0.0
                    if mbr == mbc and ibr == ibc:
                        v = pre * aa * _sdoti(self.sa, mar, mac, self.ia, iar, iac)
                    if mar == mac and iar == iac:
                        v += pre * ab * _sdoti(self.sb, mbr, mbc, self.ib, ibr, ibc)
                    if self.ident:
                        sg = -1.0 if (fsym + lr) & 1 else 1.0
                        if mar == mbc and iar == ibc:
                            v += sg * pre * aa * _sdoti(self.sa, mbr, mac, self.ia, ibr, iac)
                        if mbr == mac and ibr == iac:
                            v += sg * pre * aa * _sdoti(self.sa, mar, mbc, self.ia, iar, ibc)
                    terms[p, self.nspin + 1] = v
                p += 1
        zee = np.array([(self.gsa * ps[k][0] + self.gsb * ps[k][2] + self.ga * ps[k][1] + self.gb * ps[k][3])
                        * _MU_B_CM_PER_G * 0.5 for k, _ in ch])
        lval = np.array([ell for _, ell in ch])
        return terms, zee, lval

    def breit_rabi(self, f2: int, m2: int, atom: str, field_g: float) -> float:
        """Energy (GHz) of the hyperfine-Zeeman state |2f, 2m> of atom 'a'
        or 'b' (the Breit-Rabi formula)."""
        s2, i2, gs, gn, hfs = ((self.sa, self.ia, self.gsa, self.ga, self.hfsa) if atom == "a" else
                               (self.sb, self.ib, self.gsb, self.gb, self.hfsb))
        if abs(f2 - i2) != 1 or abs(m2) > f2 or (m2 + f2) % 2:
            raise ValueError("invalid (2f, 2m)")
        mub = _MU_B_CM_PER_G * _GHZ_CM
        if abs(m2) == i2 + 1:
            return (i2 * hfs / (2.0 * (i2 + 1)) + math.copysign(1.0, m2) * mub * field_g
                    * (gs * s2 * 0.5 + gn * i2 * 0.5))
        e1 = -hfs / (2.0 * (i2 + 1)) + 0.5 * gn * mub * m2 * field_g
        x = mub * field_g * (gs - gn) / hfs
        e2 = 0.5 * hfs * math.sqrt(1.0 + 2.0 * m2 * x / (i2 + 1) + x * x)
        return e1 + e2 if f2 == i2 + 1 else e1 - e2

    def threshold_cm(self, monqn, field_g: float) -> float:
        """EREF (cm-1) of the pair state (2f_a, 2m_a, 2f_b, 2m_b)."""
        return (self.breit_rabi(monqn[0], monqn[1], "a", field_g)
                + self.breit_rabi(monqn[2], monqn[3], "b", field_g)) / _GHZ_CM


# --------------------------------------------------------------------------
# the synthetic BOUND/FIELD workload: a heteronuclear pair with i = 3/2
# --------------------------------------------------------------------------
C6_AU = 4700.0
C6_CM_A6 = C6_AU * _HARTREE_CM * _BOHR_A ** 6


def morse_c6(de: float, re: float, a: float, rd: float):
    """De[(1 - e^{-a(R-Re)})^2 - 1] - (1 - e^{-(R/Rd)^12}) C6/R^6 (cm-1, A)."""
    def v(r):
        x = math.exp(-a * (r - re))
        return de * ((1.0 - x) ** 2 - 1.0) - (1.0 - math.exp(-(r / rd) ** 12)) * C6_CM_A6 / r ** 6
    return v


@dataclass
class FieldSweep:
    """One (MTOT, block) of a pair at a fixed energy relative to the
    field-dependent threshold of `monqn`, over many fields, with MDPROP
    outward RMIN -> RMATCH and inward RMAX -> RMATCH on the GPU."""
    pair: AlkaliPair
    mtot: int
    block: int
    monqn: tuple
    energy_mhz: float
    singlet: object
    triplet: object
    rmin: float
    rmatch: float
    rmax: float
    nout: int
    nin: int

    def __post_init__(self):
        terms, zee, lval = self.pair.operators(self.mtot, self.block)
        self.n = lval.size
        self.nham = terms.shape[1]
        cm2ru = self.pair.cm2ru
        self.vl = np.ascontiguousarray(terms.ravel())
        self.cent = (lval * (lval + 1)).astype(np.float64)
        self.zee_ru = zee * cm2ru
        self.seg_out = Segment.build(self.rmin, (self.rmatch - self.rmin) / self.nout, self.nout, self.pvec, self.nham)
        self.seg_in = Segment.build(self.rmax, -(self.rmax - self.rmatch) / self.nin, self.nin, self.pvec, self.nham)

    def pvec(self, r: float) -> np.ndarray:
        """P at R (program units = Angstrom): singlet, triplet, the spin-spin
        radial factor -(a0/R)^3 (atomic units, so the coefficient carries
        E_h alpha^2), the hyperfine prefactor 1/GHZCM; all times CM2RU."""
        cm2ru = self.pair.cm2ru
        ps = [self.singlet(r), self.triplet(r)][: self.pair.nspin]
        return cm2ru * np.array(ps + [-(_BOHR_A / r) ** 3, 1.0 / _GHZ_CM])

    def coupling_at(self, field_g: float) -> Coupling:
        """The block at field F: the shared VL, the Zeeman diagonal as EINT."""
        return Coupling(n=self.n, nham=self.nham, vl=self.vl, eint=self.zee_ru * field_g, cent=self.cent)

    def ered_at(self, field_g: float) -> float:
        return (self.pair.threshold_cm(self.monqn, field_g) + self.energy_mhz * _MHZ_CM) * self.pair.cm2ru


def config4_sweep(mtot: int = 4, block: int = 2, nout: int = 1800, nin: int = 2400) -> FieldSweep:
    """The seeded synthetic alkali pair of the BOUND/FIELD workload: doubled
    spins s = 1/2 and i = 3/2 on both atoms (heteronuclear), hyperfine
    splittings 1.0 and 0.8 GHz, nuclear g factors -0.000995 and -0.000705,
    reduced mass 26.93 u, L <= 4; Morse singlet (De 3900 cm-1, Re 4.2 A, a 0.51
    1/A) and triplet (240 cm-1, 6.0 A, 0.47 1/A), each with a damped -C6/R^6
    tail, C6 = 4700 E_h a0^6; E = 0 relative to the lowest threshold (2f = 2,
    2m_f = 2 on both atoms); MDPROP 3 -> 12 A outward and 60 -> 12 A inward.
    MTOT = 4 (doubled), even L: N = 106."""
    pair = AlkaliPair(ured=26.93, sa=1, ia=3, ga=-0.000995, hfsa=1.0, lmax=4, sb=1, ib=3, gb=-0.000705, hfsb=0.8)
    return FieldSweep(pair, mtot, block, (2, 2, 2, 2), 0.0,
                      morse_c6(3900.0, 4.2, 0.51, 1.5 * 4.2), morse_c6(240.0, 6.0, 0.47, 1.5 * 6.0),
                      rmin=3.0, rmatch=12.0, rmax=60.0, nout=nout, nin=nin)
