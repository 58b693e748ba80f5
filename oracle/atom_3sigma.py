"""CPU ORACLE -- TEST INFRASTRUCTURE ONLY.

MOLSCAT ITYPE=9 with the atom(1S) + diatom(3Sigma) basis plug-in in a
magnetic field, and the Mg-NH potential, restated in numpy for the
bound-Mg_NH example (N = 100 channels, an asymptotically non-diagonal basis
whose internal Hamiltonian enters through four constant terms):

* levels |(n s) j m_j> ........ source_code/base9-1S_3Sigma_cpld.f:153-170
  (SET9 with LEVIN false: n = JMIN..JMAX, j = |n-s|..n+s, m_j = -j..j)
* channel basis ............... base9-1S_3Sigma_cpld.f:221-242 (BASE9:
  JTOT is |M|, L = |M - m_j|..LMAX, parity (-1)^(IBLOCK+n+L+1) kept even)
* couplings ................... base9-1S_3Sigma_cpld.f:254-338 (CPL9:
  Legendre terms from 3j/6j algebra, then the constant terms: rotation,
  spin-rotation, spin-spin, electron-spin Zeeman)
* constant-term prefactors .... base9-1S_3Sigma_cpld.f:114-126 (VCONST)
* threshold of MONQN .......... base9-1S_3Sigma_cpld.f:341-441 (THRSH9)
* Mg-NH potential ............. source_code/vstar-Mg_NH.f:1-242 (RKHS
  interpolation of each angular cut with n = 3, m = 5 (RK_INIT, VRKHS,
  GETRAD), projected on Legendre polynomials by Gauss-Lobatto quadrature over
  the cuts (CALCPL and the weights of VINIT), VSTAR's (2 lambda + 1)/2)
* physical constants .......... source_code/physical_constants_module.f
  (CODATA 2022: g_e, the Bohr magneton in cm-1/T, cm-1 per MHz)

The angular-cut data (angle, R, E) are the input of the potential; the
fixture generator reads them from the reference's data/pot-Mg_NH.data.

Argument order: the reference's SIXJ(J1,J2,J5,J4,J3,J6) is the 6j symbol
{J1 J2 J3; J4 J5 J6} (sixj.f:1-8), so every SIXJ call below is written as
the 6j symbol it evaluates.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import oracle as O
from .itype6 import threej

# physical_constants_module.f (CODATA 2022)
G_E = -2.00231930436092
BOHR_MAGNETON_CM_PER_G = 0.46686447719 / 1.0e4
MHZ_IN_CM = 3.335640951e-11 * 1.0e6


def _sgn(k: int) -> float:
    """PARSGN (parsgn.f)."""
    return -1.0 if k % 2 else 1.0


def _6j(a, b, c, d, e, f) -> float:
    return O.sixj(a, b, c, d, e, f)


def _3j0(a, b, c) -> float:
    return O.threej000(a, b, c)


# --------------------------------------------------------------------------
# the Mg-NH potential (vstar-Mg_NH.f)
# --------------------------------------------------------------------------
_BETA = (3.0 / 56.0, -4.0 * (3.0 / 56.0) / 3.0, 7.0 * (3.0 / 56.0) / 15.0)  # n = 3 (VINIT)
_RK_M = 5  # m = 5: the kernel decays as r_>^-(m+1)


def _legendre_all(nang: int, x: float) -> np.ndarray:
    """P_0..P_{nang-1}(x) by the three-term recurrence (CALCPL)."""
    p = np.empty(nang)
    p[0] = 1.0
    p[1] = x
    for i in range(1, nang - 1):
        p[i + 1] = (p[i] * p[1] * float(2 * i + 1) - p[i - 1] * float(i)) / float(i + 1)
    return p


def _rk_kernel(rs: np.ndarray, rl: np.ndarray) -> np.ndarray:
    q = _BETA[0] + _BETA[1] * (rs / rl) + _BETA[2] * (rs / rl) ** 2
    return q * (1.0 / rl) ** (_RK_M + 1)


@dataclass
class MgNHPotential:
    """Radial Legendre coefficients V_lambda(R) (cm-1, R in Angstrom) from
    the angular cuts: cuts[i] = (angle in degrees, R points, energies)."""
    cuts: list

    def __post_init__(self):
        nang = len(self.cuts)
        self.nang = nang
        cth = np.array([math.cos(float(a) * math.acos(-1.0) / 180.0) for a, _, _ in self.cuts])
        self.pol = np.stack([_legendre_all(nang, c) for c in cth], axis=1)  # pol[lambda, cut]
        # Gauss-Lobatto weights 2 / (n (n-1) P_{n-1}(x)^2) (VINIT)
        self.wt = 2.0 / (float(nang * (nang - 1)) * self.pol[nang - 1] * self.pol[nang - 1])
        self.rpt, self.alpha = [], []
        for _, r, v in self.cuts:
            r = np.asarray(r, dtype=np.float64)
            v = np.asarray(v, dtype=np.float64)
            rs = np.minimum(r[:, None], r[None, :])
            rl = np.maximum(r[:, None], r[None, :])
            self.rpt.append(r)
            self.alpha.append(np.linalg.solve(_rk_kernel(rs, rl), v))  # RK_INIT (DGESV)

    def cuts_at(self, r: float) -> np.ndarray:
        """The RKHS interpolant of every cut at R (GETRAD / VRKHS)."""
        out = np.empty(self.nang)
        for i in range(self.nang):
            rp = self.rpt[i]
            out[i] = float(np.dot(_rk_kernel(np.minimum(r, rp), np.maximum(r, rp)), self.alpha[i]))
        return out

    def vlam(self, r: float, nterm: int) -> np.ndarray:
        """V_lambda(R) for lambda = 0..nterm-1 (VSTAR for terms 1..nterm)."""
        rr = self.cuts_at(r)
        out = np.empty(nterm)
        for t in range(nterm):
            out[t] = float(np.sum(self.pol[t] * rr * self.wt)) * (2.0 * t + 1.0) / 2.0
        return out


# --------------------------------------------------------------------------
# the basis plug-in (base9-1S_3Sigma_cpld.f)
# --------------------------------------------------------------------------
@dataclass
class Atom3Sigma:
    """Atom + 3Sigma diatom in a magnetic field: &BASIS ROTI = (B, gamma,
    lambda_SS), JMIN/JMAX (n range), &BASIS9 IS, LMAX, the potential's
    LAMBDA list, the reduced mass (u) and the field (G)."""
    ured: float
    roti: tuple
    nmin: int
    nmax: int
    lmax: int
    lam: list
    pot: MgNHPotential
    field: float = 0.0
    spin: int = 1
    rm: float = 1.0
    epsil: float = 1.0

    @property
    def cm2ru(self) -> float:
        return self.ured * 1.0 * self.rm * self.rm / O.BFCT

    @property
    def ep2ru(self) -> float:
        return self.epsil * self.cm2ru

    @property
    def factor(self) -> float:
        s = self.spin
        return math.sqrt(float(s * (s + 1) * (2 * s + 1)))

    @property
    def vconst(self) -> list:
        """VCONST(1..4): rotation, spin-rotation, spin-spin prefactors and
        the field (MAPEFV = 4)."""
        return [self.roti[0], self.roti[1] * self.factor, self.roti[2] * 2.0 * math.sqrt(30.0) / 3.0, self.field]

    @property
    def fz(self) -> float:
        return (-G_E) * BOHR_MAGNETON_CM_PER_G * self.factor

    def levels(self) -> list:
        s = self.spin
        out = []
        for n in range(self.nmin, self.nmax + 1):
            for j in range(abs(n - s), n + s + 1):
                for mj in range(-j, j + 1):
                    out.append((n, j, mj))
        return out

    def channels(self, mtot: int, iblock: int) -> list:
        """[(level index, L)] in the reference's order (BASE9)."""
        out = []
        for i, (n, j, mj) in enumerate(self.levels()):
            for ell in range(abs(mtot - mj), self.lmax + 1):
                if (iblock + n + ell + 1) % 2:
                    continue
                out.append((i, ell))
        return out

    def _legendre_term(self, lamb, col, row, mtot) -> float:
        s = self.spin
        (nc, jc, mjc), lc = col
        (nr, jr, mjr), lr = row
        mlc = mtot - mjc
        mlr = mtot - mjr
        mlam = mlr - mlc
        if abs(mlam) > lamb or mlam != mjc - mjr or (nc + lamb + nr) % 2 or (lc + lamb + lr) % 2:
            return 0.0
        fac1 = math.sqrt(float((2 * nc + 1) * (2 * nr + 1) * (2 * lc + 1) * (2 * lr + 1)))
        fac2 = _3j0(nc, lamb, nr) * _3j0(lc, lamb, lr) * threej(lc, lamb, lr, -mlc, -mlam, mlr)
        fac3 = (math.sqrt(float((2 * jc + 1) * (2 * jr + 1))) * _6j(jc, jr, lamb, nr, nc, s)
                * threej(jc, lamb, jr, -mjc, mlam, mjr))
        return _sgn(s + jc + jr + lamb + mlam - mtot) * fac1 * fac2 * fac3

    def _const_term(self, k, col, row, mtot, same) -> float:
        s = self.spin
        (nc, jc, mjc), lc = col
        (nr, jr, mjr), lr = row
        mlc = mtot - mjc
        mlr = mtot - mjr
        if k == 0:  # monomer rotation
            return float(nc * (nc + 1)) if same else 0.0
        if k == 1:  # spin-rotation
            if not same:
                return 0.0
            return _sgn(nc + jc + s) * math.sqrt(float(nc * (nc + 1) * (2 * nc + 1))) * _6j(s, nc, jc, nc, s, 1)
        if k == 2:  # spin-spin
            if jc == jr and mjc == mjr and lc == lr and mlc == mlr and (nc + nr) % 2 == 0:
                return (_sgn(jc + s) * math.sqrt(float((2 * nc + 1) * (2 * nr + 1))) * _6j(s, nr, jc, nc, s, 2)
                        * _3j0(nc, 2, nr))
            return 0.0
        # electron-spin Zeeman
        if nc == nr and mjc == mjr and lc == lr and mlc == mlr:
            return (self.fz * _sgn(nc + s + 1 - mjc) * math.sqrt(float((2 * jc + 1) * (2 * jr + 1)))
                    * _6j(s, jr, nc, jc, s, 1) * threej(jc, 1, jr, -mjc, 0, mjc))
        return 0.0

    def coupling(self, mtot: int, iblock: int) -> O.Coupling:
        """VL(NHAM, N(N+1)/2) with NHAM = MXLAM + 4 (CPL9), EINT the level
        energies of SET9 (unused by W: NCONST > 0), CENT = L(L+1)."""
        lev = self.levels()
        ch = self.channels(mtot, iblock)
        n = len(ch)
        mxlam = len(self.lam)
        nham = mxlam + 4
        vl = np.zeros(nham * n * (n + 1) // 2)
        idx = 0
        for icol in range(n):
            col = (lev[ch[icol][0]], ch[icol][1])
            for irow in range(icol + 1):
                row = (lev[ch[irow][0]], ch[irow][1])
                for t, lamb in enumerate(self.lam):
                    vl[idx + t] = self._legendre_term(lamb, col, row, mtot)
                for k in range(4):
                    vl[idx + mxlam + k] = self._const_term(k, col, row, mtot, icol == irow)
                idx += nham
        eint = np.array([self.cm2ru * self.level_energy(*lev[i]) for i, _ in ch])
        cent = np.array([float(ell * (ell + 1)) for _, ell in ch])
        return O.Coupling(n=n, nham=nham, vl=vl, eint=eint, cent=cent, nconst=4)

    def level_energy(self, n: int, j: int, mj: int) -> float:
        """Zero-field diagonal energy of SET9 (cm-1)."""
        s = self.spin
        fr, fs = self.vconst[1], self.vconst[2]
        diagr = self.roti[0] * float(n * (n + 1))
        diagsr = fr * math.sqrt(float(n * (n + 1) * (2 * n + 1))) * _6j(s, n, j, n, s, 1)
        if (n + j + s) % 2:
            diagsr = -diagsr
        diagss = fs * float(2 * n + 1) * _6j(s, n, j, n, s, 2) * _3j0(n, 2, n)
        if (j + s) % 2:
            diagss = -diagss
        return diagr + diagsr + diagss

    def _diag_b(self, n, j, mj, bfield) -> float:
        s = self.spin
        d = bfield * self.fz * (2 * j + 1) * threej(j, 1, j, -mj, 0, mj) * _6j(j, j, 1, s, s, n)
        return -d if (n + s + 1 - mj) % 2 else d

    def threshold(self, monqn) -> float:
        """EREF (cm-1) of the monomer state MONQN = (n, j, m_j) in the
        field (THRSH9): diagonal, or the lower/upper root of the 2x2 block
        n = j -+ 1 that the spin-spin term mixes."""
        s = self.spin
        n, j, mj = monqn
        b = self.field
        fs = self.vconst[2]
        if n == j or j >= self.nmax:
            return self.level_energy(n, j, mj) + self._diag_b(n, j, mj, b)
        em = self.level_energy(j - 1, j, mj) + self._diag_b(j - 1, j, mj, b)
        ep = self.level_energy(j + 1, j, mj) + self._diag_b(j + 1, j, mj, b)
        nn = j + 1
        odss = fs * math.sqrt(float(2 * nn + 1) * (2 * nn - 3)) * _6j(s, j - 1, j, j + 1, s, 2) * _3j0(j - 1, 2, j + 1)
        dif = math.sqrt((em - ep) ** 2 + 4.0 * odss ** 2)
        return 0.5 * (em + ep + math.copysign(dif, float(n - j)))

    def pvec(self, r: float) -> np.ndarray:
        """The P vector SUMLAM receives (hammat.f:37-83): the radial terms,
        then VCONST, all in reduced units."""
        p = self.pot.vlam(r, len(self.lam))
        p = np.where(np.abs(p) > 1.0e60, np.sign(p) * 1.0e60, p)
        ep2cm = self.ep2ru / self.cm2ru
        pc = np.array([v / ep2cm for v in self.vconst])
        return self.ep2ru * np.concatenate([p, pc])
