"""Host-side input builders for the propagator (they stay on the host in the
reference too): the ITYPE=1 atom + rigid linear rotor basis and couplings
(source_code/base.f:276-345, couple.f:52-133, base.f:388-410), the
power/exponential potential of POTENL's evaluation case 1 (potenl.f), a
WKB diagonal initial log-derivative (yinit.f:96-110 with ADIAMN off) and the
seeded synthetic workloads the benchmark and tests use:

* ``rotor_system()``: URED 4.0 amu, B 60 cm-1, even j = 0..10,
  V0 = eps[(Rm/R)^12 - 2(Rm/R)^6], V2 = 0.3 eps exp(-(R-Rm)/0.4 A) - 0.1 eps (Rm/R)^6,
  eps = 50 cm-1, Rm = 3.5 A; LDMD from 2.5 to 40 A in 4000 steps.
* ``single_workload()``: JTOT = 10, one parity (N = 30), E = 150 cm-1.
* ``batched_workload()``: JTOT = 0..80, both parities (N = 6..36), 512
  energies drawn uniformly in 1-500 cm-1 from numpy's default_rng(20261203).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from fractions import Fraction
from functools import lru_cache

import numpy as np

from .propagators import Coupling, Segment

# CODATA 2022 values as in source_code/physical_constants_module.f
_H = 6.62607015e-34
_C = 2.99792458e8
_U = 1.66053906892e-27
_PI = 3.141592653589793
BFCT = (_H / 2.0 / _PI) / (4.0 * _PI * (_C * 1.0e2)) / (1.0e-10) ** 2 / _U  # cm-1 A^2 amu


@lru_cache(maxsize=None)
def _f(n: int) -> int:
    return math.factorial(n)


@lru_cache(maxsize=None)
def w3j_zero(a: int, b: int, c: int) -> float:
    """Wigner 3j (a b c; 0 0 0), integer arguments."""
    s = a + b + c
    if s & 1 or c < abs(a - b) or c > a + b:
        return 0.0
    g = s // 2
    sq = Fraction(_f(s - 2 * a) * _f(s - 2 * b) * _f(s - 2 * c), _f(s + 1))
    v = math.sqrt(sq) * _f(g) / (_f(g - a) * _f(g - b) * _f(g - c))
    return -v if g & 1 else v


def _tri2(a, b, c) -> Fraction:
    return Fraction(_f(a + b - c) * _f(a - b + c) * _f(b + c - a), _f(a + b + c + 1))


@lru_cache(maxsize=None)
def w6j(j1: int, j2: int, j3: int, l1: int, l2: int, l3: int) -> float:
    """Wigner 6j {j1 j2 j3; l1 l2 l3}, integer arguments."""
    for x, y, z in ((j1, j2, j3), (j1, l2, l3), (l1, j2, l3), (l1, l2, j3)):
        if z < abs(x - y) or z > x + y:
            return 0.0
    a1, a2, a3, a4 = j1 + j2 + j3, j1 + l2 + l3, l1 + j2 + l3, l1 + l2 + j3
    b1, b2, b3 = j1 + j2 + l1 + l2, j2 + j3 + l2 + l3, j3 + j1 + l3 + l1
    tot = 0
    for t in range(max(a1, a2, a3, a4), min(b1, b2, b3) + 1):
        term = Fraction(_f(t + 1), _f(t - a1) * _f(t - a2) * _f(t - a3) * _f(t - a4)
                        * _f(b1 - t) * _f(b2 - t) * _f(b3 - t))
        tot += -term if t & 1 else term
    if tot == 0:
        return 0.0
    d = _tri2(j1, j2, j3) * _tri2(j1, l2, l3) * _tri2(l1, j2, l3) * _tri2(l1, l2, j3)
    return math.copysign(math.sqrt(d * tot * tot), float(tot))


@dataclass
class RotorAtom:
    """MOLSCAT ITYPE=1 system (atom + rigid linear rotor)."""
    ured: float               # reduced mass, amu
    be: float                 # rotational constant, cm-1
    jlevel: tuple             # rotor levels in the basis
    lam: tuple                # Legendre order of each potential term
    terms: tuple              # per term: ((A, NPOWER, E or None), ...), R in RM units
    rm: float                 # length unit RM (Angstrom), also RUNIT
    epsil: float              # energy unit EPSIL (cm-1)

    @property
    def cm2ru(self) -> float:
        return self.ured * self.rm * self.rm / BFCT  # mol.driver.f:734

    @property
    def ep2ru(self) -> float:
        return self.epsil * self.cm2ru

    def channels(self, jtot: int, block: int):
        """[(level index, L)], ordered on L then level (base.f:276-345)."""
        ipty = block % 2
        jmax, jmin = max(self.jlevel), min(self.jlevel)
        lmin = jtot - jmax
        if lmin < 0:
            lmin = max(jmin - jtot, 0)
        out = []
        for l in range(lmin, jtot + jmax + 1):
            for i, j in enumerate(self.jlevel):
                if (l + j + jtot) % 2 == ipty and abs(jtot - l) <= j <= jtot + l:
                    out.append((i, l))
        return out

    def coupling(self, jtot: int, block: int) -> Coupling:
        """VL(NHAM, N(N+1)/2) of Percival-Seaton coefficients (couple.f:52-133)."""
        ch = self.channels(jtot, block)
        n = len(ch)
        nham = len(self.lam)
        vl = np.zeros(nham * n * (n + 1) // 2)
        k = 0
        for col in range(n):
            jc, lc = self.jlevel[ch[col][0]], ch[col][1]
            for row in range(col + 1):
                jr, lr = self.jlevel[ch[row][0]], ch[row][1]
                pre = math.sqrt((2 * jc + 1) * (2 * jr + 1) * (2 * lc + 1) * (2 * lr + 1))
                sgn = -1.0 if (jc + jr + jtot) & 1 else 1.0
                for t, lam in enumerate(self.lam):
                    vl[k + t] = sgn * pre * w3j_zero(jc, lam, jr) * w3j_zero(lc, lam, lr) * w6j(jr, lr, jtot, lc, jc, lam)
                k += nham
        eint = np.array([self.cm2ru * self.be * self.jlevel[i] * (self.jlevel[i] + 1) for i, _ in ch])
        cent = np.array([float(l * (l + 1)) for _, l in ch])
        return Coupling(n=n, nham=nham, vl=vl, eint=eint, cent=cent)

    def potenl(self, r: float) -> np.ndarray:
        """Radial coefficients in units of EPSIL, R in units of RM."""
        out = np.zeros(len(self.lam))
        for t, tl in enumerate(self.terms):
            acc = 0.0
            for a, npw, e in tl:
                if npw:
                    rr = 1.0e-8 if (npw < 0 and abs(r) < 1.0e-8) else r
                    acc += a * rr ** npw
                else:
                    acc += a * math.exp(e * r)
            out[t] = acc
        return out

    def pvec(self, r: float) -> np.ndarray:
        p = self.potenl(r)
        p = np.clip(p, -1.0e60, 1.0e60)
        return self.ep2ru * p


def rotor_system() -> RotorAtom:
    """The atom + linear rotor system of the single and batched workloads."""
    return RotorAtom(ured=4.0, be=60.0, jlevel=(0, 2, 4, 6, 8, 10), lam=(0, 2),
                     terms=(((1.0, -12, None), (-2.0, -6, None)),
                            ((0.3 * math.exp(8.75), 0, -8.75), (-0.1, -6, None))),
                     rm=3.5, epsil=50.0)


ROTOR_RMIN_A = 2.5
ROTOR_RMAX_A = 40.0
ROTOR_NSTEP = 4000


def wkb_initial_y(c: Coupling, pvec0: np.ndarray, r0: float, ered: float, bcyomn: float = 0.0) -> np.ndarray:
    """Diagonal initial log-derivative from the diabatic W at RSTART:
    sqrt(W_ii) for locally closed channels, BCYOMN otherwise (yinit.f:96-117)."""
    n = c.n
    w = np.zeros(n)
    idx = 0
    for j in range(n):
        idx = (j * (j + 1) // 2 + j) * c.nvlblk
        w[j] = float(np.dot(c.vl[idx:idx + c.nham], pvec0[:c.nham]))
    w = w + min(1.0 / (r0 * r0), 1.0e16) * c.cent + c.eint - ered
    y = np.where(w > 0.0, np.sqrt(np.abs(w)), bcyomn)
    return np.diag(y)


@dataclass
class Workload:
    name: str
    systems: list
    segments: list
    job_sys: np.ndarray
    job_ered: np.ndarray
    job_y0: list
    labels: list

    @property
    def njobs(self) -> int:
        return len(self.job_sys)

    def channel3_steps(self) -> float:
        return float(sum(self.systems[s].n ** 3 * self.segments[s].nstep for s in self.job_sys))


def _rotor_jobs(jtots, blocks, energies_cm, name, nstep=ROTOR_NSTEP):
    sysm = rotor_system()
    rmin = ROTOR_RMIN_A / sysm.rm
    rmax = ROTOR_RMAX_A / sysm.rm
    dr = (rmax - rmin) / nstep
    systems, segments, labels = [], [], []
    job_sys, job_ered, job_y0 = [], [], []
    seg_cache = None
    for jt in jtots:
        for b in blocks:
            if not sysm.channels(jt, b):
                continue
            c = sysm.coupling(jt, b)
            if seg_cache is None:
                seg_cache = Segment.build(rmin, dr, nstep, sysm.pvec, c.nham)
            s = len(systems)
            systems.append(c)
            segments.append(seg_cache)
            labels.append((jt, b))
            for e in energies_cm:
                ered = e * sysm.cm2ru
                job_sys.append(s)
                job_ered.append(ered)
                job_y0.append(wkb_initial_y(c, seg_cache.ptab[0], seg_cache.rtab[0], ered))
    return Workload(name, systems, segments, np.array(job_sys, dtype=np.int32), np.array(job_ered),
                    job_y0, labels)


def single_workload() -> Workload:
    """JTOT=10, parity block 1 (N=30), E=150 cm-1, 4000 LDMD steps 2.5-40 A."""
    return _rotor_jobs([10], [1], [150.0], "rotor J=10 block 1 N=30, E=150 cm-1, 4000 steps")


def batched_energies(count: int = 512, seed: int = 20261203) -> np.ndarray:
    return np.random.default_rng(seed).uniform(1.0, 500.0, size=count)


def batched_workload(n_energies: int = 512, jmax: int = 80, seed: int = 20261203, jtots=None,
                     nstep: int = ROTOR_NSTEP) -> Workload:
    """JTOT=0..jmax, both parity blocks, n_energies seeded energies."""
    jt = list(range(0, jmax + 1)) if jtots is None else list(jtots)
    e = batched_energies(n_energies, seed)
    return _rotor_jobs(jt, [1, 2], e, f"rotor JTOT=0..{jmax} x 2 parities x {n_energies} energies, {nstep} steps",
                       nstep=nstep)


def batched_workload_shard(rank: int, world: int, n_energies: int = 512, jmax: int = 80,
                           seed: int = 20261203, nstep: int = ROTOR_NSTEP) -> Workload:
    """This rank's part of the multi-GPU batched workload (weak scaling): the
    JTOT = 0..jmax x 2 parities blocks at world * n_energies seeded energies,
    cut into units of one block and n_energies energies, the units spread
    over ranks by LPT on N^3 * NSTEP * energies (sharding.lpt_partition), so
    every rank holds about one GPU's worth of the single-GPU workload and a
    block's energies on a rank share its 2HQ(C) table."""
    from .sharding import rank_units
    sysm = rotor_system()
    e_all = batched_energies(n_energies * world, seed)
    units = [(jt, b, k) for jt in range(jmax + 1) for b in (1, 2) if sysm.channels(jt, b) for k in range(world)]
    costs = [len(sysm.channels(jt, b)) ** 3 * float(nstep) * n_energies for jt, b, _ in units]
    mine = [units[i] for i in rank_units(costs, rank, world)]
    rmin, rmax = ROTOR_RMIN_A / sysm.rm, ROTOR_RMAX_A / sysm.rm
    dr = (rmax - rmin) / nstep
    seg = None
    systems, segments, labels, job_sys, job_ered, job_y0 = [], [], [], [], [], []
    sys_of = {}
    for jt, b, k in mine:
        if (jt, b) not in sys_of:
            c = sysm.coupling(jt, b)
            if seg is None:
                seg = Segment.build(rmin, dr, nstep, sysm.pvec, c.nham)
            sys_of[(jt, b)] = len(systems)
            systems.append(c)
            segments.append(seg)
            labels.append((jt, b))
        s = sys_of[(jt, b)]
        for e in e_all[k * n_energies:(k + 1) * n_energies]:
            ered = e * sysm.cm2ru
            job_sys.append(s)
            job_ered.append(ered)
            job_y0.append(wkb_initial_y(systems[s], seg.ptab[0], seg.rtab[0], ered))
    return Workload(f"rotor JTOT=0..{jmax} x 2 parities x {n_energies * world} energies, rank {rank}/{world}",
                    systems, segments, np.array(job_sys, dtype=np.int32), np.array(job_ered), job_y0, labels)


def synthetic_system(n: int, nstep: int = 3000, seed: int = 0, nham: int = 6):
    """A dense coupled-channel system of exactly N channels for timing large
    and mixed N: NHAM Lennard-Jones 12-6 radial terms with seeded amplitudes
    and minima (R in units of the mean minimum, energies in the reduced units
    of the propagator), seeded symmetric couplings of every pair, thresholds
    and L values.  Returns (Coupling, Segment, ERED, Y0) with Y0 the diagonal
    WKB start of yinit.f:96-117."""
    rng = np.random.default_rng(seed)
    npair = n * (n + 1) // 2
    # pairs in SUMLAM order (sumlam.f:74-86): column by column, row <= column
    col = np.repeat(np.arange(n), np.arange(1, n + 1))
    row = np.arange(npair) - col * (col + 1) // 2
    diag = row == col
    scale = 0.3 / math.sqrt(max(1.0, n / 32.0))
    coef = rng.normal(0.0, scale, size=(npair, nham))
    coef[diag, 0] = 1.0
    coef[~diag, 0] = 0.0
    coef[diag, 1:] *= 0.3
    vl = np.ascontiguousarray(coef.ravel())
    eint = np.sort(rng.uniform(0.0, 60.0, n))
    lv = rng.integers(0, 30, n)
    cent = (lv * (lv + 1)).astype(np.float64)
    amp = np.concatenate([[200.0], rng.uniform(10.0, 60.0, nham - 1)])
    rmin = rng.uniform(0.95, 1.05, nham)

    def pvec(r: float) -> np.ndarray:
        x = rmin / r
        return amp * (x ** 12 - 2.0 * x ** 6)

    r0, r1 = 0.8, 8.0
    dr = (r1 - r0) / nstep
    seg = Segment.build(r0, dr, nstep, lambda r: pvec(r), nham)
    c = Coupling(n=n, nham=nham, vl=vl, eint=eint, cent=cent)
    ered = float(rng.uniform(20.0, 80.0))
    y0 = wkb_initial_y(c, seg.ptab[0], seg.rtab[0], ered)
    return c, seg, ered, y0
