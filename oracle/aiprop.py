"""CPU ORACLE -- TEST INFRASTRUCTURE ONLY.

The AIRY log-derivative propagator (MOLSCAT IPROP = 9; Alexander,
J. Chem. Phys. 81, 4510 (1984); Alexander and Manolopoulos, J. Chem. Phys.
86, 2044 (1987)), restated for the long-range segment:

* sector loop, basis changes, node count, step control .. aiprop.f:120-380
* W at the two Gauss-Legendre points, local basis, dW/dR . potent.f:55-110
* error estimates CDIAG / COFF ........................... corr.f:43-75
* eigenvalues at RSTART .................................. waveig.f:30-47

In every sector [R_L, R_L + h] the wavevector matrix -W is diagonalised at
the midpoint (its average over the two Gauss-Legendre points) and each local
channel sees the linear reference k_i^2(R) = E_i - s_i (R - R_mid), s_i the
diagonal of the local dW/dR.  The log-derivative crosses the sector by
invariant imbedding, Z <- Y4 - Y2 (Y1 + Z)^-1 Y2, with the diagonal Y1, Y2,
Y4 of the exact solutions of the linear reference (Airy functions).  Those
three numbers per channel are the sector's whole physics; the reference
evaluates them with moduli and phases or an asymptotic series
(spropn.f); this restatement evaluates them from Ai, Bi and their
derivatives directly (scipy's exponentially scaled Airy functions, with the
growth factors exp(+-zeta) carried separately and their ratios formed from a
cancellation-free zeta difference), and switches to mpmath at raised
precision where the oscillatory phase zeta is so large (zeta > 1e6) that a
double-precision phase would lose more than 1e-9.  Both evaluate the same
mathematical functions.

The sector constant sqrt(3) is the reference's own 1.732050807 (potent.f:51).
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

SQ3 = 1.732050807  # potent.f:51
_ZETA_MP = 1.0e6


def _w(c: O.Coupling, sysm, r: float, ered: float) -> np.ndarray:
    return O.hammat(c, r, sysm.pvec(r), ered)


_Z_ASYM = 1.0e4  # above this the asymptotic series (4 terms) is exact to ~1e-22


def _asym_coeffs(nterm: int = 4):
    """u_k = Gamma(3k + 1/2) / (54^k k! Gamma(k + 1/2)), v_k = -(6k+1)/(6k-1) u_k
    (Abramowitz and Stegun 10.4.58-10.4.67)."""
    u = [1.0]
    v = [1.0]
    for k in range(1, nterm):
        uk = math.exp(math.lgamma(3 * k + 0.5) - k * math.log(54.0) - math.lgamma(k + 1) - math.lgamma(k + 0.5))
        u.append(uk)
        v.append(-(6 * k + 1) / (6 * k - 1) * uk)
    return u, v


_U, _V = _asym_coeffs()


def _airy_asym(z: np.ndarray):
    """Scaled Ai, Ai', Bi, Bi' for large positive z from the asymptotic
    series in 1/zeta (scipy's airye overflows internally near z ~ 1e6)."""
    zeta = 2.0 / 3.0 * z * np.sqrt(z)
    q = z ** 0.25
    sp = math.sqrt(math.pi)
    su_a = sum(((-1) ** k) * _U[k] / zeta ** k for k in range(len(_U)))
    sv_a = sum(((-1) ** k) * _V[k] / zeta ** k for k in range(len(_V)))
    su_b = sum(_U[k] / zeta ** k for k in range(len(_U)))
    sv_b = sum(_V[k] / zeta ** k for k in range(len(_V)))
    return su_a / (2.0 * sp * q), -q * sv_a / (2.0 * sp), su_b / (sp * q), q * sv_b / sp


def _airy_all(z: np.ndarray):
    """(Ai, Ai', Bi, Bi') at z as mantissas with the growth exponent zeta+
    (zeta = 2/3 z^1.5 for z > 0, else 0): Ai = a e^-zeta+, Bi = b e^+zeta+."""
    from scipy.special import airy, airye
    z = np.asarray(z, dtype=np.float64)
    zp = np.where(z > 0.0, z, 0.0)
    zeta = 2.0 / 3.0 * zp * np.sqrt(zp)
    a, ap, b, bp = airy(np.where(z > 0.0, 0.0, z))
    mid = (z > 0.0) & (z <= _Z_ASYM)
    ea, eap, eb, ebp = airye(np.where(mid, z, 0.0))
    big = z > _Z_ASYM
    xa, xap, xb, xbp = _airy_asym(np.where(big, z, 2.0 * _Z_ASYM))
    a = np.where(big, xa, np.where(mid, ea, a))
    ap = np.where(big, xap, np.where(mid, eap, ap))
    b = np.where(big, xb, np.where(mid, eb, b))
    bp = np.where(big, xbp, np.where(mid, ebp, bp))
    return a, ap, b, bp, zeta


def _zeta_diff(z1, z2, alpha_h):
    """zeta(z2) - zeta(z1) for z1, z2 > 0 without cancellation:
    (2/3)(z2^3 - z1^3)/(z2^1.5 + z1^1.5), z2 - z1 = alpha*h."""
    num = alpha_h * (z2 * z2 + z1 * z2 + z1 * z1)
    return 2.0 / 3.0 * num / (z2 * np.sqrt(z2) + z1 * np.sqrt(z1))


def _y124_mp(alpha, beta, width):
    """The same three numbers at raised precision: z1 and z2 are formed from
    the double inputs in mpmath, so their difference alpha*h keeps its
    digits however large z is."""
    import mpmath as mp
    zeta = 2.0 / 3.0 * (abs(alpha) * (abs(beta) + abs(width))) ** 1.5
    with mp.workdps(int(25 + 2 * math.log10(max(zeta, 10.0)))):
        al, be, h = mp.mpf(alpha), mp.mpf(beta), mp.mpf(width)
        z1 = al * (be - h / 2)
        z2 = al * (be + h / 2)
        a1, b1 = mp.airyai(z1), mp.airybi(z1)
        ap1, bp1 = mp.airyai(z1, 1), mp.airybi(z1, 1)
        a2, b2 = mp.airyai(z2), mp.airybi(z2)
        ap2, bp2 = mp.airyai(z2, 1), mp.airybi(z2, 1)
        d = a1 * b2 - b1 * a2
        y1 = al * (bp1 * a2 - ap1 * b2) / d
        y4 = al * (a1 * bp2 - b1 * ap2) / d
        y2 = al / mp.pi / d
        return float(y1), float(y2), float(y4)


def sector_y124(width: float, eig: np.ndarray, hp: np.ndarray):
    """Diagonal imbedding propagator (Y1, Y2, Y4) of one sector for every
    local channel: exact solutions of psi'' = [s x - E] psi on
    x in [-h/2, h/2] (E = eig, s = hp), in the form
    psi'(a) = -Y1 psi(a) + Y2 psi(b),  psi'(b) = -Y2 psi(a) + Y4 psi(b)."""
    s = np.where(hp == 0.0, 1.0e-30, hp)
    alpha = np.sign(s) * np.abs(s) ** (1.0 / 3.0)
    beta = -eig / s
    z1 = alpha * (beta - 0.5 * width)
    z2 = alpha * (beta + 0.5 * width)
    a1, ap1, b1, bp1, zt1 = _airy_all(z1)
    a2, ap2, b2, bp2, zt2 = _airy_all(z2)
    both = (z1 > 0.0) & (z2 > 0.0)
    e1 = np.where(both, _zeta_diff(np.where(both, z1, 1.0), np.where(both, z2, 1.0), alpha * width), zt2 - zt1)
    m = np.abs(e1)
    ep, em = np.exp(e1 - m), np.exp(-e1 - m)
    d = a1 * b2 * ep - b1 * a2 * em
    y1 = alpha * (bp1 * a2 * em - ap1 * b2 * ep) / d
    y4 = alpha * (a1 * bp2 * ep - b1 * ap2 * em) / d
    y2 = alpha / math.pi * np.exp(-m) / d
    osc = np.maximum(np.where(z1 < 0.0, 2.0 / 3.0 * np.abs(z1) ** 1.5, 0.0),
                     np.where(z2 < 0.0, 2.0 / 3.0 * np.abs(z2) ** 1.5, 0.0))
    for i in np.nonzero(osc > _ZETA_MP)[0]:
        y1[i], y2[i], y4[i] = _y124_mp(float(alpha[i]), float(beta[i]), float(width))
    return y1, y2, y4


def _potent(c, sysm, rnow: float, drnow: float, ered: float):
    """potent.f:55-110: eigenvalues (ascending) and eigenvectors of the
    average wavevector matrix -(W(RA) + W(RB))/2, the local diagonal of
    dW/dR = sqrt(3)(W(RB) - W(RA))/DR and its largest off-diagonal element."""
    ra = rnow - 0.5 * drnow / SQ3
    rb = rnow + 0.5 * drnow / SQ3
    wa = _w(c, sysm, ra, ered)
    wb = _w(c, sysm, rb, ered)
    avg = -0.5 * (wb + wa)
    dw = (SQ3 / drnow) * (wb - wa)
    eig, vec = np.linalg.eigh(avg)
    loc = vec.T @ dw @ vec
    loc = 0.5 * (loc + loc.T)
    hp = np.diag(loc).copy()
    off = np.abs(np.tril(loc, -1))
    xlarge = float(off.max()) if c.n > 1 else 0.0
    return eig, vec, hp, xlarge


def _corr(eignow, eigold, hp, drnow, drmid, xlarge):
    """corr.f:43-75: estimated errors of the neglected diagonal second
    derivative (CDIAG) and off-diagonal first derivative (COFF)."""
    fct = 2.0 / drmid ** 2
    w2p = -fct * (eignow - eigold + drmid * hp)
    cdiag = float(np.mean(np.abs(w2p)))
    cay = float(np.mean(np.sqrt(np.abs(eignow))))
    cdiag = abs(drnow ** 3) * cdiag / 12.0
    coff = cay * xlarge * abs(drnow ** 3) / 12.0
    return cdiag, coff


def drcalc(rstart: float, rstop: float, kstep: int, nstep: int, pow_: float) -> float:
    """Size of step KSTEP (0-based) when the step boundaries are equally
    spaced in R^(1-POW) (drcalc.f:22-38)."""
    powint = 1.0 - pow_
    powinv = 1.0 / powint
    if powint != 0.0:
        zstart = rstart ** powint
        zstop = rstop ** powint
        dz = (zstop - zstart) / float(nstep)
        rnow = (zstart + float(kstep + 1) * dz) ** powinv
        rlast = (zstart + float(kstep) * dz) ** powinv
        return rnow - rlast
    dz = rstart * ((rstop / rstart) ** (1.0 / float(nstep)) - 1.0)
    return dz * (1.0 + dz / rstart) ** kstep


def drset(rstart: float, rstop: float, drfit: float, tolhi: float, pow_: float):
    """(NSTEP, first DR) of a segment whose step is set from DRS/DRL
    (drset.f:54-84): with TOLHI = 0 a whole number of steps scaling as
    R^POW, the first one DR; with 0 < TOLHI < 1 just DRFIT (NSTEP 0)."""
    rsmall = min(rstart, rstop)
    rlarge = max(rstart, rstop)
    powint = 1.0 - pow_
    prange = rlarge - rsmall
    nstep = 0
    dr = drfit
    if tolhi == 0.0:
        rratio = drfit / rsmall
        if pow_ == 0.0:
            nstep = max(O.nint(prange / drfit), 1)
            dr = prange / float(nstep)
        elif pow_ == 1.0:
            nstep = O.nint(math.log(rlarge / rsmall) / math.log(rratio + 1.0))
            dr = drcalc(rstart, rstop, 0, nstep, pow_)
        else:
            zrm1 = (rlarge / rsmall) ** powint - 1.0
            nstep = O.nint(zrm1 / ((rratio + 1.0) ** powint - 1.0))
            dr = drcalc(rstart, rstop, 0, nstep, pow_)
    if rstop < rstart:
        dr = -abs(dr)
    return nstep, dr


def aiprop(c: O.Coupling, sysm, z: np.ndarray, rstart: float, rstop: float, drnow: float, ered: float,
           tolhi: float = 1.0e-4, powr: float = 3.0, maxstp: int = 500000, nstep: int = 0):
    """AIPROP from RSTART to RSTOP, outward or inward (DRNOW < 0), variable
    steps controlled by TOLHI and POWR (aiprop.f:305-330), or with TOLHI = 0
    NSTEP steps scaling as R^POWR (DRCALC, aiprop.f:320-328).  z:
    log-derivative at RSTART in the free basis.  Returns (Z at RSTOP, NODES,
    number of sectors).  Inward, a sector adds N - KOUNT nodes
    (aiprop.f:196-200) and the step factor carries (1 + DR/R)^3 for the
    rising potential (aiprop.f:317-318)."""
    if tolhi == 0.0 and nstep < 1:
        raise ValueError("TOLHI = 0 needs NSTEP (drset)")
    if rstop == rstart or (rstop > rstart) != (drnow > 0.0):
        raise ValueError("DRNOW must point from RSTART to RSTOP")
    outward = rstop > rstart
    n = c.n
    z = np.array(z, dtype=np.float64)
    eigold = np.linalg.eigvalsh(-_w(c, sysm, rstart, ered))
    nodes = 0
    drmid = 0.5 * drnow
    rlast = rstart
    rnow = rlast + drmid
    rnext = rlast + drnow
    last = False
    vecnow = None
    kstep = 0
    for kstep in range(1, maxstp + 1):
        eig, vec, hp, xlarge = _potent(c, sysm, rnow, drnow, ered)
        if vecnow is None:
            tmat = vec
        else:
            tmat = vecnow.T @ vec  # E_old^T E_new: old local basis -> new local basis
        vecnow = vec
        z = tmat.T @ z @ tmat
        z = 0.5 * (z + z.T)
        cdiag, coff = _corr(eig, eigold, hp, drnow, drmid, xlarge)
        eigold = eig
        y1, y2, y4 = sector_y124(drnow, eig, hp)
        a = z + np.diag(y1)
        inv, kount = O.syminv(a)
        if kount > n:
            raise RuntimeError("AIPROP: instability in SYMINV")
        nodes += kount if outward else n - kount
        inv = np.tril(inv) + np.tril(inv, -1).T
        z = -(y2[:, None] * inv * y2[None, :]) + np.diag(y4)
        if last:
            break
        if 0.0 < tolhi < 1.0:
            cmax = max(abs(cdiag), abs(coff))
            factor = 2.0 if cmax == 0.0 else (tolhi / cmax) ** (1.0 / powr)
            if drnow < 0.0 and rnext + drnow > 0.0:
                factor = factor * (1.0 + drnow / rnext) ** 3
            if factor > 2.0:
                factor = 2.0
            drnow = drnow * factor
            rlast = rnext
            rnext = rnext + drnow
            last = (rstop - rstart) * (rstop - rnext) < 0.0
        elif tolhi == 0.0:
            drnow = drcalc(rstart, rstop, kstep, nstep, powr)
            rlast = rnext
            rnext = rnext + drnow
            last = nstep - kstep <= 1
        else:
            raise ValueError("the restatement covers 0 <= TOLHI < 1")
        if last:
            rnext = rstop
            drnow = rnext - rlast
        rnew = rlast + 0.5 * drnow
        drmid = rnew - rnow
        rnow = rnew
    z = vecnow @ z @ vecnow.T
    return 0.5 * (z + z.T), nodes, kstep


def molscat_two_segment(sysm, c: O.Coupling, energy_cm: float, rmin: float, rmax: float, steps: float,
                        irmset: int, rvfac: float, tolhi: float = 1.0e-4, powr: float = 3.0, short_range=None):
    """One (JTOT, block) of a MOLSCAT run at one energy with LDMD from RMIN
    to RMID and AIRY from RMID to RMAX (mol.driver.f:1488-1549 with NSEG = 2:
    FINDRM at the energy, RMID = RTURN*RVFAC, CAYS = CAYL = CALCK(0, E);
    scpset.f:27-55 and drset.f:33-66 for the segments: LDMD in whole steps of
    about pi/(CAY*STEPS), AIRY starting from that step size).

    short_range(rtab, ptab, nstep, dr, ered, y0) -> (Y, NODES) runs the
    LDMD segment (default: the oracle's MDPROP).  Returns a dict with the
    S matrix (SR, SI in CHNSRT order), NOPEN, NB, the radii and step counts."""
    ered = energy_cm * sysm.cm2ru
    rstart, rturn = O.findrm(sysm, c, rmin, ered, irmset)
    rmid = rturn * rvfac
    cay = O.calck(0.0, ered, c.eint)
    nstep, dr = O.drset_fixed(rstart, rmid, steps, cay)
    rtab = O.radial_grid(rstart, dr, nstep)
    ptab = O.ptable(sysm, rtab)
    y0 = O.yinit_adiabatic_wkb(sysm, c, rstart, ered)
    if short_range is None:
        y, nodes, st, kf = O.mdprop(c, rtab, ptab, nstep, dr, ered, y0)
        if st != 0:
            raise RuntimeError(f"MDPROP: inversion error at step {kf}")
    else:
        y, nodes = short_range(rtab, ptab, nstep, dr, ered, y0)
    dr_airy = math.pi / (cay * steps)
    z, nodes_l, nsect = aiprop(c, sysm, y, float(rtab[-1]), rmax, dr_airy, ered, tolhi, powr)
    wvec, nopen = O.gtwvec(ered, c.eint)
    nb = O.chnsrt(c.eint)
    k = O.ytok(nb, wvec, c.n, nopen, z, rmax, c.cent)
    sr, si = O.ktos(k)
    return {"sr": sr, "si": si, "nopen": nopen, "nb": nb, "wvec": wvec, "rstart": rstart, "rmid": float(rtab[-1]),
            "nstep": nstep, "dr": dr, "sectors": nsect, "nodes": nodes + nodes_l, "y_rmid": y}


def partial_cross_sections(sysm, c: O.Coupling, ch, res, jtot: int) -> dict:
    """State-to-state partial cross sections (Angstrom^2) of one (JTOT,
    block) between rotor levels (sproc.f:371-430 with JHALF = 1, no
    weights): sigma(i -> f) = pi (2 JTOT + 1) / ((2 j_i + 1) k_i^2)
    * sum over open channels of |delta - S|^2, k_i in 1/Angstrom.  Keys are
    (final level, initial level), 1-based as printed."""
    sr, si, nopen, nb, wvec = res["sr"], res["si"], res["nopen"], res["nb"], res["wvec"]
    lev = [sysm.states[ch[nb[i]][0]].level + 1 for i in range(nopen)]
    jlev = {sysm.states[s].level + 1: sysm.states[s].j for s, _ in ch}
    xj = (2 * jtot + 1) * math.pi
    out = {}
    for icol in range(nopen):
        for irow in range(nopen):
            smag = sr[irow, icol] ** 2 + si[irow, icol] ** 2
            if irow == icol:
                smag = (1.0 - sr[irow, icol]) ** 2 + si[irow, icol] ** 2
            kk = (wvec[nb[irow]] / sysm.rm) ** 2
            key = (lev[icol], lev[irow])
            out[key] = out.get(key, 0.0) + smag * xj / ((2 * jlev[lev[irow]] + 1) * kk)
    return out
