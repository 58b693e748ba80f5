"""Seeded propagator inputs shared by the GPU parity tests (no GPU needed to
build them)."""
import math

import numpy as np

from molscat_b200.propagators import Coupling, Segment, radial_grid
from molscat_b200 import systems as S


def rotor_case(jtot, block, nstep=4000, energies_cm=(150.0,), rmin_a=2.5, rmax_a=40.0):
    """The benchmark rotor system at one (JTOT, block)."""
    sysm = S.rotor_system()
    c = sysm.coupling(jtot, block)
    rmin, rmax = rmin_a / sysm.rm, rmax_a / sysm.rm
    dr = (rmax - rmin) / nstep
    seg = Segment.build(rmin, dr, nstep, sysm.pvec, c.nham)
    jobs = []
    for e in energies_cm:
        ered = e * sysm.cm2ru
        jobs.append((ered, S.wkb_initial_y(c, seg.ptab[0], seg.rtab[0], ered)))
    return c, seg, jobs


def random_case(n, nstep, seed, nham_pot=3, ivlfl=0, nconst=0, nrsq=0, conlen=0.0, inward=False, kind="LD"):
    """A random but physical-looking coupled-channel problem: a Lennard-Jones
    isotropic term plus anisotropic exponential/power terms with random
    symmetric coupling coefficients, random thresholds and L values.

    nconst: thresholds enter through a VL term with constant P (EINT is then
    not added, hammat.f:95).  nrsq: L(L+1) enters through a VL term with
    P = min(1/R^2, 1e16) (hammat.f:77-83,89).  ivlfl: VL slots read P through
    a random permutation IV, and NVLBLK = NHAM+1 leaves a slot SUMLAM must
    skip.  inward: propagate from the long-range side in (DR < 0).  kind: the
    segment's radii ("LD", or "LDMG4"/"LDMG5" for MGPROP's stages); the
    potential is kept as seg.pvec(R)."""
    rng = np.random.default_rng(seed)
    npair = n * (n + 1) // 2
    eint = np.sort(rng.uniform(0.0, 60.0, n))
    lvals = rng.integers(0, 12, n)
    cent = (lvals * (lvals + 1)).astype(np.float64)
    nham = nham_pot + (1 if nconst else 0) + (1 if nrsq else 0)
    nvlblk = nham + (1 if ivlfl else 0)
    # coefficient of term t for pair (row, col), in P order
    coef = np.zeros((npair, nham))
    k = 0
    for col in range(n):
        for row in range(col + 1):
            if row == col:
                coef[k, 0] = 1.0
            for t in range(1, nham_pot):
                coef[k, t] = rng.normal(0.0, 0.3) if row != col else rng.normal(0.0, 0.1)
            t = nham_pot
            if nconst:
                coef[k, t] = eint[col] if row == col else 0.0
                t += 1
            if nrsq:
                coef[k, t] = cent[col] if row == col else 0.0
            k += 1
    vl = np.zeros(nvlblk * npair)
    iv = np.ones(nvlblk * npair, dtype=np.int32)
    for k in range(npair):
        if ivlfl:
            perm = rng.permutation(nham)
            for slot in range(nham):
                vl[k * nvlblk + slot] = coef[k, perm[slot]]
                iv[k * nvlblk + slot] = perm[slot] + 1
            vl[k * nvlblk + nham] = 123.0  # beyond NHAM: SUMLAM never reads it
        else:
            vl[k * nvlblk:k * nvlblk + nham] = coef[k]
    eps = 200.0
    amp = rng.uniform(0.5, 1.5, nham_pot)

    def pot(r):
        p = np.zeros(nham)
        p[0] = eps * (r ** -12 - 2.0 * r ** -6)
        for t in range(1, nham_pot):
            p[t] = eps * amp[t] * (math.exp(-3.0 * (r - 1.0)) - 0.2 * r ** -6)
        t = nham_pot
        if nconst:
            p[t] = 1.0
            t += 1
        if nrsq:
            p[t] = min(1.0 / (r * r), 1.0e16)
        return p

    r0, r1 = (6.0, 0.85) if inward else (0.85, 6.0)
    dr = (r1 - r0) / nstep
    if kind == "LD":
        rtab = radial_grid(r0, dr, nstep)
    else:
        from molscat_b200.propagators import ldmg_radii
        rtab = ldmg_radii(kind, r0, dr, nstep)
    ptab = np.stack([pot(float(r)) for r in rtab])
    c = Coupling(n=n, nham=nham, vl=vl, eint=eint, cent=cent, nvlblk=nvlblk, iv=iv if ivlfl else None,
                 ivlfl=ivlfl, nconst=nconst, nrsq=nrsq, conlen=conlen)
    seg = Segment(nstep, dr, rtab, ptab, kind)
    seg.pvec = pot
    ered = float(rng.uniform(20.0, 80.0))
    w0 = _diag_w(c, seg, 0, ered)
    sgn = -1.0 if inward else 1.0
    y0 = np.diag(np.where(w0 > 0, sgn * np.sqrt(np.abs(w0)), 0.0))
    return c, seg, ered, y0


def _diag_w(c, seg, ir, ered):
    r = seg.rtab[ir]
    p = seg.ptab[ir]
    w = np.zeros(c.n)
    for i in range(c.n):
        k = i * (i + 1) // 2 + i
        blk = c.vl[k * c.nvlblk:k * c.nvlblk + c.nham]
        if c.ivlfl > 0:
            idx = c.iv[k * c.nvlblk:k * c.nvlblk + c.nham] - 1
            w[i] = float(np.dot(blk, p[idx]))
        else:
            w[i] = float(np.dot(blk, p[:c.nham]))
    if c.nrsq == 0:
        w += min(1.0 / (r * r), 1e16) * c.cent
    if c.nconst == 0:
        w += c.eint
    if c.conlen > 0:
        w += r * r / c.conlen ** 4
    return w - ered


def to_oracle(c):
    from oracle import oracle as O
    return O.Coupling(n=c.n, nham=c.nham, vl=c.vl, eint=c.eint, cent=c.cent, nvlblk=c.nvlblk,
                      iv=c.iv if c.ivlfl > 0 else None, ivlfl=c.ivlfl, nconst=c.nconst, nrsq=c.nrsq,
                      conlen=c.conlen)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(1.0, np.abs(b).max()))


# ---------------------------------------------------------------------------
# large dense N on a physical basis: atom + rigid asymmetric top (ITYPE=6)
# ---------------------------------------------------------------------------
ASYM_ROTI = (9.6, 0.0, 4.3, 0.0, 2.8, 0.0, 0.0, 0.0, 0.0, 0.0)  # A, B, C (cm-1)
ASYM_LAMBDA = [(0, 0), (1, 0), (2, 0), (2, 2), (3, 2), (4, 4)]
ASYM_URED = 12.0
ASYM_R = (2.8, 30.0)  # Angstrom (RM = 1 Angstrom)
# (level cutoff cm-1, JTOT, block, channels kept): below 400 cm-1 the largest
# block has 500 channels, so the N = 1024 block takes levels below 700 cm-1
ASYM_BLOCKS = {256: (400.0, 4, 1, 256), 512: (400.0, 10, 2, 500), 1024: (700.0, 10, 1, 1024)}


def asym_top_system(emax_cm: float, seed: int = 20261203):
    """The large-N workload's physical basis: an asymmetric top (A 9.6,
    B 4.3, C 2.8 cm-1) with its levels below emax_cm, and six V(lambda, mu)
    Lennard-Jones 12-6 terms with seeded well depths 5-40 cm-1 (the
    isotropic term the deepest) and minima 3.6-4.0 Angstrom."""
    from oracle import itype6 as I6
    rng = np.random.default_rng(seed)
    amp = np.sort(rng.uniform(5.0, 40.0, len(ASYM_LAMBDA)))[::-1].copy()
    rmn = rng.uniform(3.6, 4.0, len(ASYM_LAMBDA))

    def pfunc(r):
        x = rmn / r
        return amp * (x ** 12 - 2.0 * x ** 6)

    return I6.Itype6(ured=ASYM_URED, roti=ASYM_ROTI, jmax=30, lam=ASYM_LAMBDA, pfunc=pfunc, rm=1.0, epsil=1.0,
                     emax=emax_cm)


def asym_top_case(n_target: int, nstep: int, energies_cm=(150.0,), seed: int = 20261203):
    """(Coupling, Segment, [(ERED, Y0)], system) of the N ~ n_target block:
    MDPROP from 2.8 to 30 Angstrom in nstep steps, Y0 the diagonal WKB start."""
    from oracle import oracle as O
    emax, jtot, block, nmax = ASYM_BLOCKS[n_target]
    sysm = asym_top_system(emax, seed)
    oc = sysm.coupling(jtot, block, nmax=nmax)
    c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent)
    r0, r1 = ASYM_R
    dr = (r1 - r0) / nstep
    rtab = radial_grid(r0, dr, nstep)
    seg = Segment(nstep, dr, rtab, O.ptable(sysm, rtab))
    jobs = []
    for e in energies_cm:
        ered = e * sysm.cm2ru
        jobs.append((ered, S.wkb_initial_y(c, seg.ptab[0], seg.rtab[0], ered)))
    return c, seg, jobs, sysm


def smatrix(c, y, r: float, ered: float):
    """S = (SR, SI) from Y at the last radius by the oracle's YTOK/KTOS, in
    CHNSRT order (open channels first); returns (SR, SI, NOPEN)."""
    from oracle import oracle as O
    wvec, nopen = O.gtwvec(ered, c.eint)
    nb = O.chnsrt(c.eint)
    k = O.ytok(nb, wvec, c.n, nopen, y, r, c.cent)
    sr, si = O.ktos(k)
    return sr, si, nopen
