"""YTRANS (source_code/ytrans.f90): the asymptotic basis in which YTOK
matches, for bases whose asymptotic Hamiltonian is not diagonal (NCONST > 0:
the R-independent terms; NRSQ > 0: the 1/R^2 terms).

The host part runs once per (JTOT, block) system — it does not depend on the
energy — and hands its result to a plan (`Plan.set_asymptote`); the
transform Y' = EVEC^T Y EVEC and the matching run on the device with the
rest of Y -> K -> S.

    w = asymptotic_operator(coupling, p_const)       # sum_l VL_l P_l
    basis = asymptotic_basis(coupling, w, lvals)     # EVEC, EINT, CENT
    plan.set_asymptote(s, basis.eint, basis.cent, basis.evec, rmatch)

Covered: one operator to diagonalise — NCONST > 0 (thresholds) or NRSQ > 0
(the L^2 eigenvalues), without the extra operators (NEXTRA) that only
MOLSCAT's degenerate-threshold labelling uses (MULTOP's recursion and
EV_ORD ordering, multop.f90:115-247): `asymptotic_basis` raises for both
NCONST > 0 and NRSQ > 0 and IVLFL > 0, as ytrans.f90:103-106 stops there.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .propagators import Coupling


@dataclass
class AsymptoticBasis:
    evec: np.ndarray   # (n, n): column i is asymptotic channel i in the primitive basis
    eint: np.ndarray   # (n,) thresholds, reduced units (YTRANS's EINT)
    cent: np.ndarray   # (n,) L(L+1) of the asymptotic channels (YTRANS's CENT)
    lval: np.ndarray   # (n,) integer L where L(L+1) is integral, else -1


def asymptotic_operator(c: Coupling, p: np.ndarray) -> np.ndarray:
    """sum_l VL_l P_l over the coupling's NHAM terms as a full symmetric n x n
    matrix.  For the thresholds (ytrans.f90:111-139), P is zero for the MXLAM
    potential terms and VCONST (reduced units) for the NCONST constant ones;
    for the L^2 operator of NRSQ > 0, P is one for the NRSQ 1/R^2 terms."""
    n, nb = c.n, c.nvlblk
    npair = n * (n + 1) // 2
    v = c.vl[: nb * npair].reshape(npair, nb)[:, : c.nham]
    w = v @ np.asarray(p, dtype=np.float64)[: c.nham]
    j = np.repeat(np.arange(n), np.arange(1, n + 1))   # column of each packed pair
    i = np.arange(npair) - j * (j + 1) // 2             # row
    out = np.zeros((n, n))
    out[i, j] = w
    out[j, i] = w
    return out


def _groups(c: Coupling, lvals, bound: bool, degtol: float) -> list:
    """Channel sets diagonalised separately (ytrans.f90:146-176)."""
    n = c.n
    if c.nrsq > 0:
        return [np.arange(n)]
    if not bound:
        lv = np.asarray(lvals, dtype=np.int64)
        return [np.flatnonzero(lv == ell) for ell in range(int(lv.min()), int(lv.max()) + 1) if np.any(lv == ell)]
    # BOUND / FIELD: by CENT value, ascending, within DEGTOL
    left = np.ones(n, dtype=bool)
    out = []
    while left.any():
        ref = c.cent[left].min()
        g = np.flatnonzero(left & (np.abs(c.cent[:n] - ref) <= degtol))
        left[g] = False
        out.append(g)
    return out


def asymptotic_basis(c: Coupling, w: np.ndarray, lvals=None, bound: bool = False,
                     degtol: float = 1.0e-10) -> AsymptoticBasis:
    """Eigenvectors and eigenvalues of the asymptotic operator w, group by
    group (eigenvalues ascending, as DSYEVR gives them); each eigenvector's
    element of largest magnitude (the first of equals) made positive
    (ytrans.f90:281-294).  lvals: the basis functions' L (MOLSCAT, NRSQ = 0);
    bound=True groups by CENT instead (BOUND/FIELD)."""
    if c.ivlfl > 0:
        raise NotImplementedError("YTRANS with IVLFL > 0 (the reference stops there too)")
    if c.nconst > 0 and c.nrsq > 0:
        raise NotImplementedError("YTRANS with both NCONST and NRSQ (two operators, MULTOP's recursion)")
    if c.nconst == 0 and c.nrsq == 0:
        raise ValueError("the basis is asymptotically diagonal (NCONST = NRSQ = 0): YTRANS returns at once")
    n = c.n
    if lvals is None and not bound and c.nrsq == 0:
        lvals = np.rint(np.sqrt(c.cent[:n] + 0.25) - 0.5).astype(np.int64)
    evec = np.zeros((n, n))
    vals = np.zeros(n)
    for g in _groups(c, lvals, bound, degtol):
        ev, vec = np.linalg.eigh(w[np.ix_(g, g)])
        big = np.argmax(np.abs(vec), axis=0)
        sign = np.where(vec[big, np.arange(len(g))] < 0.0, -1.0, 1.0)
        evec[np.ix_(g, g)] = vec * sign[None, :]
        vals[g] = ev
    if c.nrsq > 0:
        # the eigenvalues are those of L^2; EINT stays the coupling's
        cent = vals.copy()
        eint = c.eint[:n].copy()
        if np.any(cent < -1.0e-10):
            raise ValueError("an eigenvalue of the centrifugal operator is not physical")
    else:
        cent = c.cent[:n].copy()
        eint = vals
    lr = np.sqrt(np.maximum(cent, 0.0) + 0.25) - 0.5
    lval = np.where(np.abs(lr - np.rint(lr)) <= 1.0e-10, np.rint(lr), -1).astype(np.int64)
    return AsymptoticBasis(evec=evec, eint=eint, cent=cent, lval=lval)


def scattering_lengths(sr: np.ndarray, si: np.ndarray, eint, cent, ered: float, lrpow: int = 6) -> list:
    """CALCA (calca.f:33-57) for the open channels of one S matrix in CHNSRT
    order: A = (1 - S_ii) / (1 + S_ii) / (i k^m), m = min(LRPOW - 2, 2L + 1);
    |S_ii| > 1 is renormalised first and S_ii <= -1 gives 1e30.  Returns
    (L, m, k, A) per open channel."""
    eint = np.asarray(eint, dtype=np.float64)
    # CHNSRT's order: by threshold, equal thresholds (within 1e-11) in index order
    nb = list(range(len(eint)))
    for a in range(len(nb) - 1):
        for b in range(a + 1, len(nb)):
            if eint[nb[a]] > eint[nb[b]] and abs(eint[nb[a]] - eint[nb[b]]) >= 1.0e-11:
                nb[a], nb[b] = nb[b], nb[a]
    out = []
    for i in range(sr.shape[0]):
        ch = nb[i]
        k = float(np.sqrt(ered - eint[ch]))
        ell = int(round(float(np.sqrt(cent[ch] + 0.25) - 0.5)))
        s_re, s_im = float(sr[i, i]), float(si[i, i])
        mag = np.hypot(s_re, s_im)
        if mag > 1.0:
            s_re, s_im = s_re / mag, s_im / mag
        m = min(lrpow - 2, 2 * ell + 1)
        if s_re <= -1.0:
            a = complex(1.0e30, 0.0)
        else:
            a = complex(1.0 - s_re, -s_im) / (complex(1.0 + s_re, s_im) * complex(0.0, k ** m))
        out.append((ell, m, k, a))
    return out
