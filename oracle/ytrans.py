"""CPU restatement of YTRANS (source_code/ytrans.f90) and CALCA
(source_code/calca.f) — test infrastructure: the checker for the device's
asymptotic-basis transform and the scattering lengths computed from its S
matrices.  Pinned by the thresholds and scattering lengths of
examples/output/molscat-basic_Rb2.output (tests/test_ytrans.py).

What is restated (the one-operator case every shipped basis with NCONST > 0
or NRSQ > 0 and no extra operators reaches):

* the asymptotic operator (ytrans.f90:111-139): W = sum_l VL_l P_l with P
  zero for the MXLAM potential terms and VCONST for the NCONST constant
  terms, or, for NRSQ > 0 alone, the NRSQ 1/R^2 terms with P = 1;
* blocking (ytrans.f90:146-176): by L for MOLSCAT (NRSQ = 0, IBOUND = 0), by
  the CENT values within DEGTOL for BOUND/FIELD (IBOUND != 0), one block for
  NRSQ > 0;
* per block, the eigenvalues in ascending order and their eigenvectors
  (MULTOP with one operator is one DIAGVC = DSYEVR call, multop.f90:70-75),
  each eigenvector's largest element made positive (the first of equal
  magnitudes, IDAMAX; ytrans.f90:281-294);
* EINT(i) = the eigenvalue of channel i's place in its block, EVEC the
  eigenvectors in those columns (ytrans.f90:365-386); with NRSQ > 0, CENT
  = the eigenvalues of the L^2 operator (ytrans.f90:436-458);
* the transform Y' = EVEC^T Y EVEC (TRNSFM, ytrans.f90:410-413);
* CALCA (calca.f:33-57): A = (1 - S_ii) / (1 + S_ii) / (i k^m),
  m = min(LRPOW - 2, 2L + 1), |S_ii| > 1 renormalised, S_ii <= -1 giving
  1e30.
"""
from __future__ import annotations

import numpy as np


def pair_index(n: int):
    """(row, col) of every pair of the packed upper triangle, column after column."""
    col = np.repeat(np.arange(n), np.arange(1, n + 1))
    row = np.arange(n * (n + 1) // 2) - col * (col + 1) // 2
    return row, col


def operator(vl: np.ndarray, nham: int, n: int, p: np.ndarray) -> np.ndarray:
    """sum_l VL_l P_l as a full symmetric n x n matrix (SUMLAM's sum)."""
    v = np.asarray(vl, dtype=np.float64).reshape(-1, nham)[: n * (n + 1) // 2]
    w = v @ np.asarray(p, dtype=np.float64)
    row, col = pair_index(n)
    m = np.zeros((n, n))
    m[row, col] = w
    m[col, row] = w
    return m


def _blocks(n: int, lval, cent, nrsq: int, ibound: int, degtol: float) -> list:
    if nrsq > 0:
        return [list(range(n))]
    if ibound == 0:
        ls = np.asarray(lval)
        return [list(np.nonzero(ls == ll)[0]) for ll in range(int(ls.min()), int(ls.max()) + 1)
                if np.any(ls == ll)]
    cent = np.asarray(cent, dtype=np.float64)
    mask = np.zeros(n, dtype=int)
    out = []
    cur = cent.min()
    k = 0
    while True:
        k += 1
        members = [i for i in range(n) if mask[i] == 0 and abs(cent[i] - cur) <= degtol]
        for i in members:
            mask[i] = k
        out.append(members)
        rest = cent[mask == 0]
        if rest.size == 0:
            break
        cur = rest.min()
    return out


def ytrans(w: np.ndarray, lval, cent, nrsq: int = 0, ibound: int = 0, degtol: float = 1.0e-10):
    """EVEC (n x n), EINT (n) and CENT (n) from the asymptotic operator w."""
    n = w.shape[0]
    evec = np.zeros((n, n))
    eint = np.zeros(n)
    for idx in _blocks(n, lval, cent, nrsq, ibound, degtol):
        sub = w[np.ix_(idx, idx)]
        ev, vec = np.linalg.eigh(sub)
        for c in range(len(idx)):
            imax = int(np.argmax(np.abs(vec[:, c])))
            if vec[imax, c] < 0.0:
                vec[:, c] = -vec[:, c]
        evec[np.ix_(idx, idx)] = vec
        eint[idx] = ev
    cent_out = eint.copy() if nrsq > 0 else np.asarray(cent, dtype=np.float64).copy()
    return evec, eint, cent_out


def transform(y: np.ndarray, evec: np.ndarray) -> np.ndarray:
    return evec.T @ y @ evec


def calca(sr: np.ndarray, si: np.ndarray, nb, lval, wvec, lrpow: int = 6) -> list:
    """Scattering lengths (volumes, ...) of the open channels, in order."""
    out = []
    for i in range(sr.shape[0]):
        ch = nb[i]
        dd = wvec[ch]
        ll = int(lval[ch])
        s_re, s_im = sr[i, i], si[i, i]
        mag = np.hypot(s_re, s_im)
        if mag > 1.0:
            s_re, s_im = s_re / mag, s_im / mag
        m = min(lrpow - 2, 2 * ll + 1)
        if s_re <= -1.0:
            a = complex(1.0e30, 0.0)
        else:
            a = complex(1.0 - s_re, -s_im) / (complex(1.0 + s_re, s_im) * complex(0.0, dd ** m))
        out.append((ll, m, dd, a))
    return out
