"""Bound states by node counting (the BOUND search of bd.driver.f over the
BDCTRL matching of bdctrl.f), with the propagations batched on the GPU.

At energy E a system is propagated outward from RMIN to RMATCH and inward
from RMAX to RMATCH (BDPSET's two segments, bdpset.f:26-44).  The number of
bound states below E is

    NODES_out + NODES_in + #{eigenvalues of Y_out(RMATCH) - Y_in(RMATCH) <= 0}

(bdctrl.f:197,221-257): the propagators' negative-pivot counts plus the
matching matrix's non-positive eigenvalues.  A state with node count k lies
where that count steps from k to k+1; bisection on E (bd.driver.f:993-1054)
brackets it, every state's trial energy going into one batched plan per
round, so one GPU launch set serves all states.  The matching step is an N x
N symmetric eigenvalue count on the host (the propagation is the cost).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable

import numpy as np

from ._lib import MGPU_ERR_UNSUPPORTED
from .propagators import Coupling, Plan, PropagatorError, Segment


def w_matrix(c: Coupling, r: float, p: np.ndarray, ered: float) -> np.ndarray:
    """W(R) of HAMMAT/SUMLAM (hammat.f:85-113, sumlam.f:74-86) on the host,
    for the initial log-derivative matrices."""
    n = c.n
    npair = n * (n + 1) // 2
    col = np.repeat(np.arange(n), np.arange(1, n + 1))
    row = np.arange(npair) - col * (col + 1) // 2
    blk = c.vl[:npair * c.nvlblk].reshape(npair, c.nvlblk)[:, :c.nham]
    if c.ivlfl > 0:
        idx = c.iv[:npair * c.nvlblk].reshape(npair, c.nvlblk)[:, :c.nham] - 1
        vals = np.sum(blk * p[idx], axis=1)
    else:
        vals = blk @ p[:c.nham]
    w = np.zeros((n, n))
    w[row, col] = vals
    w[col, row] = vals
    d = np.zeros(n)
    if c.nrsq == 0:
        d += min(1.0 / (r * r), 1.0e16) * c.cent
    if c.nconst == 0:
        d += c.eint
    if c.conlen > 0.0:
        d += r * r / c.conlen ** 4
    return w + np.diag(d - ered)


def adiabatic_wkb_y(c: Coupling, r: float, p: np.ndarray, ered: float, outward: bool,
                    open_value: float = 0.0) -> np.ndarray:
    """YINIT in the local eigenbasis of W(R) (yinit.f:96-117 with ADIAMN):
    +-sqrt(lambda) for locally closed channels (+ outward, - inward), the
    given value for locally open ones."""
    lam, vec = np.linalg.eigh(w_matrix(c, r, p, ered))
    sgn = 1.0 if outward else -1.0
    yl = np.where(lam > 0.0, sgn * np.sqrt(np.abs(lam)), open_value)
    return (vec * yl) @ vec.T


@dataclass
class BoundProblem:
    """One (JTOT, block) system with its two propagation segments.

    `inward(ered) -> (Y_in at RMATCH, NODES_in)`, when given, propagates the
    long-range segment on the host instead of seg_in (BDPSET's IPROPL for a
    propagator other than the log-derivative ones, e.g. AIRY); the GPU plan
    then runs the outward segment alone."""
    coupling: Coupling
    seg_out: Segment  # RMIN -> RMATCH
    seg_in: Segment | None = None   # RMAX -> RMATCH (DR < 0)
    prop: str = "LDMD"
    y_out0: Callable[[float], np.ndarray] | None = None
    y_in0: Callable[[float], np.ndarray] | None = None
    inward: Callable[[float], tuple] | None = None

    def __post_init__(self):
        c, so, si = self.coupling, self.seg_out, self.seg_in
        if si is None and self.inward is None:
            raise ValueError("BoundProblem needs seg_in or an inward propagator")
        if self.y_out0 is None:
            self.y_out0 = lambda e: adiabatic_wkb_y(c, float(so.rtab[0]), so.ptab[0], e, True)
        if self.y_in0 is None and si is not None:
            self.y_in0 = lambda e: adiabatic_wkb_y(c, float(si.rtab[0]), si.ptab[0], e, False)


def node_counts(bp: BoundProblem, ereds, eig: bool = True) -> tuple:
    """(counts, NODES_out, NODES_in, matching counts, smallest matching
    eigenvalue) at every ERED, the propagations of all energies in one plan.
    eig=False counts the matching matrices' negative eigenvalues on the
    device (LDL^T inertia) and returns NaN for the smallest eigenvalues."""
    ereds = np.asarray(ereds, dtype=np.float64)
    m = ereds.size
    host_in = bp.inward is not None
    if host_in:
        job_sys = np.zeros(m, dtype=np.int32)
        job_e = ereds.copy()
        plan = Plan(bp.prop, [bp.coupling], [bp.seg_out], job_sys, job_e)
    else:
        job_sys = np.concatenate([np.zeros(m, dtype=np.int32), np.ones(m, dtype=np.int32)])
        job_e = np.concatenate([ereds, ereds])
        plan = Plan(bp.prop, [bp.coupling, bp.coupling], [bp.seg_out, bp.seg_in], job_sys, job_e)
    try:
        y0 = [bp.y_out0(float(e)) for e in ereds]
        if not host_in:
            y0 += [bp.y_in0(float(e)) for e in ereds]
        ybuf, nodes, status, kfail = plan.run_host(plan.pack(y0))
        if (status != 0).any():
            j = int(np.nonzero(status)[0][0])
            raise RuntimeError(f"propagation failed at ERED={job_e[j]} (status {int(status[j])}, step {int(kfail[j])})")
        if host_in:
            inner = [bp.inward(float(e)) for e in ereds]
            y_in = [np.asarray(y) for y, _ in inner]
            n_in = np.array([int(k) for _, k in inner], dtype=np.int64)
        else:
            y_in = [plan.unpack(ybuf, m + k) for k in range(m)]
            n_in = nodes[m:].astype(np.int64)
        nmatch, eigmin = matching_counts(plan, ybuf, y_in, m, eig, host_in)
        n_out = nodes[:m].astype(np.int64)
        return n_out + n_in + nmatch, n_out, n_in, nmatch, eigmin
    finally:
        plan.close()


def matching_counts(plan, ybuf, y_in, m: int, eig: bool, host_in: bool):
    """Non-positive eigenvalue counts of Y_out - Y_in (job k against job
    m + k, or the host's Y_in) and the smallest-magnitude eigenvalues (NaN
    when eig is False: the counts then come from the device)."""
    nmatch = np.zeros(m, dtype=np.int64)
    eigmin = np.full(m, np.nan)
    dev = None
    if not eig and not host_in and m > 0:
        try:
            dev = plan.match_counts(np.stack([np.arange(m), np.arange(m, 2 * m)], axis=1))
        except PropagatorError as err:  # N above the kernel's limit: count on the host
            if err.status != MGPU_ERR_UNSUPPORTED:
                raise
    for k in range(m):
        if dev is not None and dev[k] >= 0:
            nmatch[k] = int(dev[k])
            continue
        ev = np.linalg.eigvalsh(plan.unpack(ybuf, k) - y_in[k])
        nmatch[k] = int(np.sum(ev <= 0.0))
        eigmin[k] = ev[np.argmin(np.abs(ev))]
    return nmatch, eigmin


def bisect_steps(count: Callable, lo: float, hi: float, c_lo: int, c_hi: int, tol: float,
                 max_rounds: int = 200) -> list:
    """Every step of a monotone count between lo and hi, bisected until its
    bracket is narrower than tol; every live bracket's midpoint goes into one
    call of count(xs) -> counts per round.  Returns [(k, x, lo, hi)] for the
    step between counts k and k + 1, at the bracket midpoint.  An increasing
    count (c_hi > c_lo) is BOUND's in energy; a decreasing one is FIELD's
    case of levels rising with the field (fld.driver.f:864-881)."""
    inc = c_hi >= c_lo
    brackets = {k: [lo, hi] for k in range(min(c_lo, c_hi), max(c_lo, c_hi))}
    for _ in range(max_rounds):
        live = [k for k, (a, b) in brackets.items() if b - a > tol]
        if not live:
            break
        mids = np.array([0.5 * (brackets[k][0] + brackets[k][1]) for k in live])
        counts = count(mids)
        for x, cnt in zip(mids, counts):
            # tighten every bracket this point informs
            for kk, br in brackets.items():
                if br[0] < x < br[1]:
                    below = (cnt <= kk) if inc else (cnt > kk)  # the step lies above x
                    if below:
                        br[0] = x
                    else:
                        br[1] = x
    return [(k, 0.5 * (a + b), a, b) for k, (a, b) in sorted(brackets.items())]


def _zeroin(a: float, b: float, fa: float, fb: float, tol: float):
    """Brent's zero finder (R. P. Brent, Algorithms for Minimization without
    Derivatives, 1973, ch. 4) as a generator: yields the next abscissa,
    receives f there, returns the root once the bracket is narrower than
    about tol.  f(a) and f(b) must have opposite signs."""
    eps = 2.220446049250313e-16
    c, fc = a, fa
    d = e = b - a
    while True:
        if fb * fc > 0.0:
            c, fc = a, fa
            d = e = b - a
        if abs(fc) < abs(fb):
            a, b, c = b, c, b
            fa, fb, fc = fb, fc, fb
        tol1 = 2.0 * eps * abs(b) + 0.5 * tol
        xm = 0.5 * (c - b)
        if abs(xm) <= tol1 or fb == 0.0:
            return b
        if abs(e) >= tol1 and abs(fa) > abs(fb):
            s = fb / fa
            if a == c:  # secant
                p = 2.0 * xm * s
                q = 1.0 - s
            else:  # inverse quadratic interpolation
                q = fa / fc
                r = fb / fc
                p = s * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0))
                q = (q - 1.0) * (r - 1.0) * (s - 1.0)
            if p > 0.0:
                q = -q
            p = abs(p)
            if 2.0 * p < min(3.0 * xm * q - abs(tol1 * q), abs(e * q)):
                e, d = d, p / q
            else:
                d = e = xm
        else:
            d = e = xm
        a, fa = b, fb
        b = b + d if abs(d) > tol1 else b + math.copysign(tol1, xm)
        fb = yield b


def converge_steps(evaluate: Callable, lo: float, hi: float, tol: float, coarse: float,
                   max_rounds: int = 200):
    """BOUND's search with its converging step (bd.driver.f:993-1215):
    every step of a monotone count between lo and hi is bracketed by
    bisection until only its own step lies inside, at most `coarse` wide,
    and the matching eigenvalue of smallest magnitude has opposite signs at
    the two ends; then that eigenvalue's zero is found by Brent's method to
    `tol` (the reference's VWDB step, bd.driver.f:1139-1215).  Every live
    bracket's next trial point goes into one call of evaluate(xs) ->
    (counts, smallest matching eigenvalues) per round.

    Returns ([(k, x, lo, hi)], rounds): the step between counts k and k+1 at
    x, within its final bracket, and the number of evaluate calls."""
    c, g = evaluate(np.array([lo, hi]))
    c_lo, c_hi = int(c[0]), int(c[1])
    inc = c_hi >= c_lo
    rounds = 1
    br = {k: dict(lo=lo, hi=hi, clo=c_lo, chi=c_hi, glo=float(g[0]), ghi=float(g[1]))
          for k in range(min(c_lo, c_hi), max(c_lo, c_hi))}
    # count at the low end of step k's bracket is k (increasing) or k+1
    want_lo = (lambda k: k) if inc else (lambda k: k + 1)
    want_hi = (lambda k: k + 1) if inc else (lambda k: k)
    done = {}
    gens = {}
    pending = {}

    def ready(k, b):
        if b["clo"] != want_lo(k) or b["chi"] != want_hi(k) or b["hi"] - b["lo"] > coarse:
            return False
        return b["glo"] * b["ghi"] < 0.0

    while len(done) < len(br) and rounds < max_rounds:
        xs, who = [], []
        for k, b in br.items():
            if k in done:
                continue
            if k in gens:
                xs.append(pending[k])
                who.append((k, "brent"))
            elif ready(k, b):
                gen = _zeroin(b["lo"], b["hi"], b["glo"], b["ghi"], tol)
                gens[k] = gen
                pending[k] = next(gen)
                xs.append(pending[k])
                who.append((k, "brent"))
            elif b["hi"] - b["lo"] <= tol:
                done[k] = 0.5 * (b["lo"] + b["hi"])
            else:
                xs.append(0.5 * (b["lo"] + b["hi"]))
                who.append((k, "bisect"))
        if not xs:
            break
        cnt, eig = evaluate(np.array(xs))
        rounds += 1
        for (k, how), x, cn, gv in zip(who, xs, cnt, eig):
            cn, gv = int(cn), float(gv)
            # every bisection point tightens the brackets it falls in
            for kk, b in br.items():
                if kk in done or kk in gens or not (b["lo"] < x < b["hi"]):
                    continue
                below = (cn <= kk) if inc else (cn > kk)
                if below:
                    b.update(lo=x, clo=cn, glo=gv)
                else:
                    b.update(hi=x, chi=cn, ghi=gv)
            if how == "brent":
                try:
                    pending[k] = gens[k].send(gv)
                except StopIteration as stop:
                    done[k] = stop.value
                    del gens[k]
    for k in br:
        if k not in done:
            done[k] = pending.get(k, 0.5 * (br[k]["lo"] + br[k]["hi"]))
    return [(k, done[k], br[k]["lo"], br[k]["hi"]) for k in sorted(br)], rounds


def find_states(bp: BoundProblem, emin: float, emax: float, tol: float, max_rounds: int = 200,
                counter: Callable | None = None) -> list:
    """Every state with EMIN < E < EMAX (reduced energies), bisected until its
    bracket is narrower than tol.  Returns [(node count k, energy, lo, hi)]:
    the state where the count steps from k to k+1 (the reference prints it as
    state number k+1), at the bracket midpoint.  `counter(bp, ereds) ->
    counts` defaults to the GPU node count."""
    count = counter or (lambda b, e: node_counts(b, e, eig=False)[0])
    c0, c1 = (int(x) for x in count(bp, [emin, emax]))
    return bisect_steps(lambda xs: count(bp, xs), emin, emax, c0, c1, tol, max_rounds)


def find_states_converged(bp: BoundProblem, emin: float, emax: float, tol: float, coarse: float = math.inf,
                          max_rounds: int = 200, evaluate: Callable | None = None):
    """Every state with EMIN < E < EMAX (reduced energies) by bisection to a
    bracket at most `coarse` wide holding that state alone, then Brent's
    method on the smallest matching eigenvalue to `tol` (converge_steps).
    Returns ([(node count k, energy, lo, hi)], propagation rounds).
    `evaluate(bp, ereds) -> (counts, smallest matching eigenvalues)` defaults
    to the GPU (node_counts)."""
    ev = evaluate or (lambda b, e: (lambda r: (r[0], r[4]))(node_counts(b, e)))
    return converge_steps(lambda xs: ev(bp, xs), emin, emax, tol, coarse, max_rounds)
