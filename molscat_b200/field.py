"""Fields at which bound states cross a fixed energy (FIELD's search,
fld.driver.f), with the propagations batched on the GPU.

At a fixed energy E the number of bound states below E changes with an
external field F as the levels move with it.  FIELD counts states at FLDMIN
and FLDMAX, assumes the count changes monotonically in between and seeks
|NODES(FLDMAX) - NODES(FLDMIN)| states (fld.driver.f:855-881), each by
bisection on the field (fld.driver.f:889-1060).  The count at one field is
BOUND's: NODES_out + NODES_in + the non-positive eigenvalues of
Y_out - Y_in at RMATCH (bdctrl.f:197,221-257).

A trial field is its own coupled-channel system: the caller's
coupling_at(F) returns the channel thresholds (and couplings) at F, which
FIELD obtains through SETEFV / CHEINT (fld.driver.f:926-935).  Every trial
field of a bisection round goes into one batched plan (outward and inward
segments of all fields together), so one GPU launch set serves all states.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable

import numpy as np

from .bound import adiabatic_wkb_y, bisect_steps, converge_steps, matching_counts
from .propagators import Coupling, Plan, Segment


@dataclass
class FieldProblem:
    """One (JTOT, block) at one energy, with its field-dependent coupling.

    Where more than the coupling moves with the field, `segments_at(F) ->
    (seg_out, seg_in)` gives the segments (their P tables hold any
    field-dependent constant terms, e.g. a Zeeman prefactor) and
    `ered_at(F)` the energy (an energy fixed relative to a field-dependent
    threshold, the MONQN reference of fld.driver.f).  `inward(F, coupling,
    ered) -> (Y_in at RMATCH, NODES_in)` propagates the long-range segment
    on the host instead (e.g. AIRY); the plan then runs the outward segments
    alone.  y_out0 / y_in0 default to the adiabatic WKB start."""
    coupling_at: Callable[[float], Coupling]
    seg_out: Segment | None = None  # RMIN -> RMATCH
    seg_in: Segment | None = None   # RMAX -> RMATCH (DR < 0)
    ered: float = 0.0
    prop: str = "LDMD"
    y_out0: Callable[[Coupling], np.ndarray] | None = None
    y_in0: Callable[[Coupling], np.ndarray] | None = None
    segments_at: Callable[[float], tuple] | None = None
    ered_at: Callable[[float], float] | None = None
    inward: Callable[[float, Coupling, float], tuple] | None = None

    def __post_init__(self):
        if self.segments_at is None and self.seg_out is None:
            raise ValueError("FieldProblem needs seg_out or segments_at")
        if self.inward is None and self.segments_at is None and self.seg_in is None:
            raise ValueError("FieldProblem needs seg_in, segments_at or an inward propagator")
        if self.segments_at is None and self.ered_at is None:
            so, si, e = self.seg_out, self.seg_in, self.ered
            if self.y_out0 is None:
                self.y_out0 = lambda c: adiabatic_wkb_y(c, float(so.rtab[0]), so.ptab[0], e, True)
            if self.y_in0 is None and si is not None:
                self.y_in0 = lambda c: adiabatic_wkb_y(c, float(si.rtab[0]), si.ptab[0], e, False)

    def at(self, f: float):
        """(coupling, seg_out, seg_in, ERED) at field f."""
        c = self.coupling_at(f)
        so, si = self.segments_at(f) if self.segments_at is not None else (self.seg_out, self.seg_in)
        e = self.ered_at(f) if self.ered_at is not None else self.ered
        return c, so, si, e

    def start_out(self, c, so, e):
        if self.y_out0 is not None:
            return self.y_out0(c)
        return adiabatic_wkb_y(c, float(so.rtab[0]), so.ptab[0], e, True)

    def start_in(self, c, si, e):
        if self.y_in0 is not None:
            return self.y_in0(c)
        return adiabatic_wkb_y(c, float(si.rtab[0]), si.ptab[0], e, False)


def field_node_counts(fp: FieldProblem, fields, eig: bool = True) -> tuple:
    """(counts, NODES_out, NODES_in, matching counts, smallest-magnitude
    matching eigenvalues) at every field, all fields' propagations in one
    plan.  eig=False counts the matching matrices' negative eigenvalues on
    the device (LDL^T inertia; the eigenvalues only where a pivot is zero)
    and returns NaN for the smallest eigenvalues."""
    fields = np.asarray(fields, dtype=np.float64)
    m = fields.size
    sys_at = [fp.at(float(f)) for f in fields]
    cs = [a[0] for a in sys_at]
    outs = [a[1] for a in sys_at]
    ins = [a[2] for a in sys_at]
    es = np.array([a[3] for a in sys_at], dtype=np.float64)
    host_in = fp.inward is not None
    if host_in:
        plan = Plan(fp.prop, cs, outs, np.arange(m, dtype=np.int32), es)
    else:
        plan = Plan(fp.prop, cs + cs, outs + ins, np.arange(2 * m, dtype=np.int32), np.concatenate([es, es]))
    try:
        y0 = [fp.start_out(c, so, e) for c, so, e in zip(cs, outs, es)]
        if not host_in:
            y0 += [fp.start_in(c, si, e) for c, si, e in zip(cs, ins, es)]
        ybuf, nodes, status, kfail = plan.run_host(plan.pack(y0))
        if (status != 0).any():
            j = int(np.nonzero(status)[0][0])
            raise RuntimeError(f"propagation failed at F={fields[j % m]} (status {int(status[j])}, "
                               f"step {int(kfail[j])})")
        if host_in:
            inner = [fp.inward(float(f), c, float(e)) for f, c, e in zip(fields, cs, es)]
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


def find_fields(fp: FieldProblem, fmin: float, fmax: float, tol: float, max_rounds: int = 200,
                counter: Callable | None = None) -> list:
    """Every field in (FMIN, FMAX) where a state crosses the energy, bisected
    until its bracket is narrower than tol.  Returns [(k, field, lo, hi)]:
    the crossing where the count of states below the energy steps between k
    and k + 1 (up or down with the field, whichever the end counts say).
    `counter(fp, fields) -> counts` defaults to the GPU node count."""
    count = counter or (lambda p, f: field_node_counts(p, f, eig=False)[0])
    c0, c1 = (int(x) for x in count(fp, [fmin, fmax]))
    return bisect_steps(lambda xs: count(fp, xs), fmin, fmax, c0, c1, tol, max_rounds)


def find_fields_converged(fp: FieldProblem, fmin: float, fmax: float, tol: float, coarse: float = math.inf,
                          max_rounds: int = 200, evaluate: Callable | None = None):
    """FIELD's search with its converging step (fld.driver.f:1102-1217):
    bisection on the field until each crossing sits alone in its bracket with
    the matching eigenvalue changing sign, then Brent's method on that
    eigenvalue to `tol` (bound.converge_steps).  Returns ([(k, field, lo,
    hi)], propagation rounds).  `evaluate(fp, fields) -> (counts, smallest
    matching eigenvalues)` defaults to the GPU."""
    ev = evaluate or (lambda p, f: (lambda r: (r[0], r[4]))(field_node_counts(p, f)))
    return converge_steps(lambda xs: ev(fp, xs), fmin, fmax, tol, coarse, max_rounds)
