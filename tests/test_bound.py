"""Bound states by node counting against the reference's printed
bound-basic1 energies (examples/output/bound-basic1.output: JTOT=1, block 2,
states 4 and 5), with the propagations on the CPU oracle (pins the restated
BOUND logic: segments, YINIT, node count, matching) and on the GPU (equal
node counts at every energy, energies within 1e-9 relative of the oracle's)."""
import json
import os

import numpy as np
import pytest

import cases
from molscat_b200.bound import BoundProblem, adiabatic_wkb_y, find_states, find_states_converged
from molscat_b200.propagators import Coupling, Segment, radial_grid

HERE = os.path.dirname(os.path.abspath(__file__))
TOL_CM = 1.0e-9          # bisection width
REF_TOL_CM = 2.0e-7      # the reference converged its steps to 1e-7 cm-1


@pytest.fixture(scope="module")
def basic1():
    from oracle import oracle as O
    with open(os.path.join(HERE, "golden", "bound_basic1.json")) as f:
        g = json.load(f)
    s = g["system"]
    sysm = O.Itype1(ured=s["ured"], be=s["be"], jlevel=s["jlevel"], lam=s["lambda"],
                    terms=[[tuple(t) for t in tl] for tl in s["terms"]], rm=s["rm"], epsil=s["epsil"])
    oc = sysm.coupling(s["jtot"], s["block"])
    c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent)
    n_out = int(round((s["rmatch"] - s["rmin"]) / s["dr"]))
    n_in = int(round((s["rmax"] - s["rmatch"]) / s["dr"]))
    r_out = radial_grid(s["rmin"], (s["rmatch"] - s["rmin"]) / n_out, n_out)
    r_in = radial_grid(s["rmax"], -(s["rmax"] - s["rmatch"]) / n_in, n_in)
    seg_out = Segment(n_out, (s["rmatch"] - s["rmin"]) / n_out, r_out, O.ptable(sysm, r_out))
    seg_in = Segment(n_in, -(s["rmax"] - s["rmatch"]) / n_in, r_in, O.ptable(sysm, r_in))
    return g, sysm, BoundProblem(c, seg_out, seg_in, "LDMD")


def oracle_counts(bp, ereds):
    from oracle import oracle as O
    oc = cases.to_oracle(bp.coupling)
    out = []
    for e in ereds:
        yo, no, st, _ = O.mdprop(oc, bp.seg_out.rtab, bp.seg_out.ptab, bp.seg_out.nstep, bp.seg_out.dr, e,
                                 bp.y_out0(float(e)))
        yi, ni, st2, _ = O.mdprop(oc, bp.seg_in.rtab, bp.seg_in.ptab, bp.seg_in.nstep, bp.seg_in.dr, e,
                                  bp.y_in0(float(e)))
        assert st == 0 and st2 == 0
        out.append(no + ni + int(np.sum(np.linalg.eigvalsh(yo - yi) <= 0.0)))
    return np.array(out)


def oracle_eval(bp, ereds):
    """(counts, smallest-magnitude matching eigenvalue) with the oracle."""
    from oracle import oracle as O
    oc = cases.to_oracle(bp.coupling)
    cnt, eig = [], []
    for e in ereds:
        yo, no, st, _ = O.mdprop(oc, bp.seg_out.rtab, bp.seg_out.ptab, bp.seg_out.nstep, bp.seg_out.dr, e,
                                 bp.y_out0(float(e)))
        yi, ni, st2, _ = O.mdprop(oc, bp.seg_in.rtab, bp.seg_in.ptab, bp.seg_in.nstep, bp.seg_in.dr, e,
                                  bp.y_in0(float(e)))
        assert st == 0 and st2 == 0
        ev = np.linalg.eigvalsh(yo - yi)
        cnt.append(no + ni + int(np.sum(ev <= 0.0)))
        eig.append(float(ev[np.argmin(np.abs(ev))]))
    return np.array(cnt), np.array(eig)


def _states(bp, sysm, g, counter=None):
    """(the reference's 1-based state number, energy in cm-1): the state where
    the count steps from k to k+1 is state k+1."""
    s = g["system"]
    res = find_states(bp, s["emin_cm"] * sysm.cm2ru, s["emax_cm"] * sysm.cm2ru, TOL_CM * sysm.cm2ru,
                      counter=counter)
    return [(k + 1, e / sysm.cm2ru) for k, e, _, _ in res]


def test_oracle_reproduces_reference_bound_states(basic1):
    g, sysm, bp = basic1
    got = _states(bp, sysm, g, counter=oracle_counts)
    want = [(st["state"], st["energy_cm"]) for st in g["states"]]
    assert [k for k, _ in got] == [k for k, _ in want]
    for (_, e), (_, w) in zip(got, want):
        assert abs(e - w) < REF_TOL_CM, (e, w)


@pytest.mark.gpu
def test_gpu_bound_states_equal_oracle(basic1):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.bound import node_counts
    g, sysm, bp = basic1
    got = _states(bp, sysm, g)
    want = [(st["state"], st["energy_cm"]) for st in g["states"]]
    assert [k for k, _ in got] == [k for k, _ in want]
    for (_, e), (_, w) in zip(got, want):
        assert abs(e - w) < REF_TOL_CM, (e, w)
    # node counts identical to the oracle's, also right beside each state
    probe = [-9.0, -6.0, -3.0] + [e + d for _, e in got for d in (-1e-6, 1e-6)]
    ered = np.array(probe) * sysm.cm2ru
    assert np.array_equal(node_counts(bp, ered)[0], oracle_counts(bp, ered))
    ora = _states(bp, sysm, g, counter=oracle_counts)
    for (_, e), (_, o) in zip(got, ora):
        assert abs(e - o) <= 1e-9 * abs(o) + 2 * TOL_CM


def test_bisection_brackets_every_state_with_a_counting_stub():
    """The search logic alone (bd.driver.f:993-1054): a stub count with known
    levels stands in for the propagations; every state between EMIN and EMAX
    is found once, numbered by the count below it, within tol."""
    levels = np.array([-7.25, -3.5, -3.4999, -1.0, 0.75])
    calls = []

    def stub(bp, ereds):
        e = np.asarray(ereds, dtype=np.float64)
        calls.append(e.size)
        return np.searchsorted(levels, e, side="left")  # states strictly below E

    tol = 1.0e-9
    found = find_states(None, -5.0, 1.0, tol, counter=stub)
    inside = levels[(levels > -5.0) & (levels < 1.0)]
    assert [k for k, *_ in found] == [1, 2, 3, 4]
    for (k, e, lo, hi), lev in zip(found, inside):
        assert hi - lo <= tol and lo <= lev <= hi
        assert abs(e - lev) <= tol
    # every round puts all unresolved states' trial energies into one batch
    assert calls[0] == 2 and max(calls[1:]) <= len(inside)


def _converged(bp, sysm, g, evaluate=None):
    s = g["system"]
    res, rounds = find_states_converged(bp, s["emin_cm"] * sysm.cm2ru, s["emax_cm"] * sysm.cm2ru,
                                        TOL_CM * sysm.cm2ru, evaluate=evaluate)
    return [(k + 1, e / sysm.cm2ru) for k, e, _, _ in res], rounds


def test_converged_search_with_oracle_matches_reference(basic1):
    """Bisection until each state sits alone in its bracket with the matching
    eigenvalue changing sign, then Brent on that eigenvalue (the VWDB step of
    bd.driver.f:1139-1215): the reference's energies in far fewer
    propagation rounds than bisecting to the same width."""
    g, sysm, bp = basic1
    got, rounds = _converged(bp, sysm, g, evaluate=oracle_eval)
    want = [(st["state"], st["energy_cm"]) for st in g["states"]]
    assert [k for k, _ in got] == [k for k, _ in want]
    for (_, e), (_, w) in zip(got, want):
        assert abs(e - w) < REF_TOL_CM, (e, w)
    calls = []
    _states(bp, sysm, g, counter=lambda b, e: (calls.append(1), oracle_counts(b, e))[1])
    assert rounds < len(calls) / 2, (rounds, len(calls))


def test_converged_search_with_a_stub():
    """The search logic alone: counts and a matching eigenvalue with known
    zeros stand in for the propagations."""
    levels = np.array([-7.25, -3.5, -3.4999, -1.0, 0.75])
    rounds_seen = []

    def stub(bp, ereds):
        e = np.asarray(ereds, dtype=np.float64)
        cnt = np.searchsorted(levels, e, side="left")
        near = levels[np.argmin(np.abs(e[:, None] - levels[None, :]), axis=1)]
        rounds_seen.append(e.size)
        return cnt, -(e - near) * (1.0 + 0.3 * (e - near))  # positive below a level, negative above

    found, rounds = find_states_converged(None, -5.0, 1.0, 1e-12, evaluate=stub)
    inside = levels[(levels > -5.0) & (levels < 1.0)]
    assert [k for k, *_ in found] == [1, 2, 3, 4]
    for (k, e, lo, hi), lev in zip(found, inside):
        assert abs(e - lev) <= 1e-11
    assert rounds == len(rounds_seen) and rounds < 60


@pytest.mark.gpu
def test_gpu_converged_search_equals_oracle(basic1):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    g, sysm, bp = basic1
    got, rounds = _converged(bp, sysm, g)
    ora, _ = _converged(bp, sysm, g, evaluate=oracle_eval)
    assert [k for k, _ in got] == [k for k, _ in ora]
    for (_, e), (_, o) in zip(got, ora):
        assert abs(e - o) <= 1e-9 * abs(o), (e, o)
