"""Atom + asymmetric top (MOLSCAT ITYPE=6) on the propagator.

Pinned to the reference's bound-Ar_CH4 example (examples/input/
bound-Ar_CH4.input, examples/output/bound-Ar_CH4.output; fixture made by
tests/golden/make_golden.py): CH4 as a spherical top with centrifugal
distortion, the Buck MSV potential through its VSTAR plug-in, JTOT = 1,
block 2 (N = 26), MDPROP outward from RMIN (FINDRM, IRMSET = 8) to RMATCH and
inward from RMAX, DR = 0.01, four bound states in -100..-60 cm-1.

* CPU: the oracle's basis (oracle/itype6.py) reproduces the printed pair
  energies (1e-7 cm-1, the print's precision), symmetry codes and channel
  list, and its node-count search the printed energies (2e-7 cm-1: the
  reference converged its steps to 1e-7 cm-1).
* GPU: node counts equal the oracle's at every probed energy; the GPU's
  search gives the oracle search's energies exactly (both bisect the same
  midpoints) and so the reference's.
* GPU, large N on the physical basis (tests/cases.py asym_top_case: A 9.6,
  B 4.3, C 2.8 cm-1, six V(lambda, mu) terms): N = 256 over the full 3000
  steps, N = 500 and 1024 over 1000 steps, against the oracle's results in
  tests/golden/asym_top_large_n.json (made by make_asym_top_golden.py):
  NODES exact, Y(RSTOP) within 5e-8 relative to max|Y| (diagonal, first
  column, Frobenius norm), S within 1e-8 absolute (first four columns), and
  the GPU's S unitary within 1e-8.
* molscat-ityp6 (examples/input/molscat-ityp6.input, examples/output/
  molscat-ityp6.output; fixture by make_golden.py): the same molecule with
  ISYM = 224, LDMD from RMIN (IRMSET = 8) to RMID = 1.3 RTURN and AIRY
  (oracle/aiprop.py) to RMAX, 300 cm-1.  The oracle alone reproduces the
  printed state-to-state partial cross sections (six digits) for JTOT = 0..80,
  N = 2..59; with the GPU propagating the LDMD segment (N = 39..59, above
  the reference's N = 30 switch from SYMINV to DSYTRF/DSYNEG) the same
  printed values come out, with Y(RMID) within 5e-8 of the oracle's and
  NODES equal.
"""
import json
import os

import numpy as np
import pytest

import cases
from molscat_b200.bound import BoundProblem, find_states
from molscat_b200.propagators import Coupling, Segment, radial_grid

HERE = os.path.dirname(os.path.abspath(__file__))
TOL_CM = 1.0e-9
REF_TOL_CM = 2.0e-7
Y_TOL = 5e-8
S_TOL = 1e-8


@pytest.fixture(scope="module")
def arch4():
    from oracle import itype6 as I6
    from oracle import oracle as O
    with open(os.path.join(HERE, "golden", "bound_ar_ch4.json")) as f:
        g = json.load(f)
    s = g["system"]
    pot = I6.BuckMSV(*s["beta"], *s["c6c8"], *s["x1234"], [tuple(a) for a in s["alphas"]],
                     [lm for lm, _ in s["lambda"][1:]])
    sysm = I6.Itype6(ured=s["ured"], roti=tuple(s["roti"]), jmax=s["jmax"], lam=[tuple(x) for x in s["lambda"]],
                     pfunc=pot, rm=s["rm"], epsil=s["epsil"], isym=s["isym"])
    oc = sysm.coupling(s["jtot"], s["block"])
    # FINDRM at the top of the energy window (bd.driver.f:849-857), BOUND branch
    rmin, _ = O.findrm(sysm, oc, s["rmin"], s["emax_cm"] * sysm.cm2ru, irmset=s["irmset"], bound=True)
    # DRSET with DR given: a whole number of steps per segment (drset.f:56-66)
    n_out = max(O.nint((s["rmatch"] - rmin) / s["dr"]), 1)
    n_in = max(O.nint((s["rmax"] - s["rmatch"]) / s["dr"]), 1)
    dr_out, dr_in = (s["rmatch"] - rmin) / n_out, (s["rmax"] - s["rmatch"]) / n_in
    r_out = radial_grid(rmin, dr_out, n_out)
    r_in = radial_grid(s["rmax"], -dr_in, n_in)
    c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent)
    bp = BoundProblem(c, Segment(n_out, dr_out, r_out, O.ptable(sysm, r_out)),
                      Segment(n_in, -dr_in, r_in, O.ptable(sysm, r_in)), "LDMD")
    return g, sysm, bp


def oracle_counts(bp, ereds):
    from oracle import oracle as O
    oc = cases.to_oracle(bp.coupling)
    out = []
    for e in ereds:
        so, si = bp.seg_out, bp.seg_in
        yo, no, st, _ = O.mdprop(oc, so.rtab, so.ptab, so.nstep, so.dr, e, bp.y_out0(float(e)))
        yi, ni, st2, _ = O.mdprop(oc, si.rtab, si.ptab, si.nstep, si.dr, e, bp.y_in0(float(e)))
        assert st == 0 and st2 == 0
        out.append(no + ni + int(np.sum(np.linalg.eigvalsh(yo - yi) <= 0.0)))
    return np.array(out)


def _search(arch4, counter=None):
    g, sysm, bp = arch4
    s = g["system"]
    res = find_states(bp, s["emin_cm"] * sysm.cm2ru, s["emax_cm"] * sysm.cm2ru, TOL_CM * sysm.cm2ru,
                      counter=counter)
    return [(k + 1, e / sysm.cm2ru) for k, e, _, _ in res]


def test_ar_ch4_basis_matches_reference(arch4):
    g, sysm, _ = arch4
    ps = g["pair_states"]
    assert len(sysm.states) == len(ps)
    for st, ref in zip(sysm.states, ps):
        assert st.j == ref["j"] and st.iplev == ref["prty"]
        assert abs(sysm.elevel[st.level] - ref["energy_cm"]) < 1.0e-7
    ch = sysm.channels(g["system"]["jtot"], g["system"]["block"])
    assert [(i + 1, l) for i, l in ch] == [(x["pair_state"], x["l"]) for x in g["channels"]]


def test_ar_ch4_oracle_bound_states_match_reference(arch4):
    g = arch4[0]
    found = _search(arch4, counter=oracle_counts)
    want = [(x["state"], x["energy_cm"]) for x in g["states"]]
    assert [k for k, _ in found] == [k for k, _ in want]
    for (_, e), (_, w) in zip(found, want):
        assert abs(e - w) < REF_TOL_CM, (e, w)


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    return torch


@pytest.mark.gpu
def test_ar_ch4_gpu_bound_states(arch4, gpu):
    from molscat_b200.bound import node_counts
    g, sysm, bp = arch4
    want = [x["energy_cm"] for x in g["states"]]
    probe = np.array([g["system"]["emin_cm"], g["system"]["emax_cm"]] + [w + d for w in want for d in (-1e-6, 1e-6)])
    probe = probe * sysm.cm2ru
    assert np.array_equal(node_counts(bp, probe)[0], oracle_counts(bp, probe))
    got = _search(arch4)
    assert [k for k, _ in got] == [x["state"] for x in g["states"]]
    for (_, e), w in zip(got, want):
        assert abs(e - w) < REF_TOL_CM, (e, w)
    assert got == _search(arch4, counter=oracle_counts)


@pytest.fixture(scope="module")
def large_golden():
    with open(os.path.join(HERE, "golden", "asym_top_large_n.json")) as f:
        return json.load(f)


@pytest.mark.gpu
@pytest.mark.parametrize("n_target", [256, 512, 1024])
def test_asym_top_large_n_against_oracle(large_golden, gpu, n_target):
    from molscat_b200.propagators import propagate
    run = next(r for r in large_golden["runs"] if r["n_target"] == n_target)
    c, seg, jobs, _ = cases.asym_top_case(n_target, run["nstep"], (large_golden["energy_cm"],))
    ered, y0 = jobs[0]
    assert c.n == run["n"] and abs(ered - run["ered"]) <= 1e-12 * abs(ered)
    y, nodes = propagate("LDMD", c, seg, ered, y0)
    assert nodes == run["nodes"]
    scale = max(1.0, float(np.max(np.abs(run["y_diag"]))), float(np.max(np.abs(run["y_col0"]))))
    assert np.abs(np.diag(y) - run["y_diag"]).max() / scale < Y_TOL
    assert np.abs(y[:, 0] - run["y_col0"]).max() / scale < Y_TOL
    assert abs(np.linalg.norm(y) - run["y_fro"]) / run["y_fro"] < Y_TOL
    sr, si, nopen = cases.smatrix(c, y, float(seg.rtab[-1]), ered)
    assert nopen == run["nopen"]
    m = len(run["sr_cols"])
    assert np.abs(sr[:, :m].T - np.array(run["sr_cols"])).max() < S_TOL
    assert np.abs(si[:, :m].T - np.array(run["si_cols"])).max() < S_TOL
    s = sr + 1j * si
    assert np.abs(s @ s.conj().T - np.eye(nopen)).max() < S_TOL


# ---------------------------------------------------------------------------
# molscat-ityp6: LDMD to RMID, AIRY to RMAX, state-to-state cross sections
# ---------------------------------------------------------------------------
def _ityp6_system():
    from oracle import itype6 as I6
    with open(os.path.join(HERE, "golden", "molscat_ityp6.json")) as f:
        g = json.load(f)
    s = g["system"]
    pot = I6.BuckMSV(*s["beta"], *s["c6c8"], *s["x1234"], [tuple(a) for a in s["alphas"]],
                     [lm for lm, _ in s["lambda"][1:]])
    sysm = I6.Itype6(ured=s["ured"], roti=tuple(s["roti"]), jmax=s["jmax"], lam=[tuple(x) for x in s["lambda"]],
                     pfunc=pot, rm=s["rm"], epsil=s["epsil"], isym=s["isym"])
    return g, sysm


def _ityp6_block(g, sysm, blk, short_range=None):
    from oracle import aiprop as A
    s = g["system"]
    ch = sysm.channels(blk["jtot"], blk["block"])
    c = sysm.coupling(blk["jtot"], blk["block"])
    res = A.molscat_two_segment(sysm, c, s["energy_cm"], s["rmin"], s["rmax"], s["steps"], s["irmset"], s["rvfac"],
                                s["tolhi"], short_range=short_range)
    return c, res, A.partial_cross_sections(sysm, c, ch, res, blk["jtot"])


def _check_sigma(xs, blk):
    # six significant digits printed: half a unit of the sixth digit, plus an
    # absolute floor for entries at the rounding-noise level of the block
    big = max(x["sigma"] for x in blk["sigma"])
    for x in blk["sigma"]:
        got = xs[(x["final"], x["initial"])]
        assert abs(got - x["sigma"]) <= 6e-6 * x["sigma"] + 1e-9 * big, (blk["jtot"], blk["block"], x, got)


@pytest.mark.parametrize("jtot", [0, 1, 2, 5, 10, 20, 30, 40, 60, 80])
def test_ityp6_oracle_cross_sections_match_reference(jtot):
    """The oracle alone (MDPROP + AIRY): N = 2..59."""
    g, sysm = _ityp6_system()
    for blk in g["blocks"]:
        if blk["jtot"] == jtot:
            _check_sigma(_ityp6_block(g, sysm, blk)[2], blk)


@pytest.mark.gpu
@pytest.mark.parametrize("jtot", [5, 10, 20, 40, 60, 80])
def test_ityp6_gpu_short_range_matches_reference(gpu, jtot):
    """The GPU propagates the LDMD segment (N = 39..59, past the reference's
    N > 30 switch to DSYTRF/DSYNEG), the oracle's AIRY the long range: the
    reference's printed cross sections, the oracle's Y(RMID) within 5e-8 and
    its NODES exactly."""
    from oracle import oracle as O
    from molscat_b200.propagators import propagate
    g, sysm = _ityp6_system()
    for blk in g["blocks"]:
        if blk["jtot"] != jtot:
            continue
        seen = {}

        def gpu_ldmd(rtab, ptab, nstep, dr, ered, y0, c_holder=seen):
            oc = c_holder["c"]
            c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent)
            y, nodes = propagate("LDMD", c, Segment(nstep, dr, rtab, ptab), ered, y0)
            yo, no, st, _ = O.mdprop(oc, rtab, ptab, nstep, dr, ered, y0)
            assert st == 0 and nodes == no
            assert cases.rel_err(y, yo) < Y_TOL
            c_holder["checked"] = True
            return y, nodes

        seen["c"] = sysm.coupling(blk["jtot"], blk["block"])
        assert seen["c"].n > 30
        _, _, xs = _ityp6_block(g, sysm, blk, short_range=gpu_ldmd)
        assert seen.get("checked")
        _check_sigma(xs, blk)
