"""bound-Mg_NH and field-Mg_NH (examples/output/*-Mg_NH.output): Mg + NH(3Sigma) in a
magnetic field, ITYPE=9 with the atom(1S) + 3Sigma basis plug-in, MTOT = -1,
parity block 2, N = 100 channels in an asymptotically non-diagonal basis;
MDPROP outward RMIN = 2.3 -> RMATCH = 7 A (DR = 0.01), AIRY inward RMAX = 50
-> RMATCH (TOLHI = 1e-6, POWR = 3); state 170 converged to 1e-4 MHz at four
fields, energies relative to the field-dependent threshold of n=0, j=1,
m_j=-1.

* oracle (CPU): the threshold EREF at every field to the printed digits, the
  node counts at EMIN and EMAX, and the converged energy at 370 G within the
  reference's own convergence tolerance DTOL of the printed one.
* GPU: the outward MDPROP segment on the device (the one-CTA kernels, N =
  100) with the oracle's AIRY for the inward segment: node counts at EMIN and
  EMAX and the converged energies within DTOL of the printed ones, and the
  matching eigenvalue at the converged energy equal to the oracle's.

field-Mg_NH: the same system at fixed energies (0, -20, -40 MHz relative to
the field-dependent threshold), AIRY with TOLHI = 0 (a whole number of steps
growing as R^(4/3), drset.f / drcalc.f), state 170 crossing each energy as
the field rises from 1 to 400 G, converged to 1e-4 G:
* oracle: node counts at FLDMIN and FLDMAX, and the crossing field at 0 MHz
  converged inside a bracket of +-2 G around the printed one;
* GPU: the full search from FLDMIN to FLDMAX with the outward segments of
  every trial field batched on the device and the oracle's AIRY inward.
"""
import json
import os

import numpy as np
import pytest

import cases
from molscat_b200.bound import BoundProblem, adiabatic_wkb_y, converge_steps, find_states_converged
from molscat_b200.field import FieldProblem, field_node_counts, find_fields_converged
from molscat_b200.propagators import Coupling, Segment, radial_grid

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "bound_mg_nh.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def field_golden():
    with open(os.path.join(HERE, "golden", "field_mg_nh.json")) as f:
        return json.load(f)


def _system(g, field):
    from oracle import atom_3sigma as A
    s = g["system"]
    pot = A.MgNHPotential([(c["angle"], c["r"], c["e"]) for c in g["cuts"]])
    return A.Atom3Sigma(ured=s["ured"], roti=tuple(s["roti"]), nmin=s["nmin"], nmax=s["nmax"], lmax=s["lmax"],
                        lam=s["lambda"], pot=pot, field=field, spin=s["spin"])


class _Run:
    """The example at one field: system, coupling, outward segment, AIRY."""

    def __init__(self, g, field):
        from oracle import atom_3sigma as A
        from oracle import oracle as O
        s = g["system"]
        self.s = s
        self.sysm = _system(g, field)
        self.eref = self.sysm.threshold(s["monqn"])
        self.cm2ru = self.sysm.cm2ru
        self.mhz = A.MHZ_IN_CM
        self.oc = self.sysm.coupling(s["jtot"], s["block"])
        oc = self.oc
        self.c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent, nconst=oc.nconst)
        nout = int(round((s["rmatch"] - s["rmin"]) / s["drs"]))
        dr = (s["rmatch"] - s["rmin"]) / nout
        rtab = radial_grid(s["rmin"], dr, nout)
        self.seg_out = Segment(nout, dr, rtab, O.ptable(self.sysm, rtab))

    def ered(self, mhz):
        return (self.eref + mhz * self.mhz) * self.cm2ru

    def to_mhz(self, e):
        return (e / self.cm2ru - self.eref) / self.mhz

    def airy_in(self, e):
        from oracle import aiprop as AI
        s = self.s
        z0 = adiabatic_wkb_y(self.c, s["rmax"], self.sysm.pvec(s["rmax"]), e, False)
        y, nodes, _ = AI.aiprop(self.oc, self.sysm, z0, s["rmax"], s["rmatch"], -s["drl"], e,
                                tolhi=s["tolhil"], powr=3.0)
        return y, nodes

    def oracle_eval(self, ereds):
        from oracle import oracle as O
        so = self.seg_out
        cnt, eig = [], []
        for e in ereds:
            y0 = adiabatic_wkb_y(self.c, float(so.rtab[0]), so.ptab[0], float(e), True)
            yo, no, st, _ = O.mdprop(self.oc, so.rtab, so.ptab, so.nstep, so.dr, float(e), y0)
            assert st == 0
            yi, ni = self.airy_in(float(e))
            ev = np.linalg.eigvalsh(yo - yi)
            cnt.append(no + ni + int(np.sum(ev <= 0.0)))
            eig.append(float(ev[np.argmin(np.abs(ev))]))
        return np.array(cnt), np.array(eig)

    def tolerances(self):
        s = self.s
        tol = 1.0e-7 * self.mhz * self.cm2ru      # converge well inside the reference's DTOL
        coarse = 1.0 * self.mhz * self.cm2ru
        return tol, coarse


def test_thresholds_match_reference(golden):
    from oracle import atom_3sigma as A
    for st in golden["sets"]:
        sysm = _system(golden, st["field"])
        e = sysm.threshold(golden["system"]["monqn"])
        assert abs(e - st["eref_cm"]) < 6e-13          # printed to 11 significant digits
        assert abs(e / A.MHZ_IN_CM - st["eref_mhz"]) < 6e-7


def test_basis_size(golden):
    sysm = _system(golden, golden["sets"][0]["field"])
    s = golden["system"]
    assert len(sysm.channels(s["jtot"], s["block"])) == golden["nchan"]


def test_oracle_reproduces_reference_bound_state(golden):
    st = golden["sets"][0]
    run = _Run(golden, st["field"])
    s = golden["system"]
    lo, hi = run.ered(s["emin_mhz"]), run.ered(s["emax_mhz"])
    c, _ = run.oracle_eval([lo, hi])
    assert (int(c[0]), int(c[1])) == (st["count_emin"], st["count_emax"])
    tol, coarse = run.tolerances()
    res, rounds = converge_steps(run.oracle_eval, lo, hi, tol, coarse)
    assert len(res) == len(st["states"])
    for (k, e, _, _), ref in zip(res, st["states"]):
        assert k + 1 == ref["state"]
        assert abs(run.to_mhz(e) - ref["energy_mhz"]) < s["dtol_mhz"]


@pytest.mark.gpu
@pytest.mark.parametrize("iset", [0, 3])
def test_gpu_mdprop_with_airy_reproduces_reference(golden, iset):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    st = golden["sets"][iset]
    s = golden["system"]
    run = _Run(golden, st["field"])
    bp = BoundProblem(run.c, run.seg_out, prop="LDMD", inward=run.airy_in)
    tol, coarse = run.tolerances()
    res, rounds = find_states_converged(bp, run.ered(s["emin_mhz"]), run.ered(s["emax_mhz"]), tol, coarse)
    assert len(res) == len(st["states"])
    from molscat_b200.bound import node_counts
    for (k, e, _, _), ref in zip(res, st["states"]):
        assert k + 1 == ref["state"]
        assert abs(run.to_mhz(e) - ref["energy_mhz"]) < s["dtol_mhz"]
        cg, _, _, _, eg = node_counts(bp, [e])
        co, eo = run.oracle_eval([e])
        assert int(cg[0]) == int(co[0])
        assert abs(eg[0] - eo[0]) < 1e-7 * max(1.0, abs(eo[0]))
    cg = node_counts(bp, [run.ered(s["emin_mhz"]), run.ered(s["emax_mhz"])])[0]
    assert (int(cg[0]), int(cg[1])) == (st["count_emin"], st["count_emax"])


class _FieldRun:
    """field-Mg_NH at one energy: the field enters the P table (the Zeeman
    constant term) and the threshold the energy is measured from."""

    def __init__(self, g, fg, energy_mhz):
        import copy

        from oracle import aiprop as AI
        from oracle import atom_3sigma as A
        s, fs = g["system"], fg["system"]
        self.s, self.fs = s, fs
        self.base = _system(g, 0.0)
        self.copy = copy.copy
        self.mhz = A.MHZ_IN_CM
        self.emhz = energy_mhz
        self.cm2ru = self.base.cm2ru
        self.oc = self.base.coupling(s["jtot"], s["block"])
        oc = self.oc
        self.c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent, nconst=oc.nconst)
        nout = int(round((fs["rmatch"] - fs["rmin"]) / fs["drs"]))
        self.dr = (fs["rmatch"] - fs["rmin"]) / nout
        self.nout = nout
        self.rtab = radial_grid(fs["rmin"], self.dr, nout)
        self.nin, self.drin = AI.drset(fs["rmax"], fs["rmatch"], fs["drl"], fs["tolhil"], fs["powrl"])

    def sysm(self, f):
        m = self.copy(self.base)
        m.field = float(f)
        return m

    def ered(self, f):
        return (self.sysm(f).threshold(self.s["monqn"]) + self.emhz * self.mhz) * self.cm2ru

    def seg_out(self, f):
        from oracle import oracle as O
        return Segment(self.nout, self.dr, self.rtab, O.ptable(self.sysm(f), self.rtab))

    def airy_in(self, f, c, e):
        from oracle import aiprop as AI
        fs = self.fs
        m = self.sysm(f)
        z0 = adiabatic_wkb_y(self.c, fs["rmax"], m.pvec(fs["rmax"]), e, False)
        y, nodes, _ = AI.aiprop(self.oc, m, z0, fs["rmax"], fs["rmatch"], self.drin, e, tolhi=0.0,
                                powr=fs["powrl"], nstep=self.nin)
        return y, nodes

    def oracle_eval(self, fields):
        from oracle import oracle as O
        cnt, eig = [], []
        for f in fields:
            e = self.ered(f)
            so = self.seg_out(f)
            y0 = adiabatic_wkb_y(self.c, float(so.rtab[0]), so.ptab[0], e, True)
            yo, no, st, _ = O.mdprop(self.oc, so.rtab, so.ptab, so.nstep, so.dr, e, y0)
            assert st == 0
            yi, ni = self.airy_in(f, self.c, e)
            ev = np.linalg.eigvalsh(yo - yi)
            cnt.append(no + ni + int(np.sum(ev <= 0.0)))
            eig.append(float(ev[np.argmin(np.abs(ev))]))
        return np.array(cnt), np.array(eig)

    def problem(self):
        return FieldProblem(lambda f: self.c, ered_at=self.ered, segments_at=lambda f: (self.seg_out(f), None),
                            inward=self.airy_in, prop="LDMD")


def test_field_oracle_reproduces_reference_crossing(golden, field_golden):
    fs = field_golden["system"]
    ref = field_golden["energies"][0]
    run = _FieldRun(golden, field_golden, ref["energy_mhz"])
    c, _ = run.oracle_eval([fs["fldmin"], fs["fldmax"]])
    assert (int(c[0]), int(c[1])) == (ref["count_fldmin"], ref["count_fldmax"])
    f_ref = ref["states"][0]["field_g"]
    res, _ = converge_steps(run.oracle_eval, f_ref - 2.0, f_ref + 2.0, 1.0e-7, 4.0)
    assert len(res) == 1
    k, f, _, _ = res[0]
    assert k + 1 == ref["states"][0]["state"]
    assert abs(f - f_ref) < fs["dtol_g"]


@pytest.mark.gpu
@pytest.mark.parametrize("ie", [0, 2])
def test_field_gpu_mdprop_with_airy_reproduces_reference(golden, field_golden, ie):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    fs = field_golden["system"]
    ref = field_golden["energies"][ie]
    run = _FieldRun(golden, field_golden, ref["energy_mhz"])
    fp = run.problem()
    cnt = field_node_counts(fp, [fs["fldmin"], fs["fldmax"]])[0]
    assert (int(cnt[0]), int(cnt[1])) == (ref["count_fldmin"], ref["count_fldmax"])
    res, rounds = find_fields_converged(fp, fs["fldmin"], fs["fldmax"], 1.0e-7, 1.0)
    assert len(res) == len(ref["states"])
    for (k, f, _, _), st in zip(res, ref["states"]):
        assert k + 1 == st["state"]
        assert abs(f - st["field_g"]) < fs["dtol_g"]
