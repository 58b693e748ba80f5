"""bound-Mg_NH (examples/output/bound-Mg_NH.output): Mg + NH(3Sigma) in a
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
"""
import json
import os

import numpy as np
import pytest

import cases
from molscat_b200.bound import BoundProblem, adiabatic_wkb_y, converge_steps, find_states_converged
from molscat_b200.propagators import Coupling, Segment, radial_grid

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "bound_mg_nh.json")) as f:
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
