"""AIRY, the long-range propagator (aiprop.f; the reference's IPROPL = 9):
the host's sector geometry and Airy sector functions (molscat_b200/airy.py)
and the device's sweep (mgpu_airy_run_host) against the oracle's
restatement (oracle/aiprop.py), which the molscat-ityp6, Mg-NH and Rb2
pins hold to the reference (tests/test_itype6.py, test_mg_nh.py,
test_rb2.py, test_ytrans.py).

* CPU: the tables and sector functions driven through a numpy model of the
  device's sweep give the oracle's Z (1e-10 of max|Z|), NODES and sector
  count: outward and inward with TOLHI step control, and the TOLHI = 0
  series.
* GPU: the device's sweep against the oracle on random systems;
  molscat-basic_Rb2 on product code alone -- MDPROP to 21 bohr and AIRY to
  15000 bohr on the device, YTRANS, YTOK and KTOS on the device -- giving
  the printed s-wave scattering lengths; bound-Mg_NH (N = 100) with the
  product's AIRY inward, the printed bound states within DTOL.
"""
import json
import os

import numpy as np
import pytest

import cases
from molscat_b200 import airy as AY

HERE = os.path.dirname(os.path.abspath(__file__))


class _Pot:
    def __init__(self, f):
        self.pvec = f


def _sweep(t: AY.AiryTables, z0, ered):
    """The device's sweep in numpy."""
    from oracle import oracle as O
    n = t.n
    z = np.array(z0, dtype=np.float64)
    y = AY.energy_y124(t, ered)
    nodes = 0
    for k in range(t.widths.size):
        z = t.tmat[k].T @ z @ t.tmat[k]
        z = 0.5 * (z + z.T)
        inv, cnt = O.syminv(z + np.diag(y[k, :, 0]))
        inv = np.tril(inv) + np.tril(inv, -1).T
        nodes += cnt if t.outward else n - cnt
        z = -(y[k, :, 1][:, None] * inv * y[k, :, 1][None, :]) + np.diag(y[k, :, 2])
    z = t.vfin @ z @ t.vfin.T
    return 0.5 * (z + z.T), nodes


CASES = [  # (n, rstart, rstop, drnow, tolhi, nstep)
    (6, 1.6, 6.0, 0.02, 1.0e-3, 0),
    (9, 6.0, 1.8, -0.05, 1.0e-3, 0),
    (7, 1.7, 5.0, 0.03, 0.0, 90),
]


@pytest.mark.parametrize("n, r0, r1, dr, tolhi, nstep", CASES, ids=["out", "in", "tolhi0"])
def test_tables_with_model_sweep_match_oracle(n, r0, r1, dr, tolhi, nstep):
    from oracle import aiprop as AI
    c, seg, ered, y0 = cases.random_case(n, 40, seed=600 + n)
    oc = cases.to_oracle(c)
    t = AY.sector_tables(c, seg.pvec, r0, r1, dr, ered, tolhi=tolhi, powr=3.0, nstep=nstep)
    zm, nm = _sweep(t, y0, ered)
    zo, no, nsect = AI.aiprop(oc, _Pot(seg.pvec), y0, r0, r1, dr, ered, tolhi=tolhi, powr=3.0, nstep=nstep)
    assert t.widths.size == nsect
    assert nm == no
    assert np.abs(zm - zo).max() <= 1e-10 * np.abs(zo).max()


# --------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()


@pytest.mark.gpu
@pytest.mark.parametrize("n, r0, r1, dr, tolhi, nstep", CASES + [(40, 1.6, 5.0, 0.02, 1.0e-3, 0)],
                         ids=["out", "in", "tolhi0", "n40"])
def test_gpu_sweep_matches_oracle(gpu, n, r0, r1, dr, tolhi, nstep):
    from oracle import aiprop as AI
    c, seg, ered, y0 = cases.random_case(n, 40, seed=600 + n)
    oc = cases.to_oracle(c)
    t = AY.sector_tables(c, seg.pvec, r0, r1, dr, ered, tolhi=tolhi, powr=3.0, nstep=nstep)
    plan = AY.AiryPlan(t)
    zs, nodes, status = plan.run_host([y0], [ered])
    assert status[0] == 0
    zo, no, _ = AI.aiprop(oc, _Pot(seg.pvec), y0, r0, r1, dr, ered, tolhi=tolhi, powr=3.0, nstep=nstep)
    assert nodes[0] == no
    assert np.abs(zs[0] - zo).max() <= 5e-8 * np.abs(zo).max()
    plan.close()


@pytest.mark.gpu
def test_gpu_rb2_scattering_lengths_on_product_code(gpu):
    """molscat-basic_Rb2 at 800 and 850 G with no oracle on the path: the
    coupling from the oracle's basis restatement is the only input taken
    from it (the product's alkali basis is the synthetic sweep's)."""
    from molscat_b200 import ytrans as YT
    from molscat_b200.bound import adiabatic_wkb_y
    from molscat_b200.propagators import Plan, Segment
    import test_ytrans as TY
    with open(os.path.join(HERE, "golden", "molscat_basic_rb2.json")) as f:
        case = TY._Case(json.load(f))
    s = case.s
    for fg in (800.0, 850.0):
        m = case.at(fg)
        e = case.ered(fg)
        seg = Segment(case.nout, case.dr, case.rtab, np.stack([m.pvec(float(r)) for r in case.rtab]))
        plan = Plan("LDMD", [case.c], [seg], np.zeros(1, dtype=np.int32), np.array([e]))
        y0 = adiabatic_wkb_y(case.c, float(case.rtab[0]), seg.ptab[0], e, True)
        ybuf, _, st, _ = plan.run_host(plan.pack([y0]))
        assert st[0] == 0
        t = AY.sector_tables(case.c, m.pvec, s["rmid"], s["rmax"], case.dr, e, tolhi=s["tolhil"], powr=3.0)
        ap = AY.AiryPlan(t)
        zs, _, ast = ap.run_host([plan.unpack(ybuf, 0)], [e])
        assert ast[0] == 0
        b = YT.asymptotic_basis(case.c, YT.asymptotic_operator(case.c, case.pconst(fg)))
        plan.set_asymptote(0, b.eint, b.cent, b.evec, rmatch=s["rmax"])
        sr, si, sst = plan.smatrix_host(plan.pack(zs))
        assert sst[0] == 0
        got = YT.scattering_lengths(plan.unpack_s(sr, 0), plan.unpack_s(si, 0), b.eint, b.cent, e)
        TY._check_lengths(got, case.field(fg)["lengths"])
        ap.close()
        plan.close()


@pytest.mark.gpu
def test_gpu_bound_mg_nh_with_product_airy(gpu):
    """bound-Mg_NH (N = 100) at 370 G: MDPROP outward on the device and
    AIRY inward (RMAX = 50 -> RMATCH = 7 bohr, TOLHI = 1e-6) through
    AiryInward, its geometry from the first energy of the search as the
    reference's ISCRU = 30 run keeps it: the printed states within DTOL."""
    import test_mg_nh as MG
    from molscat_b200.bound import BoundProblem, find_states_converged
    with open(os.path.join(HERE, "golden", "bound_mg_nh.json")) as f:
        g = json.load(f)
    st = g["sets"][0]
    s = g["system"]
    run = MG._Run(g, st["field"])
    inward = AY.AiryInward(run.c, run.sysm.pvec, s["rmax"], s["rmatch"], -s["drl"], tolhi=s["tolhil"], powr=3.0)
    bp = BoundProblem(run.c, run.seg_out, prop="LDMD", inward=inward)
    tol, coarse = run.tolerances()
    res, _ = find_states_converged(bp, run.ered(s["emin_mhz"]), run.ered(s["emax_mhz"]), tol, coarse)
    assert len(res) == len(st["states"])
    for (k, e, _, _), ref in zip(res, st["states"]):
        assert k + 1 == ref["state"]
        assert abs(run.to_mhz(e) - ref["energy_mhz"]) < s["dtol_mhz"]

