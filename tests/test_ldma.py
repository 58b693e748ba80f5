"""MAPROP, the quasi-adiabatic log-derivative propagator (maprop.f; the
reference's IPROP = 7): the host's energy-independent tables
(molscat_b200/ldma.py) and the device's sweep (mgpu_ldma_run_host) against
the oracle's restatement (oracle/oracle.py, maprop), which reproduces the
reference's LDMA S matrices of molscat-all_propagators to 5.1e-10
(tests/test_oracle_golden.py).

* CPU: the tables driven through a numpy model of the device's sweep give
  the oracle's Y (1e-10 of max|Y|) and NODES on random systems, outward and
  inward; the host W equals the oracle's HAMMAT.
* GPU: random systems N = 5..64 against the oracle (Y within 5e-8 of
  max|Y|, NODES exact), several energies from one set of tables; the
  reference's golden S matrices (N = 12, 8072 sectors) with the GPU
  propagating and Y -> S on the device.
"""
import numpy as np
import pytest

import cases
from molscat_b200 import ldma as LA


class _Pot:
    def __init__(self, f):
        self.pvec = f


def _sweep(t: LA.LDMATables, y0, ered):
    """The device's sweep in numpy (the kernel's order of operations)."""
    from oracle import oracle as O
    n = t.n
    y = np.array(y0, dtype=np.float64)
    nodes = 0
    wmax = 24.0 / (t.dr * t.dr)
    for k in range(t.nstep):
        y = t.q[k].T @ ((y + t.corr[k]) @ t.q[k])
        wref = t.eival[k] - ered
        flam = 0.5 * np.sqrt(np.abs(wref))
        g = np.where(wref < 0.0, np.tan(flam * t.dr), np.tanh(flam * t.dr))
        sg = np.where(wref < 0.0, -1.0, 1.0)
        y1 = flam / g + sg * flam * g
        y2 = flam / g - sg * flam * g
        inv, cnt = O.syminv(y + np.diag(y1))
        inv = np.tril(inv) + np.tril(inv, -1).T
        cnt = n - cnt if t.dr < 0 else cnt
        if not np.any(wref > wmax):
            nodes += cnt
        y = -(y2[:, None] * inv * y2[None, :]) + np.diag(y1)
    return t.tfin @ y @ t.tfin.T + t.qfin, nodes


@pytest.mark.parametrize("n, inward", [(6, False), (14, False), (9, True)])
def test_tables_with_model_sweep_match_oracle(n, inward):
    from oracle import oracle as O
    nstep = 120
    c, seg, ered, y0 = cases.random_case(n, nstep, seed=500 + n, inward=inward)
    t = LA.ldma_tables(c, seg)
    oc = cases.to_oracle(c)
    for e in (ered, ered + 4.0):
        ym, nm = _sweep(t, y0, e)
        yo, no = O.maprop(oc, _Pot(seg.pvec), float(seg.rtab[0]), seg.dr, nstep, e, y0)
        assert nm == no
        assert np.abs(ym - yo).max() <= 1e-10 * np.abs(yo).max()


def test_host_w_equals_oracle_hammat():
    from oracle import oracle as O
    for kw in ({}, dict(ivlfl=1), dict(nconst=1, nrsq=1)):
        c, seg, ered, _ = cases.random_case(11, 10, seed=7, **kw)
        oc = cases.to_oracle(c)
        for ir in (0, 5, 20):
            r = float(seg.rtab[ir])
            assert np.allclose(LA.hammat_host(c, r, seg.ptab[ir], ered), O.hammat(oc, r, seg.ptab[ir], ered),
                               rtol=1e-14, atol=1e-12)


# --------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [5, 12, 33, 64])
def test_gpu_random_systems_match_oracle(gpu, n):
    from oracle import oracle as O
    nstep = 200
    c, seg, ered, y0 = cases.random_case(n, nstep, seed=520 + n)
    plan = LA.LDMAPlan(c, seg)
    erg = ered + np.array([0.0, 2.5, 5.0])
    ys, nodes, status = plan.run_host([y0] * len(erg), erg)
    assert (status == 0).all()
    oc = cases.to_oracle(c)
    for j, e in enumerate(erg):
        yo, no = O.maprop(oc, _Pot(seg.pvec), float(seg.rtab[0]), seg.dr, nstep, float(e), y0)
        assert nodes[j] == no
        assert np.abs(ys[j] - yo).max() <= 5e-8 * np.abs(yo).max()
    plan.close()


@pytest.mark.gpu
def test_gpu_reproduces_reference_smatrix(gpu, golden):
    """molscat-all_propagators IPROPS=7: FINDRM, DRSET and YINIT from the
    oracle's driver restatement; the sweep and Y -> S (a plan's S kernels at
    the segment's last radius) on the device."""
    from oracle import oracle as O
    from molscat_b200.propagators import Coupling, Plan, Segment
    s = golden["system"]
    run = golden["runs"]["LDMA"]
    sysm = O.Itype1(ured=s["ured"], be=s["be"], jlevel=s["jlevel"], lam=s["lambda"],
                    terms=[[tuple(t) for t in tl] for tl in s["terms"]], rm=s["rm"], epsil=s["epsil"])
    oc = sysm.coupling(s["jtot"], s["block"])
    c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent)
    eredmx = max(run["energies_cm"]) * sysm.cm2ru
    rstart, _ = O.findrm(sysm, oc, s["rmin"], eredmx, s["irmset"])
    nstep, dr = O.drset_fixed(rstart, s["rmax"], s["steps"], O.calck(0.0, eredmx, oc.eint))
    assert nstep == run["nstep"][0]
    seg = Segment.build(rstart, dr, nstep, sysm.pvec, oc.nham)
    es = np.array(run["energies_cm"]) * sysm.cm2ru
    y0 = [O.yinit_adiabatic_wkb(sysm, oc, rstart, e) for e in es]
    plan = LA.LDMAPlan(c, seg)
    ys, nodes, status = plan.run_host(y0, es)
    assert (status == 0).all()
    sp = Plan("LDMD", [c], [seg], np.zeros(len(es), dtype=np.int32), es)
    sr, si, st = sp.smatrix_host(sp.pack(ys))
    assert (st == 0).all()
    for j, blk in enumerate(run["smatrix"]):
        srj, sij = sp.unpack_s(sr, j), sp.unpack_s(si, j)
        err = max(max(abs(srj[e["row"] - 1, e["col"] - 1] - e["re"]), abs(sij[e["row"] - 1, e["col"] - 1] - e["im"]))
                  for e in blk)
        assert err < 1e-8, err
    plan.close()
    sp.close()
