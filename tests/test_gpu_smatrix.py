"""Y -> K -> S on the device (YTOK/YTOKG/KSYM + KTOS) against the oracle's
restatement and the reference's printed S matrices (absolute 1e-8), up to
N = 1024 (matrices in shared memory to N = 64, in a device scratch above)."""
import numpy as np
import pytest

import cases
from molscat_b200 import _lib
from molscat_b200.propagators import Coupling, Plan, Segment

pytestmark = pytest.mark.gpu

S_TOL = 1e-8


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    _lib.load()


def oracle_s(c, seg, ered, y):
    from oracle import oracle as O
    oc = cases.to_oracle(c)
    wvec, nopen = O.gtwvec(ered, oc.eint)
    nb = O.chnsrt(oc.eint)
    return O.ktos(O.ytok(nb, wvec, oc.n, nopen, y, seg.rtab[-1], oc.cent))


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
def test_golden_smatrix_on_device(golden, prop):
    """The reference's printed S matrix (N=12, 8072 steps, E = 1000 and 900
    cm-1) from the propagation and the S-matrix kernel, all on the GPU."""
    from oracle import oracle as O
    s = golden["system"]
    run = golden["runs"][prop]
    sysm = O.Itype1(ured=s["ured"], be=s["be"], jlevel=s["jlevel"], lam=s["lambda"],
                    terms=[[tuple(t) for t in tl] for tl in s["terms"]], rm=s["rm"], epsil=s["epsil"])
    oc = sysm.coupling(s["jtot"], s["block"])
    c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent)
    emx = max(run["energies_cm"]) * sysm.cm2ru
    rstart, _ = O.findrm(sysm, oc, s["rmin"], emx, s["irmset"])
    nstep, dr = O.drset_fixed(rstart, s["rmax"], s["steps"], O.calck(0.0, emx, oc.eint))
    rtab = O.radial_grid(rstart, dr, nstep)
    seg = Segment(nstep, dr, rtab, O.ptable(sysm, rtab))
    ereds = [e * sysm.cm2ru for e in run["energies_cm"]]
    y0s = [O.yinit_adiabatic_wkb(sysm, oc, rstart, e) for e in ereds]
    plan = Plan(prop, [c], [seg], np.zeros(len(ereds), dtype=np.int32), np.array(ereds))
    sr, si, nodes, status, kfail = plan.run_host_smatrix(plan.pack(y0s))
    assert (status == 0).all()
    for j, blk in enumerate(run["smatrix"]):
        srj, sij = plan.unpack_s(sr, j), plan.unpack_s(si, j)
        err = max(max(abs(srj[x["row"] - 1, x["col"] - 1] - x["re"]), abs(sij[x["row"] - 1, x["col"] - 1] - x["im"]))
                  for x in blk)
        assert err < S_TOL, err
    plan.close()


@pytest.mark.parametrize("jtot,block", [(10, 1), (10, 2), (30, 1), (0, 2)])
def test_rotor_smatrix_on_device_equals_oracle(jtot, block):
    """The benchmark system (4000 steps 2.5-40 A) at energies with few and
    many open channels: device S against YTOK/KTOS restated on the oracle's Y."""
    from oracle import oracle as O
    energies = (150.0, 480.0)
    c, seg, jobs = cases.rotor_case(jtot, block, energies_cm=energies)
    plan = Plan("LDMD", [c], [seg], np.zeros(len(jobs), dtype=np.int32), np.array([e for e, _ in jobs]))
    sr, si, nodes, status, kfail = plan.run_host_smatrix(plan.pack([y0 for _, y0 in jobs]))
    assert (status == 0).all()
    for j, (ered, y0) in enumerate(jobs):
        yo, no, st, _ = O.mdprop(cases.to_oracle(c), seg.rtab, seg.ptab, seg.nstep, seg.dr, ered, y0)
        assert nodes[j] == no
        so_r, so_i = oracle_s(c, seg, ered, yo)
        assert plan.nopen(j) == so_r.shape[0]
        if so_r.size == 0:
            continue
        err = max(np.abs(plan.unpack_s(sr, j) - so_r).max(), np.abs(plan.unpack_s(si, j) - so_i).max())
        assert err < S_TOL, err
        # unitarity of the device S
        sm = plan.unpack_s(sr, j) + 1j * plan.unpack_s(si, j)
        assert np.abs(sm @ sm.conj().T - np.eye(sm.shape[0])).max() < 1e-9
    plan.close()


@pytest.mark.parametrize("ns", [(70,), (100, 36), (200,), (300, 130)])
def test_smatrix_large_n_on_device_equals_oracle(ns):
    """N above 64 (matrices in the device scratch), mixed with N <= 64 jobs
    in one plan: S against YTOK/KTOS on the device's own Y, per job, every
    energy with open and closed channels."""
    systems, segs, job_sys, job_e, y0s = [], [], [], [], []
    for s, n in enumerate(ns):
        c, seg, ered, y0 = cases.random_case(n, 40, seed=600 + n)
        systems.append(c)
        segs.append(seg)
        for de in (0.0, 7.0):
            job_sys.append(s)
            job_e.append(ered + de)
            y0s.append(y0)
    plan = Plan("LDMD", systems, segs, np.array(job_sys, dtype=np.int32), np.array(job_e))
    ybuf, nodes, status, _ = plan.run_host(plan.pack(y0s))
    sr, si, nodes2, status2, _ = plan.run_host_smatrix(plan.pack(y0s))
    assert (status == 0).all() and (status2 == 0).all()
    assert np.array_equal(nodes, nodes2)
    for j in range(plan.njobs):
        c, seg = systems[job_sys[j]], segs[job_sys[j]]
        so_r, so_i = oracle_s(c, seg, job_e[j], plan.unpack(ybuf, j))
        assert plan.nopen(j) == so_r.shape[0] and so_r.size > 0
        err = max(np.abs(plan.unpack_s(sr, j) - so_r).max(), np.abs(plan.unpack_s(si, j) - so_i).max())
        assert err < S_TOL, (j, err)
        sm = plan.unpack_s(sr, j) + 1j * plan.unpack_s(si, j)
        assert np.abs(sm @ sm.conj().T - np.eye(sm.shape[0])).max() < 1e-9
    plan.close()


def test_smatrix_needs_n_up_to_1024():
    c, seg, ered, y0 = cases.random_case(1100, 2, seed=5)
    from molscat_b200.propagators import PropagatorError
    try:
        plan = Plan("LDMD", [c], [seg], np.zeros(1, dtype=np.int32), np.array([ered]))
    except PropagatorError as e:  # the propagation's own limit
        assert e.status == _lib.MGPU_ERR_UNSUPPORTED
        return
    with pytest.raises(PropagatorError) as e:
        plan.run_host_smatrix(plan.pack([y0]))
    assert e.value.status == _lib.MGPU_ERR_UNSUPPORTED
    plan.close()
