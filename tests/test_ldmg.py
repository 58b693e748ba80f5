"""MGPROP, the symplectic log-derivative propagator (mgprop.f; the
reference's IPROP = 8 with IMGSEL = 4 (CS4) or 5 (MA5)), on the one-warp
(N <= 40), one-CTA (N <= 200) and batched large-N kernels against the oracle's restatement
(oracle/oracle.py, mgprop), which reproduces the reference's MA5 S
matrices of molscat-all_propagators (tests/test_oracle_golden.py, 3.5e-12).

* CPU: the library's stage radii (mgpu_ldmg_radii) equal an independent
  accumulation R = RSTART + s*DR, R += a_k*DR (mgprop.f:76,129), bit for
  bit, with CS4's last-stage reuse; a plan rejects a segment of the wrong
  kind.
* GPU: the reference's golden S matrices (N = 12, 8072 sectors, both
  energies) with the GPU propagating; random systems N = 5..300 for CS4 and
  MA5 against the oracle (Y within 5e-8 of max|Y|, NODES exact).
"""
import numpy as np
import pytest

import cases
from molscat_b200.propagators import Plan, Segment, ldmg_radii

COEF_A = {
    "LDMG4": (0.20517766154229, 0.40302128160421, -0.12092087633891, 0.51272193319241, 0.0),
    "LDMG5": (0.33983962583911, -0.088601336903027, 0.58585647682596, -0.60303935653649, 0.32358079655470,
              0.44236379421975),
}


def _radii_by_hand(kind, r0, dr, nstep):
    a = COEF_A[kind]
    out = []
    for s in range(nstep):
        r = r0 + s * dr
        for k, ak in enumerate(a):
            if not (k == 0 and s > 0 and a[-1] == 0.0):
                out.append(r)
            r = r + ak * dr
    return np.array(out)


@pytest.mark.parametrize("kind", ["LDMG4", "LDMG5"])
def test_stage_radii(kind):
    for r0, dr, ns in ((0.6417, 0.0024, 37), (6.0, -0.01, 5), (1.0, 0.5, 1)):
        got = ldmg_radii(kind, r0, dr, ns)
        assert np.array_equal(got, _radii_by_hand(kind, r0, dr, ns))
        assert got.size == (4 * ns + 1 if kind == "LDMG4" else 6 * ns)


def test_segment_kind_checked():
    c, seg, ered, y0 = cases.random_case(6, 10, seed=3, kind="LDMG4")
    with pytest.raises(ValueError):
        Segment(10, seg.dr, seg.rtab, seg.ptab)  # an LD segment needs 2*NSTEP+1 rows
    with pytest.raises(ValueError):
        Plan("LDMG5", [c], [seg], np.zeros(1, dtype=np.int32), np.array([ered]))


# --------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()


class _Pot:
    def __init__(self, f):
        self.pvec = f


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["LDMG4", "LDMG5"])
@pytest.mark.parametrize("n", [5, 12, 24, 33, 40, 57, 106, 150])
def test_gpu_random_systems_match_oracle(gpu, kind, n):
    """N <= 40 on the one-warp kernels, above on the one-CTA kernels."""
    from oracle import oracle as O
    nstep = 300 if n <= 64 else 80
    c, seg, ered, y0 = cases.random_case(n, nstep, seed=60 + n, kind=kind)
    erg = ered + np.array([0.0, 3.0])
    plan = Plan(kind, [c], [seg], np.zeros(2, dtype=np.int32), erg)
    ybuf, nodes, status, _ = plan.run_host(plan.pack([y0, y0]))
    assert (status == 0).all()
    oc = cases.to_oracle(c)
    for j, e in enumerate(erg):
        yo, no = O.mgprop(oc, _Pot(seg.pvec), float(seg.rtab[0]), seg.dr, nstep, float(e), y0, int(kind[-1]))
        yg = plan.unpack(ybuf, j)
        assert nodes[j] == no
        assert np.abs(yg - yo).max() <= 5e-8 * np.abs(yo).max()
    plan.close()


@pytest.mark.gpu
def test_gpu_single_call_equals_plan(gpu):
    """mgpu_mgprop (the MGPROP drop-in, Python mgprop with MGPROP's argument
    list) gives the plan's result bit for bit."""
    from molscat_b200.propagators import mgprop, propagate
    c, seg, ered, y0 = cases.random_case(20, 50, seed=9, kind="LDMG5")
    plan = Plan("LDMG5", [c], [seg], np.zeros(1, dtype=np.int32), np.array([ered]))
    ybuf, nodes, status, _ = plan.run_host(plan.pack([y0]))
    ys, ns = propagate("LDMG5", c, seg, ered, y0)
    yf, nf = mgprop(c.n, c.nham, c.nham, y0, c.vl, None, c.eint, c.cent, float(seg.rtab[0]), None, 50, seg.dr,
                    ered, potential=seg.pvec, imgsel=5)
    assert np.array_equal(plan.unpack(ybuf, 0), ys) and np.array_equal(ys, yf)
    assert nodes[0] == ns == nf
    plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["LDMG4", "LDMG5"])
@pytest.mark.parametrize("n", [212, 300])
def test_gpu_large_n_matches_oracle(gpu, kind, n):
    """N > 200: the batched large-N kernels (64-pivot rounds), the stages as
    elementwise kernels between the inversions, a_k < 0 stages counted with
    sign -1."""
    from oracle import oracle as O
    nstep = 12
    c, seg, ered, y0 = cases.random_case(n, nstep, seed=80 + n, kind=kind)
    erg = ered + np.array([0.0, 2.0])
    plan = Plan(kind, [c], [seg], np.zeros(2, dtype=np.int32), erg)
    ybuf, nodes, status, _ = plan.run_host(plan.pack([y0, y0]))
    assert (status == 0).all()
    oc = cases.to_oracle(c)
    for j, e in enumerate(erg):
        yo, no = O.mgprop(oc, _Pot(seg.pvec), float(seg.rtab[0]), seg.dr, nstep, float(e), y0, int(kind[-1]))
        assert nodes[j] == no
        assert np.abs(plan.unpack(ybuf, j) - yo).max() <= 5e-8 * np.abs(yo).max()
    plan.close()


@pytest.mark.gpu
def test_gpu_reproduces_reference_smatrix(gpu, golden):
    """molscat-all_propagators IPROPS=8 (MA5): FINDRM, DRSET and YINIT from
    the oracle's driver restatement, the propagation and Y -> S on the device."""
    from oracle import oracle as O
    from molscat_b200.propagators import Coupling
    s = golden["system"]
    run = golden["runs"]["LDMG"]
    sysm = O.Itype1(ured=s["ured"], be=s["be"], jlevel=s["jlevel"], lam=s["lambda"],
                    terms=[[tuple(t) for t in tl] for tl in s["terms"]], rm=s["rm"], epsil=s["epsil"])
    oc = sysm.coupling(s["jtot"], s["block"])
    c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent)
    cm2ru = sysm.cm2ru
    eredmx = max(run["energies_cm"]) * cm2ru
    rstart, _ = O.findrm(sysm, oc, s["rmin"], eredmx, s["irmset"])
    nstep, dr = O.drset_fixed(rstart, s["rmax"], s["steps"], O.calck(0.0, eredmx, oc.eint))
    assert nstep == run["nstep"][0]
    seg = Segment.build(rstart, dr, nstep, sysm.pvec, oc.nham, kind="LDMG5")
    es = np.array(run["energies_cm"]) * cm2ru
    y0 = [O.yinit_adiabatic_wkb(sysm, oc, rstart, e) for e in es]
    plan = Plan("LDMG5", [c], [seg], np.zeros(len(es), dtype=np.int32), es)
    sr, si, nodes, status, _ = plan.run_host_smatrix(plan.pack(y0))
    assert (status == 0).all()
    for j, blk in enumerate(run["smatrix"]):
        srj, sij = plan.unpack_s(sr, j), plan.unpack_s(si, j)
        err = max(max(abs(srj[e["row"] - 1, e["col"] - 1] - e["re"]), abs(sij[e["row"] - 1, e["col"] - 1] - e["im"]))
                  for e in blk)
        assert err < 1e-8, err
    plan.close()
