"""GPU parity: libmolscat_gpu (through its C ABI) against the CPU oracle.

Tolerances (FP64 throughout):
* Y at RSTOP: max|Y_gpu - Y_oracle| / max(1, max|Y_oracle|) < 5e-8.  The GPU
  inverts in blocks of four pivots on tensor cores, the oracle pivot by pivot;
  over hundreds of steps of random strongly coupled systems the two rounding
  orders drift apart by up to ~1e-8 relative (both kernel families; node
  counts stay identical).  The physically meaningful comparisons below (S
  matrices) keep the 1e-8 absolute bound.
* S matrices: absolute 1e-8 (against the oracle and the reference's golden print)
* NODES and channel ordering: exact
"""
import numpy as np
import pytest

import cases
from molscat_b200 import _lib
from molscat_b200.propagators import Plan, PropagatorError, Segment, propagate, Coupling

pytestmark = pytest.mark.gpu

Y_TOL = 5e-8
S_TOL = 1e-8


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    _lib.load()


def oracle_prop(prop, c, seg, ered, y0):
    from oracle import oracle as O
    f = O.mdprop if prop == "LDMD" else O.ldprop
    y, nodes, st, kf = f(cases.to_oracle(c), seg.rtab, seg.ptab, seg.nstep, seg.dr, ered, y0)
    return y, nodes, st, kf


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 12, 17, 30, 31, 36, 40, 41, 45, 64, 80, 100, 128, 150, 200,
                               201, 256, 300, 512])
def test_random_systems(prop, n):
    """One warp per matrix (N <= 40), one CTA per matrix (N <= 200; LDPROP
    <= 128), batched large-N kernels over matrices in global memory above
    that; all on FP64 tensor cores."""
    nstep = 160 if n <= 64 else (60 if n <= 300 else 20)
    c, seg, ered, y0 = cases.random_case(n, nstep, seed=1000 + n)
    yg, ng = propagate(prop, c, seg, ered, y0)
    yo, no, st, _ = oracle_prop(prop, c, seg, ered, y0)
    assert st == 0
    assert ng == no
    assert cases.rel_err(yg, yo) < Y_TOL
    assert np.array_equal(yg, yg.T)


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
@pytest.mark.parametrize("n", [3, 17, 36, 45, 64])
def test_register_tile_family(prop, n):
    """The 4x4 register-tile kernels (scalar sweep) selected explicitly."""
    old = _lib.set_kernel_family(_lib.FAMILY_TILE4)
    try:
        c, seg, ered, y0 = cases.random_case(n, 160, seed=2000 + n)
        yg, ng = propagate(prop, c, seg, ered, y0)
    finally:
        _lib.set_kernel_family(old)
    yo, no, st, _ = oracle_prop(prop, c, seg, ered, y0)
    assert st == 0 and ng == no
    assert cases.rel_err(yg, yo) < Y_TOL


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
@pytest.mark.parametrize("kw", [dict(ivlfl=1), dict(nconst=1, nrsq=1, conlen=3.0), dict(inward=True),
                                dict(ivlfl=1, nconst=1, inward=True)], ids=["iv", "const-rsq-conf", "inward", "iv-const-inward"])
def test_hammat_variants(prop, kw):
    c, seg, ered, y0 = cases.random_case(9, 200, seed=77, **kw)
    yg, ng = propagate(prop, c, seg, ered, y0)
    yo, no, st, _ = oracle_prop(prop, c, seg, ered, y0)
    assert st == 0 and ng == no
    assert cases.rel_err(yg, yo) < Y_TOL


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
def test_golden_smatrix_through_gpu(golden, prop):
    """The reference's printed S matrix (N=12, 8072 steps) with the GPU doing
    the propagation inside the restated MOLSCAT driver."""
    from oracle import oracle as O
    s = golden["system"]
    run = golden["runs"][prop]
    sysm = O.Itype1(ured=s["ured"], be=s["be"], jlevel=s["jlevel"], lam=s["lambda"],
                    terms=[[tuple(t) for t in tl] for tl in s["terms"]], rm=s["rm"], epsil=s["epsil"])
    oc = sysm.coupling(s["jtot"], s["block"])
    c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent)
    cm2ru = sysm.cm2ru
    emx = max(run["energies_cm"]) * cm2ru
    rstart, _ = O.findrm(sysm, oc, s["rmin"], emx, s["irmset"])
    nstep, dr = O.drset_fixed(rstart, s["rmax"], s["steps"], O.calck(0.0, emx, oc.eint))
    assert nstep == run["nstep"][0]
    rtab = O.radial_grid(rstart, dr, nstep)
    seg = Segment(nstep, dr, rtab, O.ptable(sysm, rtab))
    for e, blk in zip(run["energies_cm"], run["smatrix"]):
        ered = e * cm2ru
        y0 = O.yinit_adiabatic_wkb(sysm, oc, rstart, ered)
        yg, ng = propagate(prop, c, seg, ered, y0)
        yo, no, st, _ = oracle_prop(prop, c, seg, ered, y0)
        assert ng == no
        wvec, nopen = O.gtwvec(ered, oc.eint)
        nb = O.chnsrt(oc.eint)
        sr, si = O.ktos(O.ytok(nb, wvec, oc.n, nopen, yg, rtab[-1], oc.cent))
        err = max(max(abs(sr[x["row"] - 1, x["col"] - 1] - x["re"]), abs(si[x["row"] - 1, x["col"] - 1] - x["im"]))
                  for x in blk)
        assert err < S_TOL, err


@pytest.mark.parametrize("jtot,block,n", [(10, 1, 30), (10, 2, 36)])
def test_rotor_full_grid(jtot, block, n):
    """The benchmark system (4000 steps 2.5-40 A): N=30 takes the reference's
    unpivoted SYMINV path, N=36 its DSYTRF/DSYNEG/DSYTRI path."""
    from oracle import oracle as O
    c, seg, jobs = cases.rotor_case(jtot, block, energies_cm=(150.0, 480.0))
    assert c.n == n
    for ered, y0 in jobs:
        yg, ng = propagate("LDMD", c, seg, ered, y0)
        yo, no, st, _ = oracle_prop("LDMD", c, seg, ered, y0)
        assert st == 0 and ng == no
        assert cases.rel_err(yg, yo) < Y_TOL
        oc = cases.to_oracle(c)
        wvec, nopen = O.gtwvec(ered, oc.eint)
        if nopen == 0:  # E=150 cm-1 lies below every threshold of the N=30 block
            continue
        nb = O.chnsrt(oc.eint)
        sg = O.ktos(O.ytok(nb, wvec, n, nopen, yg, seg.rtab[-1], oc.cent))
        so = O.ktos(O.ytok(nb, wvec, n, nopen, yo, seg.rtab[-1], oc.cent))
        assert max(np.abs(sg[0] - so[0]).max(), np.abs(sg[1] - so[1]).max()) < S_TOL


def test_batch_equals_alone():
    """Every job of a mixed batch (several N buckets, energies, both
    propagators' systems) gives exactly the result it gives alone."""
    items = [cases.random_case(n, 120, seed=500 + n) for n in (3, 9, 16, 30, 33, 47, 90, 260)]
    systems = [it[0] for it in items]
    segs = [it[1] for it in items]
    job_sys, job_e, y0s = [], [], []
    for s, (c, seg, ered, y0) in enumerate(items):
        for de in (0.0, 5.0, 11.0):
            job_sys.append(s)
            job_e.append(ered + de)
            y0s.append(y0)
    for prop in ("LDMD", "LDJ"):
        plan = Plan(prop, systems, segs, np.array(job_sys), np.array(job_e))
        ybuf, nodes, status, kfail = plan.run_host(plan.pack(y0s))
        assert (status == 0).all()
        for j in range(plan.njobs):
            c, seg = systems[job_sys[j]], segs[job_sys[j]]
            ya, na = propagate(prop, c, seg, job_e[j], y0s[j])
            assert np.array_equal(plan.unpack(ybuf, j), ya)
            assert nodes[j] == na
        plan.close()


def _ref_y14(wref, half):
    """Y14 of the reference-potential solutions (mdprop.f:143-164)."""
    arg = half * np.sqrt(np.abs(wref))
    tn, th = np.tan(arg), np.tanh(arg)
    return np.where(wref < 0.0, arg / tn - arg * tn, arg / th + arg * th)


@pytest.mark.parametrize("n", [36, 64, 128, 256])
@pytest.mark.parametrize("eps", [1e-6, 1e-10])
def test_tiny_leading_pivot_against_bunch_kaufman(n, eps):
    """The first matrix MDPROP inverts is made well conditioned (eigenvalues
    +-1..3) but with a leading diagonal element eps times its largest entry:
    Bunch-Kaufman (the oracle, as the reference's SYMINL above N = 30) pivots
    there, the GPU's sweep does not.  The inertia, and so NODES, is the same;
    the unpivoted inverse loses about u/eps relative accuracy in that one
    inversion (a host model of the sweep shows 3e-12 at eps 1e-4, 3e-6 at
    1e-10), which is what the tolerance allows."""
    from molscat_b200.bound import w_matrix
    c, seg, ered, _ = cases.random_case(n, 20, seed=4000 + n)
    h = seg.dr / 2.0
    d1 = h * h / 3.0
    w0 = w_matrix(c, float(seg.rtab[0]), seg.ptab[0], ered)
    wref = np.diag(w_matrix(c, float(seg.rtab[1]), seg.ptab[1], ered))
    y14b = _ref_y14(wref, 0.5 * h) - d1 * wref
    rng = np.random.default_rng(n)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    m = (q * (rng.uniform(1.0, 3.0, n) * rng.choice([-1.0, 1.0], n))) @ q.T
    m[0, 0] = eps * np.abs(m).max()
    y0 = (m - d1 * w0 - np.diag(y14b)) / h
    y0 = 0.5 * (y0 + y0.T)
    yg, ng = propagate("LDMD", c, seg, ered, y0)
    yo, no, st, _ = oracle_prop("LDMD", c, seg, ered, y0)
    assert st == 0
    assert ng == no
    assert cases.rel_err(yg, yo) < max(Y_TOL, 100.0 * 1.1e-16 / eps)


def test_empty_plan():
    c, seg, ered, y0 = cases.random_case(4, 10, seed=3)
    plan = Plan("LDMD", [c], [seg], np.zeros(0, dtype=np.int32), np.zeros(0))
    y, nodes, status, kfail = plan.run_host(np.zeros(0))
    assert nodes.size == 0
    plan.close()


def test_zero_pivot_reports_step_like_reference():
    """Z(1,1)=0 on the first LDPROP inversion: the reference stops with
    'ERROR IN SYMINV CALLED FROM LDPROP' (ldprop.f:151-153)."""
    n = 2
    c = Coupling(n=n, nham=1, vl=np.zeros(3), eint=np.zeros(n), cent=np.zeros(n))
    seg = Segment(3, 1.0, np.array([1.0, 1.5, 2.0, 2.5, 3.0, 3.5, 4.0]), np.zeros((7, 1)))
    y0 = np.array([[-2.0, 1.0], [1.0, 0.0]])  # h=0.5: Z = h*Y + I -> Z11 = 0
    with pytest.raises(PropagatorError) as e:
        propagate("LDJ", c, seg, 0.0, y0)
    assert e.value.status == _lib.MGPU_ERR_INVERSION and e.value.step == 1
    assert "LDPROP" in str(e.value)
    _, _, st, kf = oracle_prop("LDJ", c, seg, 0.0, y0)
    assert st == 1 and kf == 1


@pytest.mark.parametrize("n", [6, 260])
def test_nonfinite_potential_is_flagged(n):
    c, seg, ered, y0 = cases.random_case(n, 50, seed=11)
    ptab = seg.ptab.copy()
    ptab[41, 1] = np.nan
    bad = Segment(seg.nstep, seg.dr, seg.rtab, ptab)
    for prop in ("LDMD", "LDJ"):
        with pytest.raises(PropagatorError) as e:
            propagate(prop, c, bad, ered, y0)
        assert e.value.status == _lib.MGPU_ERR_NONFINITE
        assert e.value.step == 21  # R index 41 = C of step 21


def test_unsupported_size():
    assert _lib.load().mgpu_max_n() == 1024
    for prop, n in (("LDMD", 1025), ("LDJ", 1025)):
        c = Coupling(n=n, nham=1, vl=np.zeros(n * (n + 1) // 2), eint=np.zeros(n), cent=np.zeros(n))
        seg = Segment(1, 0.1, np.array([1.0, 1.05, 1.1]), np.zeros((3, 1)))
        with pytest.raises(PropagatorError) as e:
            propagate(prop, c, seg, 1.0, np.eye(n))
        assert e.value.status == _lib.MGPU_ERR_UNSUPPORTED


def test_large_n_1024():
    """The largest bucket (N = 1024, 16 rounds of 64 pivots per inversion)."""
    c, seg, ered, y0 = cases.random_case(1024, 6, seed=1024)
    yg, ng = propagate("LDMD", c, seg, ered, y0)
    yo, no, st, _ = oracle_prop("LDMD", c, seg, ered, y0)
    assert st == 0 and ng == no
    assert cases.rel_err(yg, yo) < Y_TOL


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
@pytest.mark.parametrize("n", [5, 36, 64, 100, 150])
def test_batched_large_n_family_at_small_n(prop, n):
    """The batched global-memory kernels selected for small N (the
    autotuner's family 2; one to three 64-pivot rounds)."""
    _lib.set_family_for_n(n, n, _lib.FAMILY_BIG)
    try:
        c, seg, ered, y0 = cases.random_case(n, 120, seed=4000 + n)
        yg, ng = propagate(prop, c, seg, ered, y0)
    finally:
        _lib.set_family_for_n(-1, -1, -1)
    yo, no, st, _ = oracle_prop(prop, c, seg, ered, y0)
    assert st == 0 and ng == no
    assert cases.rel_err(yg, yo) < Y_TOL


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
@pytest.mark.parametrize("n", [100, 260])
@pytest.mark.parametrize("kw", [dict(ivlfl=1), dict(nconst=1, nrsq=1, conlen=3.0), dict(inward=True)],
                         ids=["iv", "const-rsq-conf", "inward"])
def test_hammat_variants_large(prop, n, kw):
    """IV indexing, NCONST/NRSQ/CONLEN and inward propagation through the
    one-CTA (N = 100) and batched large-N (N = 260) kernels."""
    c, seg, ered, y0 = cases.random_case(n, 40, seed=88 + n, **kw)
    yg, ng = propagate(prop, c, seg, ered, y0)
    yo, no, st, _ = oracle_prop(prop, c, seg, ered, y0)
    assert st == 0 and ng == no
    assert cases.rel_err(yg, yo) < Y_TOL
