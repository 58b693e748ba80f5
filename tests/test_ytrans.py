"""YTRANS before YTOK: the asymptotic basis of the alkali-pair channels and
the scattering lengths of molscat-basic_Rb2 (examples/output/
molscat-basic_Rb2.output; tests/golden/molscat_basic_rb2.json).

85Rb + 85Rb, uncoupled basis (ITYPE=9), MTOT = 8/2, block 2, N = 28: MDPROP
RMIN = 3 -> RMID = 21 bohr (DR = 0.002), AIRY RMID -> RMAX = 15000 bohr
(TOLHI = 1e-7), YTRANS at RMAX (the hyperfine + Zeeman Hamiltonian is not
diagonal in this basis: NCONST = 2), YTOK, KTOS, CALCA; E = 1e-7 K above the
aa threshold, two open channels (L = 0 and 2).

* CPU: the oracle's YTRANS (oracle/ytrans.py) gives the 28 printed
  thresholds at 800, 850 and 900 G (to 1e-12 cm-1, the print's precision);
  the product's host half (molscat_b200/ytrans.py) gives the oracle's
  basis; the oracle's whole chain gives the printed s-wave scattering length
  at 800 G to 1e-6 (real part) and 1e-5 (imaginary part).
* GPU: the short-range segment on the device, the oracle's AIRY between,
  YTRANS's transform and YTOK/KTOS on the device (Plan.set_asymptote,
  Plan.smatrix_host) give the oracle's S matrices and the printed s-wave
  scattering lengths at three fields; a random basis on the device equals
  the same basis applied on the host.

The L = 2 "scattering volume" (POW 4) comes from 1 - S_22 ~ 4e-9: the
reference's value and the oracle's differ by 1e-3 relative (the reference
evaluates the Airy sector functions with the approximations of scairy.f /
spropn.f, the oracle exactly), so it is held to 5e-3.
"""
import json
import os

import numpy as np
import pytest

from molscat_b200 import ytrans as YT

HERE = os.path.dirname(os.path.abspath(__file__))
K_IN_CM = 0.6950348004  # physical_constants_module.f: K_in_inv_cm


@pytest.fixture(scope="module")
def rb2():
    with open(os.path.join(HERE, "golden", "molscat_basic_rb2.json")) as f:
        return _Case(json.load(f))


class _Case:
    def __init__(self, g):
        from oracle import alk_alk as K
        from oracle import oracle as O
        from molscat_b200.propagators import Coupling, radial_grid
        self.g = g
        s = self.s = g["system"]
        h = dict(g["hannover"])
        runit = K.BOHR_ANG if h.pop("runit") == "bohr" else 1.0
        hann = K.Hannover(runitm=runit, **h)
        self.base = K.AlkAlk(ured=s["ured"], isa=s["isa"], inuca=s["inuca"], gsa=s["gsa"], ga=s["ga"],
                             hfspla=s["hfspla"], lmax=s["lmax"], inucb=s["inucb"], rm=runit,
                             curves=lambda r: (hann.vstar(0, r), hann.vstar(1, r)),
                             ss_terms=[tuple(t) for t in s["ss_terms"]])
        self.oc = self.base.coupling(s["jtotl"], s["block"])
        oc = self.oc
        self.c = Coupling(n=oc.n, nham=oc.nham, vl=oc.vl, eint=oc.eint, cent=oc.cent, nconst=oc.nconst)
        self.lval = np.rint(np.sqrt(oc.cent + 0.25) - 0.5).astype(int)
        self.nout = int(round((s["rmid"] - s["rmin"]) / s["dr"]))
        self.dr = (s["rmid"] - s["rmin"]) / self.nout
        self.rtab = radial_grid(s["rmin"], self.dr, self.nout)
        self.O = O

    def at(self, field):
        import copy
        m = copy.copy(self.base)
        m.field_g = float(field)
        return m

    def ered(self, field):
        return (self.at(field).threshold(self.s["monqn"]) + self.s["energy"] * K_IN_CM) * self.base.cm2ru

    def pconst(self, field):
        m = self.at(field)
        p = m.pvec(self.s["rmax"])
        p[: m.mxlam] = 0.0
        return p

    def field(self, fg):
        return next(f for f in self.g["fields"] if abs(f["field_g"] - fg) < 1e-9)

    def oracle_basis(self, fg):
        from oracle import ytrans as OY
        w = OY.operator(self.oc.vl, self.oc.nham, self.oc.n, self.pconst(fg))
        return OY.ytrans(w, self.lval, self.oc.cent)

    def short_range_oracle(self, fg):
        m = self.at(fg)
        e = self.ered(fg)
        pt = self.O.ptable(m, self.rtab)
        y0 = self.O.yinit_adiabatic_wkb(m, self.oc, self.s["rmin"], e)
        y, _, st, _ = self.O.mdprop(self.oc, self.rtab, pt, self.nout, self.dr, e, y0)
        assert st == 0
        return y

    def airy_out(self, fg, y):
        from oracle import aiprop as AI
        z, _, _ = AI.aiprop(self.oc, self.at(fg), y, self.s["rmid"], self.s["rmax"], self.dr, self.ered(fg),
                            tolhi=self.s["tolhil"], powr=3.0)
        return z

    def oracle_lengths(self, fg, z):
        from oracle import ytrans as OY
        O = self.O
        evec, eint, cent = self.oracle_basis(fg)
        e = self.ered(fg)
        wvec, nopen = O.gtwvec(e, eint)
        nb = O.chnsrt(eint)
        k = O.ytok(nb, wvec, self.oc.n, nopen, OY.transform(z, evec), self.s["rmax"], cent)
        sr, si = O.ktos(k)
        return sr, si, OY.calca(sr, si, nb, self.lval, wvec)


def _check_lengths(got, ref):
    """got: [(L, m, k, A)], ref: the printed [CHAN, L, POW, WVEC, RE, IM]."""
    assert len(got) == len(ref) == 2
    for (ell, m, k, a), (ch, lr, pw, wv, re_, im_) in zip(got, ref):
        assert (ell, m) == (lr, pw)
        assert abs(k - wv) <= 1e-8 * wv
        tol_re, tol_im = (1e-6, 1e-5) if ell == 0 else (5e-3, 5e-3)
        assert abs(a.real - re_) <= tol_re * abs(re_), (ell, a, re_)
        assert abs(a.imag - im_) <= tol_im * abs(im_), (ell, a, im_)


# --------------------------------------------------------------------------- CPU
def test_oracle_thresholds_match_reference(rb2):
    for f in rb2.g["fields"]:
        if "thresholds" not in f:
            continue
        _, eint, _ = rb2.oracle_basis(f["field_g"])
        ref = np.array([t[2] for t in f["thresholds"]])
        assert [t[1] for t in f["thresholds"]] == list(rb2.lval)
        assert np.max(np.abs(eint / rb2.base.cm2ru - ref)) < 1e-12


def test_product_basis_equals_oracle(rb2):
    for fg in (800.0, 850.0, 900.0):
        ev_o, ei_o, ce_o = rb2.oracle_basis(fg)
        w = YT.asymptotic_operator(rb2.c, rb2.pconst(fg))
        b = YT.asymptotic_basis(rb2.c, w)
        assert np.allclose(b.eint, ei_o, rtol=0, atol=1e-15 * np.abs(ei_o).max())
        assert np.allclose(b.evec, ev_o, rtol=0, atol=1e-12)
        assert np.array_equal(b.cent, ce_o)
        assert np.allclose(b.evec.T @ b.evec, np.eye(rb2.c.n), atol=1e-13)


def test_product_basis_rejects_unsupported_cases(rb2):
    import copy
    c = copy.copy(rb2.c)
    c.nrsq = 1
    with pytest.raises(NotImplementedError):
        YT.asymptotic_basis(c, np.eye(c.n))
    c.nconst = 0
    c.nrsq = 0
    with pytest.raises(ValueError):
        YT.asymptotic_basis(c, np.eye(c.n))


def test_oracle_scattering_length_matches_reference(rb2):
    fg = 800.0
    z = rb2.airy_out(fg, rb2.short_range_oracle(fg))
    _, _, got = rb2.oracle_lengths(fg, z)
    _check_lengths(got, rb2.field(fg)["lengths"])


# --------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()


@pytest.mark.gpu
def test_gpu_scattering_lengths_reproduce_reference(gpu, rb2):
    """Every field a system of one plan (LDMD on the device), the oracle's
    AIRY to RMAX, then YTRANS + YTOK + KTOS on the device."""
    from molscat_b200.bound import adiabatic_wkb_y
    from molscat_b200.propagators import Plan, Segment
    fields = (800.0, 850.0, 900.0)
    segs = [Segment(rb2.nout, rb2.dr, rb2.rtab, rb2.O.ptable(rb2.at(f), rb2.rtab)) for f in fields]
    es = np.array([rb2.ered(f) for f in fields])
    plan = Plan("LDMD", [rb2.c] * len(fields), segs, np.arange(len(fields)), es)
    y0 = [adiabatic_wkb_y(rb2.c, float(rb2.rtab[0]), s.ptab[0], e, True) for s, e in zip(segs, es)]
    ybuf, _, status, _ = plan.run_host(plan.pack(y0))
    assert (status == 0).all()
    zs = []
    for j, f in enumerate(fields):
        zs.append(rb2.airy_out(f, plan.unpack(ybuf, j)))
        b = YT.asymptotic_basis(rb2.c, YT.asymptotic_operator(rb2.c, rb2.pconst(f)))
        plan.set_asymptote(j, b.eint, b.cent, b.evec, rmatch=rb2.s["rmax"])
    sr, si, st = plan.smatrix_host(plan.pack(zs))
    assert (st == 0).all()
    for j, f in enumerate(fields):
        assert plan.nopen(j) == 2
        srj, sij = plan.unpack_s(sr, j), plan.unpack_s(si, j)
        b = YT.asymptotic_basis(rb2.c, YT.asymptotic_operator(rb2.c, rb2.pconst(f)))
        got = YT.scattering_lengths(srj, sij, b.eint, b.cent, es[j])
        _check_lengths(got, rb2.field(f)["lengths"])
        # the device's S against the oracle's from the same Y at RMAX
        sr_o, si_o, _ = rb2.oracle_lengths(f, zs[j])
        assert np.allclose(srj, sr_o, rtol=0, atol=1e-10) and np.allclose(sij, si_o, rtol=0, atol=1e-10)
    plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [12, 70])
def test_gpu_transform_equals_host_transform(gpu, n):
    """A random orthogonal basis given to the device equals the same basis
    applied to Y on the host (N = 12 shared-memory S kernel, 70 global)."""
    from molscat_b200.propagators import Coupling, Plan, Segment, radial_grid
    rng = np.random.default_rng(40 + n)
    a = rng.standard_normal((n, n))
    y = a + a.T + 4.0 * n * np.eye(n)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    eint = np.sort(rng.uniform(-1.0, 1.0, n))
    cent = np.array([float(ell * (ell + 1)) for ell in rng.integers(0, 4, n)])
    c = Coupling(n=n, nham=0, vl=np.zeros(0), eint=eint, cent=cent)
    rt = radial_grid(5.0, 0.1, 4)
    seg = Segment(4, 0.1, rt, np.zeros((rt.size, 0)))
    plans = [Plan("LDMD", [c], [seg], np.zeros(2, dtype=np.int32), np.array([0.3, 0.9])) for _ in range(2)]
    plans[0].set_asymptote(0, eint, cent, q, rmatch=30.0)
    plans[1].set_asymptote(0, eint, cent, None, rmatch=30.0)
    s0 = plans[0].smatrix_host(plans[0].pack([y, y]))
    s1 = plans[1].smatrix_host(plans[1].pack([q.T @ y @ q] * 2))
    for j in range(2):
        assert plans[0].nopen(j) == plans[1].nopen(j) > 0
        for b0, b1 in zip(s0[:2], s1[:2]):
            assert np.allclose(plans[0].unpack_s(b0, j), plans[1].unpack_s(b1, j), rtol=0, atol=1e-11)
    for p in plans:
        p.close()
