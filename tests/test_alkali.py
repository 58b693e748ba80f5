"""The product's alkali-pair basis (molscat_b200/alkali.py) against the
oracle's restatement of base9-alk_alk_ucpld.f (oracle/alk_alk.py), and the
synthetic BOUND/FIELD sweep on the GPU against the oracle.

* CPU: the same channels, couplings (to 1e-14) and Breit-Rabi thresholds
  for the Rb2 example (identical bosons) and the synthetic heteronuclear
  pair; the Zeeman term diagonal.
* GPU: a field sweep of the synthetic pair (every field a system that shares
  VL, P and the U(C) preparation, the Zeeman term as a per-field EINT) gives
  the oracle's node counts at every field, with the field in the P vector as
  the reference puts it; a plan whose systems share tables gives bit for bit
  the results of one whose systems do not.
"""
import json
import os

import numpy as np
import pytest

from molscat_b200 import alkali as AK
from molscat_b200.bound import adiabatic_wkb_y

HERE = os.path.dirname(os.path.abspath(__file__))


def _oracle_pair(pair, curves=None, ss_terms=()):
    from oracle import alk_alk as K
    return K.AlkAlk(ured=pair.ured, isa=pair.sa, inuca=pair.ia, gsa=pair.gsa, ga=pair.ga, hfspla=pair.hfsa,
                    lmax=pair.lmax, isb=pair.sb, inucb=-1 if pair.ident else pair.ib, gsb=pair.gsb, gb=pair.gb,
                    hfsplb=pair.hfsb, curves=curves, ss_terms=list(ss_terms), rm=pair.rm)


def _rb2_pair():
    with open(os.path.join(HERE, "golden", "field_basic_rb2.json")) as f:
        s = json.load(f)["system"]
    return AK.AlkaliPair(ured=s["ured"], sa=s["isa"], ia=s["inuca"], gsa=s["gsa"], ga=s["ga"], hfsa=s["hfspla"],
                         lmax=s["lmax"], ib=s["inucb"], rm=0.529177210544), s


def _compare(pair, mtot, block):
    ok = _oracle_pair(pair)
    assert pair.channels(mtot, block) == ok.channels(mtot, block)
    terms, zee, lval = pair.operators(mtot, block)
    oc = ok.coupling(mtot, block)
    ovl = oc.vl.reshape(-1, oc.nham)
    nt = terms.shape[1]
    assert np.allclose(terms, ovl[:, :nt], rtol=0, atol=1e-14)
    n = lval.size
    col = np.repeat(np.arange(n), np.arange(1, n + 1))
    row = np.arange(n * (n + 1) // 2) - col * (col + 1) // 2
    zo = ovl[:, nt]
    assert not zo[row != col].any()          # the Zeeman term is diagonal
    assert np.allclose(zee, zo[row == col], rtol=0, atol=1e-18)


def test_rb2_identical_bosons_match_oracle():
    pair, s = _rb2_pair()
    for mtot, block in ((s["jtotl"], s["block"]), (4, 1), (0, 2), (-2, 1)):
        _compare(pair, mtot, block)


def test_config4_heteronuclear_matches_oracle():
    sw = AK.config4_sweep(nout=10, nin=10)
    for mtot, block in ((4, 2), (8, 1), (0, 1)):
        _compare(sw.pair, mtot, block)
    assert sw.n == 106


def test_thresholds_match_oracle():
    sw = AK.config4_sweep(nout=10, nin=10)
    ok = _oracle_pair(sw.pair)
    for f in (0.0, 1.0, 333.3, 1000.0):
        ok.field_g = f
        for mq in ((2, 2, 2, 2), (4, 4, 2, -2), (2, -2, 4, 0)):
            assert abs(sw.pair.threshold_cm(mq, f) - ok.threshold(mq)) < 1e-15


# --------------------------------------------------------------------------- GPU
def _oracle_counts(sw, fields, oracle_pair):
    """Counts with the oracle: the reference's arrangement (field in P)."""
    from oracle import oracle as O
    oc = oracle_pair.coupling(sw.mtot, sw.block)
    out = []
    for f in fields:
        oracle_pair.field_g = float(f)
        e = sw.ered_at(float(f))
        res = []
        for seg, outward in ((sw.seg_out, True), (sw.seg_in, False)):
            pt = O.ptable(oracle_pair, seg.rtab)
            y0 = adiabatic_wkb_y(oc, float(seg.rtab[0]), pt[0], e, outward)
            y, nodes, st, _ = O.mdprop(oc, seg.rtab, pt, seg.nstep, seg.dr, e, y0)
            assert st == 0
            res.append((y, nodes))
        ev = np.linalg.eigvalsh(res[0][0] - res[1][0])
        out.append(res[0][1] + res[1][1] + int(np.sum(ev <= 0.0)))
    return np.array(out)


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()


@pytest.mark.gpu
@pytest.mark.parametrize("mtot,block,nfield", [(8, 1, 24), (4, 2, 2)])
def test_gpu_field_sweep_counts_match_oracle(gpu, mtot, block, nfield):
    from molscat_b200.field import FieldProblem, field_node_counts
    sw = AK.config4_sweep(mtot=mtot, block=block, nout=900, nin=1200)
    fields = np.linspace(0.0, 1000.0, nfield)
    fp = FieldProblem(sw.coupling_at, sw.seg_out, sw.seg_in, ered_at=sw.ered_at, prop="LDMD")
    cg = field_node_counts(fp, fields)[0]
    ok = _oracle_pair(sw.pair, curves=lambda r: (sw.singlet(r), sw.triplet(r)),
                      ss_terms=[(-(0.529177210544 ** 3), -3, None)])
    ok.rm = 1.0
    co = _oracle_counts(sw, fields, ok)
    assert np.array_equal(cg, co)


@pytest.mark.gpu
@pytest.mark.parametrize("mtot,block,family", [(8, 1, None), (4, 2, 0), (4, 2, 2)],
                         ids=["warp-N30", "cta-N106", "big-N106"])
def test_gpu_shared_tables_equal_separate(gpu, mtot, block, family):
    """Every kernel family: the one-warp kernels (N = 30), the one-CTA kernels
    and the batched large-N kernels (N = 106, the family forced)."""
    from molscat_b200 import _lib
    if family is not None:
        _lib.set_family_for_n(97, 112, family, "LDMD")
    try:
        _shared_vs_separate(mtot, block)
    finally:
        if family is not None:
            _lib.set_family_for_n(97, 112, -1, "LDMD")


def _shared_vs_separate(mtot, block):
    from molscat_b200.propagators import Coupling, Plan, Segment
    sw = AK.config4_sweep(mtot=mtot, block=block, nout=300, nin=300)
    fields = np.linspace(10.0, 900.0, 6)
    cs = [sw.coupling_at(f) for f in fields]
    es = np.array([sw.ered_at(f) for f in fields])
    y0 = [adiabatic_wkb_y(c, float(sw.seg_out.rtab[0]), sw.seg_out.ptab[0], e, True) for c, e in zip(cs, es)]
    shared = Plan("LDMD", cs, [sw.seg_out] * len(cs), np.arange(len(cs)), es)
    assert shared.shared_systems == len(cs) - 1
    sep_cs = [Coupling(n=c.n, nham=c.nham, vl=c.vl.copy(), eint=c.eint, cent=c.cent) for c in cs]
    sep_segs = [Segment(sw.seg_out.nstep, sw.seg_out.dr, sw.seg_out.rtab.copy(), sw.seg_out.ptab.copy())
                for _ in cs]
    sep = Plan("LDMD", sep_cs, sep_segs, np.arange(len(cs)), es)
    assert sep.shared_systems == 0
    a = shared.run_host(shared.pack(y0))
    b = sep.run_host(sep.pack(y0))
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    shared.close()
    sep.close()
