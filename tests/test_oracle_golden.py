"""Pin the CPU oracle against the reference's own printed S matrices.

examples/output/molscat-all_propagators.output prints the 6x6 open-channel
S matrix to 14 significant digits for LDMD (IPROPS=6), LDJ (IPROPS=5) and
the symplectic LDMG (IPROPS=8, IMGSEL=5: MA5) and the quasi-adiabatic LDMA
(IPROPS=7),
ITYPE=1, JTOT=10, block 1, N=12, E=1000 and 900 cm-1 (fixture made by
tests/golden/make_golden.py).  The restated MOLSCAT driver path (FINDRM,
DRSET, YINIT, propagator, YTOK, KTOS) must reproduce them within 1e-8.
"""
import numpy as np
import pytest

from oracle import oracle as O

TOL = 1e-8


def _system(g):
    s = g["system"]
    return O.Itype1(ured=s["ured"], be=s["be"], jlevel=s["jlevel"], lam=s["lambda"],
                    terms=[[tuple(t) for t in tl] for tl in s["terms"]], rm=s["rm"], epsil=s["epsil"])


@pytest.mark.parametrize("prop", ["LDMD", "LDJ", "LDMG", "LDMA"])
def test_smatrix_matches_reference_output(golden, prop):
    s = golden["system"]
    run = golden["runs"][prop]
    res = O.molscat_smatrix(_system(golden), s["jtot"], s["block"], run["energies_cm"],
                            s["rmin"], s["rmax"], s["steps"], "LDMG5" if prop == "LDMG" else prop)
    for r, blk, nstep in zip(res, run["smatrix"], run["nstep"]):
        assert r.nstep == nstep
        assert [c + 1 for c in r.nb[: r.nopen]] == [4, 7, 5, 2, 8, 10]
        err = max(max(abs(r.sr[e["row"] - 1, e["col"] - 1] - e["re"]),
                      abs(r.si[e["row"] - 1, e["col"] - 1] - e["im"])) for e in blk)
        assert err < TOL, (prop, r.energy, err)
        # unitarity of the restated S matrix
        S = r.sr + 1j * r.si
        assert np.abs(S @ S.conj().T - np.eye(r.nopen)).max() < 1e-9


def test_syminv_small_and_lapack_paths():
    rng = np.random.default_rng(7)
    for n in (1, 2, 5, 30, 31, 64):
        a = rng.standard_normal((n, n))
        a = a + a.T + np.diag(rng.uniform(-3, 3, n))
        inv, k = O.syminv(a)
        full = np.tril(inv) + np.tril(inv, -1).T
        assert np.allclose(full @ a, np.eye(n), atol=1e-8)
        assert k == int((np.linalg.eigvalsh(a) < 0).sum())


def test_syminv_zero_pivot_fails():
    a = np.array([[0.0, 1.0], [1.0, 0.0]])
    _, k = O.syminv(a)
    assert k == 3  # IFAIL = N+1 (syminv.f:95)


def test_wigner_symbols():
    # (1 1 2;000)=sqrt(2/15), {1 1 1;1 1 1}=1/6
    assert abs(O.threej000(1, 1, 2) - np.sqrt(2 / 15)) < 1e-15
    assert abs(O.sixj(1, 1, 1, 1, 1, 1) - 1 / 6) < 1e-15
    assert O.threej000(1, 1, 1) == 0.0
