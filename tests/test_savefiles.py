"""The reference's unformatted result files (molscat_b200/savefiles.py):
ILDSVU log-derivative files (ldrdwt.f) and ISAVEU S-matrix blocks
(sproc.f:255-280).  The record layout is checked byte by byte against the
Fortran statements' item lists (gfortran framing: a 4-byte length before
and after each record), and a written file reads back exactly."""
import struct

import numpy as np

from molscat_b200 import savefiles as SF


def _frame(raw: bytes, p: int):
    (n,) = struct.unpack_from("<i", raw, p)
    (m,) = struct.unpack_from("<i", raw, p + 4 + n)
    assert n == m
    return n, p + 8 + n


def test_ld_file_layout_and_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    path = str(tmp_path / "ld.bin")
    nlev, nqn, nlevel, nnrg = 4, 2, 4, 2
    jlev = rng.integers(0, 9, (nlev, nqn))
    elevel = rng.uniform(0, 100, nlevel)
    energy = np.array([1000.0, 900.0])
    n = 5
    ys = [rng.standard_normal((n, n)) for _ in range(2)]
    with SF.LDFile(path) as f:
        f.header("model system", 1, nlev, nlevel, nqn, nnrg, 20.0, 16)
        f.vectors(jlev, elevel, energy)
        for k, y in enumerate(ys):
            f.propagation(10, k + 1, energy[k], 0, 1.0, 1, n, energy[k] * 0.5, 3.2, efv=[0.0, 850.0], nefv=1)
            f.channels(np.arange(n) + 1, np.arange(n) * 2, rng.uniform(0, 60, n))
            f.matrix(20.0, y)
    raw = open(path, "rb").read()
    # LDRWGH: CHARACTER*80 + 5 INTEGER + DOUBLE + INTEGER
    n0, p = _frame(raw, 0)
    assert n0 == 80 + 5 * 4 + 8 + 4
    n1, p = _frame(raw, p)
    assert n1 == 4 * nlev * nqn + 8 * nlevel + 8 * nnrg
    n2, p = _frame(raw, p)
    assert n2 == 4 + 4 + 8 + 4 + 8 + 4 + 4 + 8 + 8 + 3 * 4  # LDRWPH item list
    n3, p = _frame(raw, p)
    assert n3 == 2 * 8  # EFV(IEFVST:NEFVP)
    n4, p = _frame(raw, p)
    assert n4 == 16 * n  # J, L, EINT
    n5, q = _frame(raw, p)
    assert n5 == 4 and struct.unpack_from("<i", raw, p + 4)[0] == SF.MATCODE
    n6, _ = _frame(raw, q)
    assert n6 == 8 + 8 * n * n
    got = SF.read_ld(path)
    assert got["label"] == "model system" and got["iprogm"] == 16 and got["ured"] == 20.0
    assert np.array_equal(got["jlev"], jlev) and np.array_equal(got["energy"], energy)
    assert len(got["propagations"]) == 2
    for k, (p_, y) in enumerate(zip(got["propagations"], ys)):
        assert (p_.jtot, p_.inrg, p_.nch) == (10, k + 1, n)
        assert len(p_.matrices) == 1 and p_.matrices[0][0] == 20.0
        assert np.array_equal(p_.matrices[0][1], y)
        assert np.array_equal(p_.l, np.arange(n) * 2)


def test_ld_file_refuses_new_output_versions(tmp_path):
    import pytest
    with SF.LDFile(str(tmp_path / "x.bin")) as f:
        with pytest.raises(ValueError):
            f.header("x", 1, 1, 1, 1, 1, 1.0, 17)


def test_s_block_layout(tmp_path):
    rng = np.random.default_rng(4)
    no = 3
    a = rng.standard_normal((no, no)) + 1j * rng.standard_normal((no, no))
    s = a + a.T
    path = str(tmp_path / "s.bin")
    with open(path, "wb") as f:
        SF.write_s_block(f, 10, 1, 1, 0, 1000.0, [0.0], -0.5, 0, 1.0, [4, 7, 5], [9, 11, 9], [31.2, 31.2, 21.8],
                         s.real, s.imag)
        SF.write_s_block(f, 10, 1, 1, 0, 1000.0, [0.0], -0.5, 0, 1.0, [4, 7, 5], [90.0, 132.0, 90.0],
                         [31.2, 31.2, 21.8], s.real, s.imag, bound=True)
    rs = SF.records(path)
    assert len(rs) == 8
    assert len(rs[0]) == 4 * 4 + 8 + 8 + 8 + 4 + 8 + 4  # JTOT..JFIELD, ENERGN, EFV(0:0), EREF, IEXCH, WGHT, NOPEN
    assert len(rs[1]) == no * (4 + 4 + 8) and len(rs[5]) == no * (4 + 8 + 8)
    tri = [(i, j) for i in range(no) for j in range(i + 1)]
    assert np.array_equal(np.frombuffer(rs[2], "<f8"), np.array([s.real[i, j] for i, j in tri]))
    assert np.array_equal(np.frombuffer(rs[3], "<f8"), np.array([s.imag[i, j] for i, j in tri]))
    assert struct.unpack_from("<i", rs[1], 0)[0] == 4 and struct.unpack_from("<i", rs[1], 4)[0] == 9
