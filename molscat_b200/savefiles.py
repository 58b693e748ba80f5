"""The reference's unformatted result files, so that tools built around them
can read what the device computed.

* ILDSVU log-derivative files (source_code/ldrdwt.f): the global header
  (LDRWGH: LABEL, ITYPE, NLEV, NLEVEL, NQN, NNRG, URED, IPROGM), the global
  vectors (LDRWGV: JLEV, ELEVEL, ENERGY), then per propagation its header
  and EFV record (LDRWPH), its channel vectors (LDRWPV: J, L, EINT) and its
  matrices (LDRWMD: the record MATCODE = -687608722, then R and Y), in the
  order mol.driver.f:1537 and scctrl.f:281-282 write them.
* ISAVEU S-matrix records of one (JTOT, energy) block (sproc.f:255-280):
  the header (JTOT, INRG, IB, JFIELD, ENERGN, EFV(0:NEFVP), EREF, IEXCH,
  WGHT, NOPEN), the open channels (level index, L or, for BOUND-style
  bases, CENT, and WVEC), then the lower triangles of SREAL and SIMAG row
  by row (or, with IPHSUM > 0, the diagonal S and the K matrix).

The layout is Fortran sequential unformatted as gfortran writes it: every
record framed by its byte length as a 4-byte little-endian integer before
and after, INTEGER as 4 bytes, DOUBLE PRECISION as 8, CHARACTER*80 as 80
bytes, arrays column-major.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

MATCODE = -687608722  # ldrdwt.f: marks another matrix in an ILDSVU file


def _rec(f, payload: bytes):
    n = struct.pack("<i", len(payload))
    f.write(n + payload + n)


def records(path: str) -> list:
    """Every record of a sequential unformatted file, as bytes."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    p = 0
    while p < len(data):
        (n,) = struct.unpack_from("<i", data, p)
        body = data[p + 4:p + 4 + n]
        (m,) = struct.unpack_from("<i", data, p + 4 + n)
        if m != n or len(body) != n:
            raise ValueError(f"broken record framing at byte {p}")
        out.append(body)
        p += 8 + n
    return out


def _i(*v) -> bytes:
    return struct.pack("<%di" % len(v), *[int(x) for x in v])


def _d(*v) -> bytes:
    return struct.pack("<%dd" % len(v), *[float(x) for x in v])


def _ia(a) -> bytes:
    return np.asarray(a, dtype="<i4").tobytes(order="F")


def _da(a) -> bytes:
    return np.asarray(a, dtype="<f8").tobytes(order="F")


class LDFile:
    """Writer of an ILDSVU log-derivative file."""

    def __init__(self, path: str):
        self.f = open(path, "wb")

    def header(self, label: str, itype: int, nlev: int, nlevel: int, nqn: int, nnrg: int, ured: float,
               iprogm: int):
        """LDRWGH; IPROGM >= 17 is refused, as ldrdwt.f refuses it."""
        if iprogm >= 17:
            raise ValueError("log-derivative files are defined for output versions below 17")
        lab = label.encode("ascii")[:80].ljust(80)
        _rec(self.f, lab + _i(itype, nlev, nlevel, nqn, nnrg) + _d(ured) + _i(iprogm))

    def vectors(self, jlev, elevel, energy):
        """LDRWGV: JLEV(NLEV, NQN), ELEVEL(NLEVEL), ENERGY(NNRG)."""
        _rec(self.f, _ia(jlev) + _da(elevel) + _da(energy))

    def propagation(self, jtot: int, inrg: int, en: float, iexch: int, wt: float, iblock: int, nch: int,
                    ered: float, ep2ru: float, efv=(), iefvst: int = 1, nefv: int = 0, isvefv: int = 0):
        """LDRWPH: the header of one propagation and its EFV(IEFVST:NEFVP) record."""
        _rec(self.f, _i(jtot, inrg) + _d(en) + _i(iexch) + _d(wt) + _i(iblock, nch) + _d(ered, ep2ru)
             + _i(iefvst, nefv, isvefv))
        _rec(self.f, _da(np.asarray(efv, dtype=np.float64)))

    def channels(self, j, l, eint):
        """LDRWPV: J(NCH), L(NCH), EINT(NCH)."""
        _rec(self.f, _ia(j) + _ia(l) + _da(eint))

    def matrix(self, r: float, y: np.ndarray):
        """LDRWMD: MATCODE, then R and Y(NCH, NCH)."""
        _rec(self.f, _i(MATCODE))
        _rec(self.f, _d(r) + _da(np.asarray(y, dtype=np.float64)))

    def close(self):
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class LDPropagation:
    jtot: int
    inrg: int
    en: float
    iexch: int
    wt: float
    iblock: int
    nch: int
    ered: float
    ep2ru: float
    efv: np.ndarray
    j: np.ndarray = None
    l: np.ndarray = None
    eint: np.ndarray = None
    matrices: list = field(default_factory=list)  # [(R, Y)]


def read_ld(path: str) -> dict:
    """Parse an ILDSVU file written in the layout above."""
    rs = records(path)
    h = rs[0]
    label = h[:80].decode("ascii").rstrip()
    itype, nlev, nlevel, nqn, nnrg = struct.unpack_from("<5i", h, 80)
    (ured,) = struct.unpack_from("<d", h, 100)
    (iprogm,) = struct.unpack_from("<i", h, 108)
    v = rs[1]
    o = 4 * nlev * nqn
    jlev = np.frombuffer(v[:o], dtype="<i4").reshape((nlev, nqn), order="F")
    elevel = np.frombuffer(v[o:o + 8 * nlevel], dtype="<f8")
    energy = np.frombuffer(v[o + 8 * nlevel:o + 8 * (nlevel + nnrg)], dtype="<f8")
    props = []
    k = 2
    while k < len(rs):
        ph = rs[k]
        jtot, inrg = struct.unpack_from("<2i", ph, 0)
        (en,) = struct.unpack_from("<d", ph, 8)
        (iexch,) = struct.unpack_from("<i", ph, 16)
        (wt,) = struct.unpack_from("<d", ph, 20)
        iblock, nch = struct.unpack_from("<2i", ph, 28)
        ered, ep2ru = struct.unpack_from("<2d", ph, 36)
        efv = np.frombuffer(rs[k + 1], dtype="<f8")
        p = LDPropagation(jtot, inrg, en, iexch, wt, iblock, nch, ered, ep2ru, efv)
        k += 2
        if k < len(rs) and len(rs[k]) == 16 * nch:
            c = rs[k]
            p.j = np.frombuffer(c[:4 * nch], dtype="<i4")
            p.l = np.frombuffer(c[4 * nch:8 * nch], dtype="<i4")
            p.eint = np.frombuffer(c[8 * nch:], dtype="<f8")
            k += 1
        while k < len(rs) and len(rs[k]) == 4 and struct.unpack("<i", rs[k])[0] == MATCODE:
            m = rs[k + 1]
            (r,) = struct.unpack_from("<d", m, 0)
            p.matrices.append((r, np.frombuffer(m[8:], dtype="<f8").reshape((nch, nch), order="F")))
            k += 2
        props.append(p)
    return {"label": label, "itype": itype, "nlev": nlev, "nlevel": nlevel, "nqn": nqn, "nnrg": nnrg,
            "ured": ured, "iprogm": iprogm, "jlev": jlev, "elevel": elevel, "energy": energy, "propagations": props}


def write_s_block(f, jtot: int, inrg: int, ib: int, jfield: int, energn: float, efv, eref: float, iexch: int,
                  wght: float, level, lval_or_cent, wvec, sr: np.ndarray, si: np.ndarray, bound: bool = False,
                  kmat: np.ndarray | None = None):
    """One (JTOT, energy) block of an ISAVEU file, open file f: the header,
    the open channels (level index, L, WVEC; CENT instead of L for a
    BOUND-style basis), then SREAL and SIMAG lower triangles row by row, or
    with kmat (IPHSUM > 0) the diagonal (SR, SI) pairs and K's lower
    triangle.  sr, si: NOPEN x NOPEN in CHNSRT order (Plan.unpack_s)."""
    nopen = sr.shape[0]
    _rec(f, _i(jtot, inrg, ib, jfield) + _d(energn) + _da(np.asarray(efv, dtype=np.float64)) + _d(eref)
         + _i(iexch) + _d(wght) + _i(nopen))
    ch = b""
    for i in range(nopen):
        ch += _i(level[i]) + (_d(lval_or_cent[i]) if bound else _i(lval_or_cent[i])) + _d(wvec[i])
    _rec(f, ch)
    tri = [(i, j) for i in range(nopen) for j in range(i + 1)]
    if kmat is None:
        _rec(f, _d(*[sr[i, j] for i, j in tri]))
        _rec(f, _d(*[si[i, j] for i, j in tri]))
    else:
        _rec(f, _d(*[x for i in range(nopen) for x in (sr[i, i], si[i, i])]))
        _rec(f, _d(*[kmat[i, j] for i, j in tri]))
