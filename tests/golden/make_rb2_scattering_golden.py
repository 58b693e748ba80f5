"""Extract the molscat-basic_Rb2 example (85Rb + 85Rb scattering length in
the lowest (aa) channel: the field-basic_Rb2 system, ITYPE=9 uncoupled
basis, MTOT = 8/2, block 2, N = 28; MDPROP RMIN = 3 -> RMID = 21 bohr, AIRY
RMID -> RMAX = 15000 bohr, then YTRANS, YTOK, KTOS and CALCA, 1e-7 K above
the aa threshold, fields 800..900 G) into a committed fixture.

    MOLSCAT_REF=<path to molscat checkout> python tests/golden/make_rb2_scattering_golden.py

writes tests/golden/molscat_basic_rb2.json with
* the run's parameters from examples/input/molscat-basic_Rb2.input;
* the Rb2 curve parameters (source_code/Hdata-Rb2-2010.f, read as
  make_rb2_golden.py reads them);
* from examples/output/molscat-basic_Rb2.output: the basis list; for every
  field the reference energy and the K-dependent scattering lengths CALCA
  prints (CHAN, L, POW, WVEC, RE(A), IM(A) in bohr); for the first, middle
  and last field the 28 thresholds YTRANS prints (THRESHOLD, L,
  ENERGY/CM-1).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_rb2_golden as M  # noqa: E402  (needs MOLSCAT_REF too)

OUT = os.path.join(HERE, "molscat_basic_rb2.json")
NUM = M.NUM


def read_input():
    with open(os.path.join(M.REF, "examples", "input", "molscat-basic_Rb2.input")) as f:
        t = re.sub(r"!.*", "", f.read())
    inp = {k.lower(): M._num(t, k) for k in ("URED", "RMIN", "RMID", "RMAX", "DR", "TOLHIL", "JTOTL", "ENERGY",
                                              "EUNITS", "FLDMIN", "FLDMAX", "DFIELD", "ISA", "GSA", "INUCA",
                                              "HFSPLA", "GA", "INUCB", "LMAX", "MXLAM")}
    inp["monqn"] = [int(x) for x in M._nums(t, "MONQN", 4)]
    inp["nterm"] = [int(x) for x in M._nums(t, "NTERM", int(inp["mxlam"]))]
    nss = inp["nterm"][2]
    a = M._nums(t, r"A", nss)
    npw = [int(x) for x in M._nums(t, "NPOWER", nss)]
    e = M._nums(t, "E", sum(1 for p in npw if p == 0))
    terms, ie = [], 0
    for ai, pi in zip(a, npw):
        if pi == 0:
            terms.append([ai, 0, e[ie]])
            ie += 1
        else:
            terms.append([ai, pi, None])
    inp["ss_terms"] = terms
    for k in ("isa", "inuca", "inucb", "lmax", "jtotl", "mxlam", "eunits"):
        inp[k] = int(inp[k])
    return inp


def read_output():
    with open(os.path.join(M.REF, "examples", "output", "molscat-basic_Rb2.output")) as f:
        t = f.read()
    block = int(re.search(r"SYMMETRY BLOCK =\s+(\d+) SELECTS", t).group(1))
    i0 = t.index("BASIS FUNCTION LIST:")
    lst = t[i0:t.index("EFV SET", i0)]
    rows = re.findall(r"^\s+(\d+)\s+(\d+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(\d+)\s*$", lst, re.M)
    channels = [[int(x) for x in r[2:]] for r in rows]
    fields = []
    parts = re.split(r"EFV SET\s+\d+:", t[i0:])[1:]
    for k, p in enumerate(parts):
        fg = float(re.search(r"MAGNETIC Z FIELD =\s+(" + NUM + ")", p).group(1))
        eref = float(re.search(r"REFERENCE ENERGY IS\s+(" + NUM + r")\s+CM-1", p).group(1))
        th = p[p.index("THRESHOLD       L"):p.index("K-DEPENDENT")]
        thr = [[int(m.group(1)), int(m.group(2)), float(m.group(3))] for m in
               re.finditer(r"^\s+(\d+)\s+(\d+)\s+(" + NUM + r")\s+" + NUM + r"\s*$", th, re.M)]
        sl = p[p.index("CHAN   L POW"):]
        lengths = [[int(m.group(1)), int(m.group(2)), int(m.group(3)), float(m.group(4)), float(m.group(5)),
                    float(m.group(6))] for m in
                   re.finditer(r"^\s+(\d+)\s+(\d+)\s+(\d+)\s+(" + NUM + r")\s+(" + NUM + r")\s+(" + NUM + r")\s*$",
                               sl.split("-----")[0], re.M)]
        f = {"field_g": fg, "eref_cm": eref, "lengths": lengths}
        if k in (0, len(parts) // 2, len(parts) - 1):  # the thresholds of three fields
            f["thresholds"] = thr
        fields.append(f)
    return block, channels, fields


def main():
    inp = read_input()
    block, channels, fields = read_output()
    inp["block"] = block
    g = {"source": "examples/input/molscat-basic_Rb2.input, examples/output/molscat-basic_Rb2.output, "
                   "source_code/Hdata-Rb2-2010.f",
         "system": inp, "hannover": M.read_hdata(), "channels": channels, "fields": fields}
    with open(OUT, "w") as f:
        json.dump(g, f, indent=0)
    print(OUT, len(channels), "channels,", len(fields), "fields")


if __name__ == "__main__":
    main()
