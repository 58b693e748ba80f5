"""Extract the field-basic_Rb2 example (85Rb + 85Rb in the uncoupled
alkali-alkali basis, ITYPE=9, MTOT = 8/2, symmetry block 2, N = 28; MDPROP
outward RMIN = 3 -> RMATCH = 21 bohr, AIRY inward RMAX = 15000 bohr ->
RMATCH; three bound states crossing threshold between 800 and 900 G) into a
committed fixture.

Run with the reference project's checkout named by $MOLSCAT_REF (required):

    MOLSCAT_REF=<path to molscat checkout> python tests/golden/make_rb2_golden.py

writes tests/golden/field_basic_rb2.json with
* the run's parameters from examples/input/field-basic_Rb2.input (&INPUT,
  &BASIS9, &POTL);
* the parameters of the Rb2 singlet and triplet curves set by
  source_code/Hdata-Rb2-2010.f (the data module vstar-Hannover.f reads);
* from examples/output/field-basic_Rb2.output: the basis size, the node
  counts at FLDMIN and FLDMAX and the converged field of each state.
"""
import json
import os
import re
import sys

REF = os.environ.get("MOLSCAT_REF")
if not REF:
    sys.exit("set MOLSCAT_REF to the reference project's checkout")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "field_basic_rb2.json")
NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[EeDd][-+]?\d+)?"


def _f(x):
    return float(x.replace("D", "E").replace("d", "e"))


def _num(text, name):
    m = re.search(r"\b" + name + r"\s*=\s*(" + NUM + ")", text)
    return _f(m.group(1))


def _nums(text, name, count):
    m = re.search(r"\b" + name + r"\s*=\s*((?:" + NUM + r"\s*,\s*)*" + NUM + ")", text)
    vals = [_f(x) for x in re.findall(NUM, m.group(1))]
    return vals[:count]


def read_input():
    with open(os.path.join(REF, "examples", "input", "field-basic_Rb2.input")) as f:
        t = re.sub(r"!.*", "", f.read())
    inp = {k.lower(): _num(t, k) for k in ("URED", "RMIN", "RMATCH", "RMAX", "DR", "TOLHIL", "JTOTL", "ENERGY",
                                            "DTOL", "FLDMIN", "FLDMAX", "ISA", "GSA", "INUCA", "HFSPLA", "GA",
                                            "INUCB", "LMAX", "MXLAM")}
    inp["monqn"] = [int(x) for x in _nums(t, "MONQN", 4)]
    inp["lambda"] = [int(x) for x in _nums(t, "LAMBDA", int(inp["mxlam"]))]
    inp["nterm"] = [int(x) for x in _nums(t, "NTERM", int(inp["mxlam"]))]
    nss = inp["nterm"][2]
    a = _nums(t, r"A", nss)
    npw = [int(x) for x in _nums(t, "NPOWER", nss)]
    ne = sum(1 for p in npw if p == 0)
    e = _nums(t, "E", ne)
    terms, ie = [], 0
    for ai, pi in zip(a, npw):
        if pi == 0:
            terms.append([ai, 0, e[ie]])
            ie += 1
        else:
            terms.append([ai, pi, None])
    inp["ss_terms"] = terms
    for k in ("isa", "inuca", "inucb", "lmax", "jtotl", "mxlam"):
        inp[k] = int(inp[k])
    return inp


def read_hdata():
    with open(os.path.join(REF, "source_code", "Hdata-Rb2-2010.f")) as f:
        t = f.read()
    body = "\n".join(ln for ln in t.splitlines() if not ln[:1] in ("C", "c", "!"))
    na = [int(x) for x in re.findall(r"\d+", re.search(r"NA\s*=\s*\(/(.*?)/\)", body).group(1))]
    flat = [_f(x) for x in re.findall(NUM, re.search(r"RESHAPE\(\(/(.*?)/\)", body, re.S).group(1))]
    ncol = max(na)
    a = [flat[:ncol][: na[0]], flat[ncol:2 * ncol][: na[1]]]

    def pair(name):
        m = re.search(r"\b" + name + r"\s*=\s*\(/(.*?)/\)", body)
        return [_f(x) for x in re.findall(NUM, m.group(1))]

    def scalar(name):
        m = re.search(r"^\s*" + name + r"\s*=\s*(" + NUM + ")", body, re.M)
        return _f(m.group(1))

    h = {"na": na, "a": a}
    for k in ("RM", "B", "RSR", "RLR", "NSR", "ASR", "BSR", "ALPSR", "EXSIGN"):
        h[k.lower()] = pair(k)
    for k in ("C6", "C8", "C10", "CEX", "AEX", "GAMMA", "BETA"):
        h[k.lower()] = scalar(k)
    h["nex"] = int(scalar("NEX"))
    h["gambet"] = int(scalar("GAMBET"))
    h["runit"] = "bohr" if re.search(r"RUNITM\s*=\s*bohr_to_Angstrom", body) else "angstrom"
    for k in ("MATCHL", "MATCHV", "MATCHD"):
        h[k.lower()] = bool(re.search(k + r"\s*=\s*\.TRUE\.", body))
    return h


def read_output():
    with open(os.path.join(REF, "examples", "output", "field-basic_Rb2.output")) as f:
        t = f.read()
    block = int(re.search(r"SYMMETRY BLOCK =\s+(\d+) SELECTS", t).group(1))
    lst = t[t.index("BASIS FUNCTION LIST:"):]
    rows = re.findall(r"^\s+(\d+)\s+(\d+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(\d+)\s*$", lst, re.M)
    channels = [[int(x) for x in r[2:]] for r in rows]
    counts = [int(x) for x in re.findall(r"IMPLIES\s+(\d+) STATES BELOW SPECIFIED ENERGY", t)]
    states = [{"state": int(m.group(1)), "field_g": float(m.group(2))} for m in
              re.finditer(r"CONVERGED ON STATE NUMBER\s+(\d+) AT\s+MAGNETIC Z FIELD =\s+(\S+)", t)]
    return block, channels, counts, states


def main():
    inp = read_input()
    block, channels, counts, states = read_output()
    inp["block"] = block
    g = {"source": "examples/input/field-basic_Rb2.input, examples/output/field-basic_Rb2.output, "
                   "source_code/Hdata-Rb2-2010.f",
         "system": inp, "hannover": read_hdata(), "channels": channels,
         "count_fldmin": counts[0], "count_fldmax": counts[1], "states": states}
    with open(OUT, "w") as f:
        json.dump(g, f, indent=1)
    print(OUT, len(channels), "channels,", len(states), "states")


if __name__ == "__main__":
    main()
