"""Extract the bound-Mg_NH and field-Mg_NH examples (ITYPE=9 atom + 3Sigma
diatom in a magnetic field, N = 100 channels, MDPROP outward + AIRY inward)
into committed fixtures.

Run with the reference project's checkout named by $MOLSCAT_REF (required):

    MOLSCAT_REF=<path to molscat checkout> python tests/golden/make_mg_nh_golden.py

writes tests/golden/bound_mg_nh.json with
* the run's parameters from examples/input/bound-Mg_NH.input (&INPUT,
  &BASIS, &BASIS9, &POTL);
* per field set of examples/output/bound-Mg_NH.output: the field, the
  reference energy EREF (cm-1 and MHz), the node counts implied at EMIN and
  EMAX, the converged state number and its energy (MHz), the matching
  eigenvalue's index;
* the potential's angular cuts (angle, R, E) read from data/pot-Mg_NH.data,
  the input of the RKHS interpolation (first two columns: R and EINT1, as
  vstar-Mg_NH.f reads them);

and tests/golden/field_mg_nh.json with the parameters of
examples/input/field-Mg_NH.input (energies relative to the field-dependent
threshold, FLDMIN/FLDMAX, DTOL, TOLHIL = 0) and, per energy of
examples/output/field-Mg_NH.output, the node counts at FLDMIN and FLDMAX and
the converged field of each state (the same system and potential as the
bound fixture).
"""
import json
import os
import re
import sys

REF = os.environ.get("MOLSCAT_REF")
if not REF:
    sys.exit("set MOLSCAT_REF to the reference project's checkout")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bound_mg_nh.json")
OUT_FIELD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "field_mg_nh.json")


def _num(text, name):
    m = re.search(r"\b" + name + r"\s*=\s*([-+0-9.EeDd]+)", text)
    return float(m.group(1).replace("D", "E").replace("d", "e"))


def _list(text, name):
    m = re.search(r"\b" + name + r"\s*=\s*([-+0-9.,\sEe]+?)(?:,\s*[A-Z!]|\n\s*/|!)", text)
    return [float(x) for x in m.group(1).replace(",", " ").split()]


def read_input():
    with open(os.path.join(REF, "examples", "input", "bound-Mg_NH.input")) as f:
        t = f.read()
    roti = _list(t, "ROTI")
    lam = [int(x) for x in _list(t, "LAMBDA")]
    monqn = [int(x) for x in _list(t, "MONQN")]
    return {
        "ured": _num(t, "URED"), "rmin": _num(t, "RMIN"), "rmatch": _num(t, "RMATCH"), "rmax": _num(t, "RMAX"),
        "drs": _num(t, "DRS"), "drl": _num(t, "DRL"), "tolhil": _num(t, "TOLHIL"),
        "jtot": int(_num(t, "JTOTL")), "emin_mhz": _num(t, "EMIN"), "emax_mhz": _num(t, "EMAX"),
        "dtol_mhz": _num(t, "DTOL"), "monqn": monqn, "fldmin": _num(t, "FLDMIN"), "fldmax": _num(t, "FLDMAX"),
        "dfield": _num(t, "DFIELD"), "roti": roti[:3], "nmin": int(_num(t, "JMIN")), "nmax": int(_num(t, "JMAX")),
        "spin": int(_num(t, "IS")), "lmax": int(_num(t, "LMAX")), "lambda": lam,
        "iprops": int(_num(t, "IPROPS")), "ipropl": int(_num(t, "IPROPL")),
    }


def read_output():
    with open(os.path.join(REF, "examples", "output", "bound-Mg_NH.output")) as f:
        t = f.read()
    block = int(re.search(r"CALCULATIONS WILL BE FOR SYMMETRY BLOCK\s+(\d+)", t).group(1))
    nchan = max(int(m.group(1)) for m in re.finditer(r"^\s+(\d+)\s+\d+\s+\d+\s+\d+\s+-?\d+\s+\d+\s*$", t, re.M))
    sets = []
    for body in re.split(r"EFV SET\s+\d+:", t)[1:]:
        s = {
            "field": float(re.search(r"MAGNETIC Z FIELD =\s*(\S+)", body).group(1)),
            "eref_cm": float(re.search(r"REFERENCE ENERGY IS\s+(\S+) CM-1", body).group(1)),
            "eref_mhz": float(re.search(r"CM-1\s+=\s+(\S+)\s+MHZ", body).group(1)),
            "count_emin": int(re.search(r"IMPLIES\s+(\d+) STATES BELOW MINIMUM", body).group(1)),
            "count_emax": int(re.search(r"IMPLIES\s+(\d+) STATES BELOW MAXIMUM", body).group(1)),
            "states": [],
        }
        for m in re.finditer(r"CONVERGED ON STATE NUMBER\s+(\d+) AT\s+ENERGY =\s+(\S+)\s+MHZ"
                             r".*?SMALLEST EIGENVALUE OF MATCHING MATRIX IS NUMBER\s+(\d+)", body, re.S):
            s["states"].append({"state": int(m.group(1)), "energy_mhz": float(m.group(2)),
                                "eig_index": int(m.group(3))})
        sets.append(s)
    return block, nchan, sets


def read_cuts():
    with open(os.path.join(REF, "data", "pot-Mg_NH.data")) as f:
        lines = [ln.split() for ln in f if ln.strip()]
    nang = int(float(lines[0][0]))
    cuts, k = [], 1
    for _ in range(nang):
        ang, nra = float(lines[k][0]), int(lines[k][1])
        k += 1
        r, v = [], []
        for _ in range(nra):
            r.append(float(lines[k][0]))
            v.append(float(lines[k][1]))
            k += 1
        cuts.append({"angle": ang, "r": r, "e": v})
    return cuts


def read_field():
    with open(os.path.join(REF, "examples", "input", "field-Mg_NH.input")) as f:
        t = f.read()
    inp = {"rmin": _num(t, "RMIN"), "rmatch": _num(t, "RMATCH"), "rmax": _num(t, "RMAX"), "drs": _num(t, "DRS"),
           "drl": _num(t, "DRL"), "tolhil": _num(t, "TOLHIL"), "fldmin": _num(t, "FLDMIN"),
           "fldmax": _num(t, "FLDMAX"), "dtol_g": _num(t, "DTOL"),
           "energies_mhz": _list(t, "ENERGY")[: int(_num(t, "NNRG"))]}
    with open(os.path.join(REF, "examples", "output", "field-Mg_NH.output")) as f:
        o = f.read()
    inp["powrl"] = 4.0 / 3.0 if re.search(r"STEP SIZE SCALES AS R\*\*1\.33", o) else None
    per = []
    for body in re.split(r"ENERGY\s+\d+ =", o)[1:]:
        cnt = [int(x) for x in re.findall(r"IMPLIES\s+(\d+) STATES BELOW SPECIFIED ENERGY", body)]
        states = [{"state": int(m.group(1)), "field_g": float(m.group(2))} for m in
                  re.finditer(r"CONVERGED ON STATE NUMBER\s+(\d+) AT\s+MAGNETIC Z FIELD =\s+(\S+)", body)]
        per.append({"energy_mhz": float(body.split()[0]), "count_fldmin": cnt[0], "count_fldmax": cnt[1],
                    "states": states})
    return inp, per


def main():
    inp = read_input()
    block, nchan, sets = read_output()
    inp["block"] = block
    g = {"source": "examples/input/bound-Mg_NH.input, examples/output/bound-Mg_NH.output, data/pot-Mg_NH.data",
         "system": inp, "nchan": nchan, "sets": sets, "cuts": read_cuts()}
    with open(OUT, "w") as f:
        json.dump(g, f, indent=1)
    print(OUT, len(sets), "field sets,", len(g["cuts"]), "cuts")
    finp, per = read_field()
    fg = {"source": "examples/input/field-Mg_NH.input, examples/output/field-Mg_NH.output",
          "system": finp, "energies": per}
    with open(OUT_FIELD, "w") as f:
        json.dump(fg, f, indent=1)
    print(OUT_FIELD, len(per), "energies")


if __name__ == "__main__":
    main()
