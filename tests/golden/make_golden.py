"""Extract golden S matrices and bound-state energies from the reference's
example outputs.

Run with the reference project's checkout named by $MOLSCAT_REF (required):

    MOLSCAT_REF=<path to molscat checkout> python tests/golden/make_golden.py

writes tests/golden/molscat_all_propagators.json,
tests/golden/bound_basic1.json, tests/golden/bound_ar_ch4.json and
tests/golden/molscat_ityp6.json.  The fixtures are committed, so nothing at
test time reads the reference tree.

Bound states: examples/output/bound-basic1.output (the same model system,
JTOT=1, symmetry block 2, MDPROP outward RMIN=0.5 -> RMATCH=1.0 and inward
RMAX=20 -> RMATCH, DR=0.001, states between -10 and -1 cm-1), input
examples/input/bound-basic1.input.

Source: examples/output/molscat-all_propagators.output, runs
"IPROPS=5" (LDPROP, lines 408-537), "IPROPS=6" (MDPROP, lines 682-811) and
"IPROPS=8" (MGPROP with IMGSEL=5, the six-step MA5 method, lines 1231-1358)
and "IPROPS=7" (MAPROP, the quasi-adiabatic log-derivative propagator,
lines 956-1084):
ITYPE=1, JTOT=10, symmetry block 1, N=12, E=1000 and 900 cm-1, 8072 steps.
The system definition is examples/input/molscat-all_propagators.input:25-71.
"""
import json
import os
import re
import sys

REF = os.environ.get("MOLSCAT_REF")
if not REF:
    sys.exit("set MOLSCAT_REF to the reference project's checkout")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "molscat_all_propagators.json")
OUT_BOUND = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bound_basic1.json")
OUT_ARCH4 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bound_ar_ch4.json")
OUT_ITYP6 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "molscat_ityp6.json")
ITYP6_JTOTS = (0, 1, 2, 5, 10, 20, 30, 40, 60, 80)


def parse_runs(text):
    runs = {}
    sections = re.split(r"=+ model system: ITYPE=1; (IPROPS=[^=]*?) =+", text)
    # sections: [pre, label1, body1, label2, body2, ...]
    for label, body in zip(sections[1::2], sections[2::2]):
        label = label.strip()
        blocks = []
        for m in re.finditer(r"ROW  COL.*?\n((?:\s+\d+\s+\d+\s+\S+\s+\S+\s+\S+\s+\S+\n)+)", body):
            entries = []
            for line in m.group(1).strip("\n").split("\n"):
                f = line.split()
                entries.append((int(f[0]), int(f[1]), float(f[4]), float(f[5])))
            blocks.append(entries)
        steps = [int(x) for x in re.findall(r"PROPAGATED FROM\s+\S+\s+TO\s+\S+\s+IN\s+(\d+)\s+STEPS", body)]
        runs[label] = {"smatrices": blocks, "nstep": steps}
    return runs


def main():
    path = os.path.join(REF, "examples", "output", "molscat-all_propagators.output")
    with open(path) as f:
        runs = parse_runs(f.read())
    sel = {}
    for label, key in (("IPROPS=6", "LDMD"), ("IPROPS=5", "LDJ"), ("IPROPS=8", "LDMG"), ("IPROPS=7", "LDMA")):
        r = runs[label]
        sel[key] = {
            "energies_cm": [1000.0, 900.0],
            "nstep": r["nstep"][:2],
            "smatrix": [
                [{"row": a, "col": b, "re": c, "im": d} for (a, b, c, d) in blk]
                for blk in r["smatrices"][:2]
            ],
        }
    doc = {
        "source": "examples/output/molscat-all_propagators.output (IPROPS=6 lines 682-811, IPROPS=5 lines 408-537, "
                  "IPROPS=8 with IMGSEL=5 lines 1231-1358, IPROPS=7 lines 956-1084)",
        "system": {
            "itype": 1, "ured": 20.0, "be": 30.0, "jlevel": [0, 2, 4, 6],
            "lambda": [0, 2], "terms": [[[1.0, -12, None], [-2.0, -6, None]], [[-0.2, -6, None]]],
            "rm": 3.5, "epsil": 50.0, "jtot": 10, "block": 1,
            "rmin": 0.5, "rmax": 20.0, "steps": 12.0, "irmset": 9, "iscru": True,
        },
        "runs": sel,
    }
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT, file=sys.stderr)


def main_bound():
    path = os.path.join(REF, "examples", "output", "bound-basic1.output")
    with open(path) as f:
        text = f.read()
    states = [{"state": int(a), "energy_cm": float(b)} for a, b in
              re.findall(r"CONVERGED ON STATE NUMBER\s+(\d+)\s+AT\s+ENERGY =\s+(\S+)\s+CM-1", text)]
    doc = {
        "source": "examples/output/bound-basic1.output (converged states), examples/input/bound-basic1.input",
        "system": {
            "itype": 1, "ured": 20.0, "be": 30.0, "jlevel": [0, 2, 4, 6],
            "lambda": [0, 2], "terms": [[[1.0, -12, None], [-2.0, -6, None]], [[-0.2, -6, None]]],
            "rm": 3.5, "epsil": 50.0, "jtot": 1, "block": 2,
            "rmin": 0.5, "rmatch": 1.0, "rmax": 20.0, "dr": 0.001, "emin_cm": -10.0, "emax_cm": -1.0,
            "convergence_cm": 1.0e-7,
        },
        "states": states,
    }
    with open(OUT_BOUND, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT_BOUND, file=sys.stderr)


def main_ar_ch4():
    """bound-Ar_CH4: ITYPE=6 (CH4 as a spherical top with centrifugal
    distortion, the MSV potential of Buck et al. through its VSTAR plug-in),
    JTOT=1 block 2, MDPROP outward from RMIN (IRMSET=8) to RMATCH and inward
    from RMAX, DR=0.01.  The system is read from the input file: the &BASIS
    and &POTL values and the five VINIT data lines."""
    with open(os.path.join(REF, "examples", "input", "bound-Ar_CH4.input")) as f:
        inp = f.read()

    def num(name):
        return float(re.search(name + r"\s*=\s*([-+0-9.Ee]+)", inp).group(1))

    roti = [float(x) for x in re.search(r"ROTI\s*=\s*(.*?)JMAX", inp, re.S).group(1)
            .replace(",", " ").split()]
    lam = [int(x) for x in re.search(r"LAMBDA\s*=\s*([0-9, ]+)", inp).group(1).replace(",", " ").split()]
    mxlam = int(num("MXLAM"))
    data = [[float(x) for x in ln.split()] for ln in inp.split("/")[-1].strip().splitlines()]
    with open(os.path.join(REF, "examples", "output", "bound-Ar_CH4.output")) as f:
        text = f.read()
    pairs = [{"state": int(m[0]), "j": int(m[1]), "tau": int(m[2]), "prty": int(m[3]), "energy_cm": float(m[7])}
             for m in re.findall(r"^\s+(\d+)\s+(\d+)\s+(-?\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\S+)\s*$",
                                 text.split("PAIR STATE    ---")[1].split("=====")[0], re.M)]
    # CHANNEL, PAIR STATE, J, TAU, PRTY, two more state numbers, L, PAIR LEVEL, PAIR ENERGY
    chans = [(int(m[1]), int(m[7])) for m in re.findall(
        r"^\s+(\d+)\s+(\d+)\s+(\d+)\s+(-?\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+(\S+)\s*$",
        text.split("CHANNEL FUNCTION LIST:")[1].split("NODE COUNT")[0], re.M)]
    states = [{"state": int(a), "energy_cm": float(b)} for a, b in
              re.findall(r"CONVERGED ON STATE NUMBER\s+(\d+)\s+AT\s+ENERGY =\s+(\S+)\s+CM-1", text)]
    doc = {
        "source": "examples/input/bound-Ar_CH4.input, examples/output/bound-Ar_CH4.output (pair states, "
                  "channel list, converged states)",
        "system": {
            "itype": 6, "ured": num("URED"), "roti": roti, "jmax": int(num("JMAX")), "isym": int(num("ISYM")),
            "lambda": [[lam[2 * i], lam[2 * i + 1]] for i in range(mxlam)],
            "epsil": data[0][0], "rm": data[0][1], "beta": data[1], "c6c8": data[2], "x1234": data[3],
            "alphas": data[4:4 + mxlam - 1],
            "jtot": int(num("JTOTL")), "block": int(num("IBFIX")), "rmin": num("RMIN"), "rmatch": num("RMATCH"),
            "rmax": num("RMAX"), "dr": num("DR"), "irmset": int(num("IRMSET")), "emin_cm": num("EMIN"),
            "emax_cm": num("EMAX"), "convergence_cm": 1.0e-7,
        },
        "pair_states": pairs,
        "channels": [{"pair_state": a, "l": b} for a, b in chans],
        "states": states,
    }
    with open(OUT_ARCH4, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT_ARCH4, file=sys.stderr)


def main_ityp6():
    """molscat-ityp6: ITYPE=6 spherical top (as bound-Ar_CH4 but ISYM=224,
    JMAX=9), LDMD from RMIN (IRMSET=8) to RMID = 1.3 x RTURN, AIRY from RMID
    to RMAX (TOLHI=1e-4), one energy (300 cm-1); the printed state-to-state
    partial cross sections of the JTOT values in ITYP6_JTOTS, both blocks."""
    with open(os.path.join(REF, "examples", "input", "molscat-ityp6.input")) as f:
        inp = f.read()

    def num(name):
        return float(re.search(r"\b" + name + r"\s*=\s*([-+0-9.Ee]+)", inp).group(1))

    roti = [float(x) for x in re.search(r"ROTI\s*=\s*(.*?)JMAX", inp, re.S).group(1).replace(",", " ").split()]
    lam = [int(x) for x in re.search(r"LAMBDA\s*=\s*([0-9, ]+)", inp).group(1).replace(",", " ").split()]
    mxlam = int(num("MXLAM"))
    data = [[float(x) for x in ln.split()] for ln in inp.split("/")[-1].strip().splitlines()]
    with open(os.path.join(REF, "examples", "output", "molscat-ityp6.output")) as f:
        text = f.read()
    blocks = []
    parts = re.split(r"ANGULAR MOMENTUM JTOT\s*=\s*(\d+)\s+AND SYMMETRY BLOCK\s*=\s*(\d+)", text)
    for jt, blk, body in zip(parts[1::3], parts[2::3], parts[3::3]):
        if int(jt) not in ITYP6_JTOTS:
            continue
        tab = body.split("FOR JTOT =")[1] if "PARTIAL CROSS SECTIONS" in body else ""
        m = re.search(r"F\s+I =([\d ]+)\n((?:\s+\d+(?:\s+\S+E[-+]\d+)+\n)+)", tab)
        if not m:
            continue
        levels = [int(x) for x in m.group(1).split()]
        rows = [ln.split() for ln in m.group(2).strip("\n").split("\n")]
        sig = [{"final": int(r[0]), "initial": levels[k], "sigma": float(v)}
               for r in rows for k, v in enumerate(r[1:])]
        blocks.append({"jtot": int(jt), "block": int(blk), "sigma": sig})
    doc = {
        "source": "examples/input/molscat-ityp6.input, examples/output/molscat-ityp6.output (state-to-state "
                  "partial cross sections)",
        "system": {
            "itype": 6, "ured": num("URED"), "roti": roti, "jmax": int(num("JMAX")), "isym": int(num("ISYM")),
            "lambda": [[lam[2 * i], lam[2 * i + 1]] for i in range(mxlam)],
            "epsil": data[0][0], "rm": data[0][1], "beta": data[1], "c6c8": data[2], "x1234": data[3],
            "alphas": data[4:4 + mxlam - 1], "rmin": num("RMIN"), "rmax": num("RMAX"), "steps": num("STEPS"),
            "irmset": int(num("IRMSET")), "rvfac": num("RVFAC"), "tolhi": num("TOLHI"), "energy_cm": num("ENERGY"),
        },
        "blocks": blocks,
    }
    with open(OUT_ITYP6, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT_ITYP6, file=sys.stderr)


if __name__ == "__main__":
    main()
    main_bound()
    main_ar_ch4()
    main_ityp6()
