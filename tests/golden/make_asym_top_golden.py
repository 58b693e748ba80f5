"""Oracle results for the large-N parity tests on the physical asymmetric-top
basis (tests/cases.py: asym_top_case), too slow to recompute in a test:

    python tests/golden/make_asym_top_golden.py

writes tests/golden/asym_top_large_n.json.  For each block (N = 256 over the
full 3000 steps, N = 500 and 1024 over 1000 steps; 2.8 -> 30 Angstrom, E =
150 cm-1) the oracle's MDPROP gives NODES, the diagonal and the first column
of Y(RSTOP), its Frobenius norm, NOPEN and the first four columns of the S
matrix (YTOK + KTOS in CHNSRT order).  The oracle's ITYPE=6 basis and
couplings (oracle/itype6.py) are pinned separately by the reference's
bound-Ar_CH4 example."""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

import cases  # noqa: E402
from oracle import oracle as O  # noqa: E402

RUNS = ((256, 3000), (512, 1000), (1024, 1000))
E_CM = 150.0


def main():
    out = {"energy_cm": E_CM, "runs": []}
    for n_target, nstep in RUNS:
        t0 = time.time()
        c, seg, jobs, sysm = cases.asym_top_case(n_target, nstep, (E_CM,))
        ered, y0 = jobs[0]
        y, nodes, st, kf = O.mdprop(cases.to_oracle(c), seg.rtab, seg.ptab, seg.nstep, seg.dr, ered, y0)
        assert st == 0, (st, kf)
        sr, si, nopen = cases.smatrix(c, y, float(seg.rtab[-1]), ered)
        m = min(4, nopen)
        out["runs"].append({
            "n_target": n_target, "n": c.n, "nstep": nstep, "ered": ered, "nodes": int(nodes), "nopen": int(nopen),
            "y_diag": np.diag(y).tolist(), "y_col0": y[:, 0].tolist(), "y_fro": float(np.linalg.norm(y)),
            "sr_cols": sr[:, :m].T.tolist(), "si_cols": si[:, :m].T.tolist()})
        print(f"N={c.n} NSTEP={nstep} NODES={nodes} NOPEN={nopen} {time.time() - t0:.0f} s", flush=True)
    with open(os.path.join(HERE, "asym_top_large_n.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
