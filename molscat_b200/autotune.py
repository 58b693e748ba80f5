"""Per-N-bucket kernel family choice by measurement.

For every N range of the bucket table the tuner times each kernel family
that can hold it on a representative batch (a dense synthetic system of the
range's largest N, many energies) and keeps the fastest:

    0  the default order: one warp per matrix (N <= 40), one CTA per matrix
       (N <= 200), the batched large-N kernels above
    1  4x4 register tiles with the scalar sweep (N <= 64)
    2  the batched large-N kernels (matrices in global memory, 64 pivots a
       round) at any N

    python -m molscat_b200.autotune [--prop LDMD] [--out molscat_b200/tuning/ldmd.json]

One family at one N, timed once (the case a profiler capture is taken on):

    python -m molscat_b200.autotune --one 106 --family 0 --jobs 1024 --nstep 50

`apply(path)` hands the saved choices to the library
(mgpu_set_family_for_n); plans created afterwards use them.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
# (lo, hi) ranges: the edges of the default buckets up to N = 200
RANGES = [(1, 8), (9, 16), (17, 24), (25, 32), (33, 40), (41, 48), (49, 56), (57, 64), (65, 80), (81, 96),
          (97, 112), (113, 128), (129, 160), (161, 200)]


def candidates(hi: int, prop: str) -> list:
    fams = [_lib.FAMILY_DMMA]
    if hi <= 64:
        fams.append(_lib.FAMILY_TILE4)
    if hi > 40:
        fams.append(_lib.FAMILY_BIG)
    return fams


def measure(n: int, prop: str, family: int, njobs: int, nstep: int, seed: int = 11) -> float:
    """Propagation-phase TFLOP/s of one family on njobs energies of one system."""
    import torch
    from .propagators import Plan
    from .systems import synthetic_system
    _lib.set_family_for_n(-1, -1, -1, prop)
    _lib.set_family_for_n(n, n, family, prop)
    try:
        c, seg, ered, y0 = synthetic_system(n, nstep, seed=seed)
        eds = ered + np.linspace(0.0, 10.0, njobs)
        plan = Plan(prop, [c], [seg], np.zeros(njobs, dtype=np.int32), eds)
    finally:
        _lib.set_family_for_n(-1, -1, -1, prop)
    try:
        y0d = torch.from_numpy(plan.pack([y0] * njobs)).cuda()
        y = torch.empty_like(y0d)
        nd = torch.zeros(njobs, dtype=torch.int32, device="cuda")
        st, kf = torch.zeros_like(nd), torch.zeros_like(nd)
        sp = torch.cuda.current_stream().cuda_stream

        def run(ph):
            y.copy_(y0d)
            plan.run_device(y.data_ptr(), nd.data_ptr(), st.data_ptr(), kf.data_ptr(), sp, phases=ph)

        run(3)
        torch.cuda.synchronize()
        if (st.cpu().numpy() != 0).any():
            return 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run(2)
        e1.record()
        torch.cuda.synchronize()
        return plan.flops_prop / (e0.elapsed_time(e1) * 1e-3) / 1e12
    finally:
        plan.close()


def tune(prop: str = "LDMD", njobs_small: int = 1024, njobs_large: int = 128, nstep: int = 100) -> dict:
    import torch
    table = []
    for lo, hi in RANGES:
        njobs = njobs_small if hi <= 64 else njobs_large
        res = {f: measure(hi, prop, f, njobs, nstep) for f in candidates(hi, prop)}
        best = max(res, key=res.get)
        table.append({"lo": lo, "hi": hi, "family": int(best), "tflops": {str(k): v for k, v in res.items()},
                      "jobs": njobs})
    return {"device": torch.cuda.get_device_name(0), "prop": prop, "nstep": nstep,
            "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()), "ranges": table}


def apply(path: str) -> int:
    """Hand a saved table's choices to the library; returns how many ranges differ from the default."""
    with open(path) as f:
        t = json.load(f)
    prop = t["prop"]
    _lib.set_family_for_n(-1, -1, -1, prop)
    changed = 0
    for r in t["ranges"]:
        if r["family"] != _lib.FAMILY_DMMA:
            _lib.set_family_for_n(r["lo"], r["hi"], r["family"], prop)
            changed += 1
    return changed


def default_path(prop: str) -> str:
    return os.path.join(HERE, "tuning", f"{prop.lower()}.json")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--prop", default="LDMD", choices=["LDMD", "LDJ"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--nstep", type=int, default=100)
    ap.add_argument("--one", type=int, default=0, help="time one family at this N and print TFLOP/s")
    ap.add_argument("--family", type=int, default=_lib.FAMILY_DMMA)
    ap.add_argument("--jobs", type=int, default=1024)
    a = ap.parse_args()
    from .build import build
    build()
    if a.one:
        tf = measure(a.one, a.prop, a.family, a.jobs, a.nstep)
        print(json.dumps({"n": a.one, "family": a.family, "jobs": a.jobs, "nstep": a.nstep, "tflops": tf}))
        if tf <= 0.0:
            raise SystemExit("propagation reported a non-zero status")
        return
    t = tune(a.prop, nstep=a.nstep)
    out = a.out or default_path(a.prop)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as f:
        json.dump(t, f, indent=1)
    for r in t["ranges"]:
        print(f"N {r['lo']:4d}-{r['hi']:4d}: family {r['family']}  " +
              "  ".join(f"{k}:{v:.2f}" for k, v in r["tflops"].items()))
    print(out)


if __name__ == "__main__":
    main()
