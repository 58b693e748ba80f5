#!/usr/bin/env python
"""Benchmark: batched FP64 LDMD (MDPROP) propagations on B200.

Workload (one step = one pass of the hot path over the whole batch): the
atom + rigid-rotor close-coupling system (URED 4 amu, B 60 cm-1, even
j = 0..10, LJ 12-6 + anisotropic exp/R^-6 terms), JTOT = 0..80 in both
parity blocks (161 coupled-channel systems, N = 5..36) at 512 collision
energies drawn uniformly in 1-500 cm-1 (numpy default_rng(20261203 + rank)),
each propagated with MDPROP from 2.5 to 40 Angstrom in 4000 steps: 82,432
propagations per step.  Synthetic seeded inputs of that shape (there is no
published dataset for this path).

Metric: channel^3*steps/s = sum over propagations of N^3*NSTEP, divided by the
device time of the step (the whole job; max over ranks).  solves/s and the
counted FP64 rate ride along.  Multi-GPU (weak scaling): N x 512 energies,
cut into units of one block and 512 energies spread over the ranks by LPT
(molscat_b200/sharding.py), so each GPU holds about the single-GPU
workload; no collective on the data path, time = max over ranks.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "channel^3*steps/s (batched LDMD propagations, FP64)"
UNIT = "channel^3*steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--energies", type=int, default=512)
    ap.add_argument("--jmax", type=int, default=80)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="batch", choices=["batch", "serve", "large"],
                    help="batch: the batched rotor workload (default); serve: the request server under "
                         "Poisson arrivals of mixed-N solves")
    ap.add_argument("--requests", type=int, default=3000, help="serve: requests in the timed stream")
    ap.add_argument("--rate", type=float, default=None,
                    help="serve: Poisson arrival rate, requests/s (default: half the saturated capacity)")
    ap.add_argument("--nmin", type=int, default=16)
    ap.add_argument("--nmax", type=int, default=1024)
    ap.add_argument("--serve-nstep", type=int, default=1000, help="serve: steps per propagation")
    ap.add_argument("--serve-systems", type=int, default=32)
    ap.add_argument("--streams", type=int, default=4)
    ap.add_argument("--plain-sample", type=int, default=24)
    ap.add_argument("--large-n", default="256,512,1024", help="large: channel counts of the dense systems")
    ap.add_argument("--large-energies", type=int, default=64)
    ap.add_argument("--large-nstep", type=int, default=3000)
    # the serving and large-N legs of the default run (1 GPU): short, fixed sizes
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg of the default run")
    ap.add_argument("--no-large", action="store_true", help="skip the large-N leg of the default run")
    ap.add_argument("--leg-serve-requests", type=int, default=240)
    ap.add_argument("--leg-serve-nstep", type=int, default=400)
    ap.add_argument("--leg-serve-systems", type=int, default=24)
    ap.add_argument("--leg-plain-sample", type=int, default=12)
    ap.add_argument("--leg-large-n", default="512,1024")
    ap.add_argument("--leg-large-energies", type=int, default=64)
    ap.add_argument("--leg-large-nstep", type=int, default=300)
    ap.add_argument("--no-fields", action="store_true", help="skip the BOUND/FIELD field-sweep leg")
    ap.add_argument("--leg-fields", type=int, default=2048, help="fields of the alkali-pair sweep (0-1000 G)")
    ap.add_argument("--leg-field-nout", type=int, default=1800)
    ap.add_argument("--leg-field-nin", type=int, default=2400)
    return ap.parse_args()


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# CPU side: the oracle (a C restatement of the reference path) as baseline
# ----------------------------------------------------------------------------
_CPU_GRID = {}


def _cpu_grid():
    """The rotor workload's radial grid and P table (identical for every
    (JTOT, block)); built once per process."""
    if not _CPU_GRID:
        from oracle import oracle as O
        from molscat_b200 import systems as S
        sysm = S.rotor_system()
        rmin, rmax = S.ROTOR_RMIN_A / sysm.rm, S.ROTOR_RMAX_A / sysm.rm
        nstep = S.ROTOR_NSTEP
        dr = (rmax - rmin) / nstep
        rtab = O.radial_grid(rmin, dr, nstep)
        ptab = O.ptable(O.Itype1(ured=sysm.ured, be=sysm.be, jlevel=list(sysm.jlevel), lam=list(sysm.lam),
                                 terms=[list(t) for t in sysm.terms], rm=sysm.rm, epsil=sysm.epsil), rtab)
        _CPU_GRID.update(nstep=nstep, dr=dr, rtab=rtab, ptab=ptab, cm2ru=sysm.cm2ru)
    return _CPU_GRID


def _cpu_inputs(job):
    """Everything one oracle propagation of (JTOT, block, E) needs, built
    outside any timed region: the coupling arrays and the WKB start."""
    from molscat_b200 import systems as S
    jt, block, energy_cm = job
    g = _cpu_grid()
    c = S.rotor_system().coupling(jt, block)
    ered = energy_cm * g["cm2ru"]
    y0 = S.wkb_initial_y(c, g["ptab"][0], g["rtab"][0], ered)
    return (c.n, c.nham, c.vl, c.eint, c.cent, ered, y0)


def _cpu_pool_init():
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    _cpu_grid()


def _cpu_propagate(inp):
    """One oracle MDPROP propagation; returns (N^3*NSTEP, seconds, status)."""
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    from oracle import oracle as O
    n, nham, vl, eint, cent, ered, y0 = inp
    g = _cpu_grid()
    oc = O.Coupling(n=n, nham=nham, vl=vl, eint=eint, cent=cent)
    t0 = time.perf_counter()
    _, nodes, st, _ = O.mdprop(oc, g["rtab"], g["ptab"], g["nstep"], g["dr"], ered, y0)
    dt = time.perf_counter() - t0
    return n ** 3 * g["nstep"], dt, st


def cpu_sample_jobs(count: int, seed: int = 7):
    """A sample of (JTOT, block, E) from the benchmark batch, weighted like it."""
    import numpy as np
    from molscat_b200 import systems as S
    rng = np.random.default_rng(seed)
    sysm = S.rotor_system()
    blocks = [(j, b) for j in range(0, 81) for b in (1, 2) if sysm.channels(j, b)]
    e = S.batched_energies(512)
    return [(*blocks[rng.integers(len(blocks))], float(e[rng.integers(512)])) for _ in range(count)]


def cpu_baseline_serial(budget_s: float):
    """Single-thread oracle on a bounded sample of the workload (inputs built
    before each propagation is timed)."""
    from oracle import oracle as O
    O.build()
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    work = tsum = 0.0
    jobs = 0
    for job in cpu_sample_jobs(400):
        w, dt, st = _cpu_propagate(_cpu_inputs(job))
        work += w
        tsum += dt
        jobs += 1
        if tsum > budget_s:
            break
    return {"value": work / tsum, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{jobs} full 4000-step MDPROP propagations drawn from the batch, oracle C restatement "
                      f"(unpivoted SYMINV N<=30, scipy-OpenBLAS DSYTRF/DSYTRI N>30), 1 thread, {tsum:.1f} s "
                      "of propagation (coupling, P table and WKB start built outside the timed region)"}


def run_reference(args):
    """--impl reference: the reference path's CPU implementation (the oracle
    port; the Fortran reference cannot be compiled here) on all host cores.
    Each step propagates 4 x `cores` jobs sampled from the batch, handed to
    the processes one at a time;
    the inputs (couplings, P table, WKB start) are built before the timed
    region, so only the propagations and the pool's dispatch are timed."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    per_step = 4 * cores  # several jobs per process and step, dealt one at a time: balanced load
    samples = cpu_sample_jobs(per_step * (args.steps + args.warmup), seed=11)
    times = []
    work_total = 0.0
    with ctx.Pool(cores, initializer=_cpu_pool_init) as pool:
        inputs = pool.map(_cpu_inputs, samples)
        for s in range(args.warmup + args.steps):
            chunk = inputs[s * per_step:(s + 1) * per_step]
            t0 = time.perf_counter()
            res = pool.map(_cpu_propagate, chunk, chunksize=1)
            dt = time.perf_counter() - t0
            if any(r[2] != 0 for r in res):
                raise RuntimeError("oracle propagation failed")
            if s >= args.warmup:
                times.append(dt)
                work_total += sum(r[0] for r in res)
    tt = sum(times)
    value = work_total / tt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "rotor close-coupling MDPROP, 4000 steps 2.5-40 A; each step = "
                               f"{per_step} propagations sampled from the JTOT=0..80 x 2 parities x 512 energies batch",
                   "parallelism": f"{cores} host processes"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{per_step} full propagations per step, spawn pool of {cores} processes (jobs dealt one at a time), "
                                   "OpenBLAS 1 thread each; inputs built before the timed region"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
def fp64_peaks(torch):
    """Measured FP64 peaks on this GPU: cuBLAS DGEMM (burst) and our DFMA probe."""
    import ctypes
    from molscat_b200 import _lib
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3))
    del a, b
    L = _lib.load()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    fl = ctypes.c_double(0.0)
    bestp = 0.0
    for it in (200, 2000, 2000):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rc = L.mgpu_probe_fp64_fma(ctypes.c_void_p(out.data_ptr()), it, ctypes.c_void_p(st.cuda_stream),
                                   ctypes.byref(fl))
        e1.record()
        e1.synchronize()
        if rc != 0:
            break
        bestp = max(bestp, fl.value / (e0.elapsed_time(e1) * 1e-3))
    torch.cuda.empty_cache()
    return best, bestp


def load_traffic():
    """DRAM bytes per launch of the dominant step kernel (the N 33-40 bucket of
    the full workload) from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ldmd_prop_frag5_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def dominant_bucket(wl, lo=33, hi=40):
    """Systems and jobs of the N lo..hi bucket (one launch of the one-warp
    NT=5 step kernel): the same jobs, in the same order, as in the full plan."""
    import numpy as np
    keep = [s for s, c in enumerate(wl.systems) if lo <= c.n <= hi]
    remap = {s: i for i, s in enumerate(keep)}
    jobs = [j for j, s in enumerate(wl.job_sys) if s in remap]
    return ([wl.systems[s] for s in keep], [wl.segments[s] for s in keep],
            np.array([remap[wl.job_sys[j]] for j in jobs], dtype=np.int32),
            np.array([wl.job_ered[j] for j in jobs]), [wl.job_y0[j] for j in jobs])


def serve_leg(requests: int, rate: float | None, nmin: int, nmax: int, nstep: int, nsys: int, streams: int,
              plain_sample: int, seed: int = 20261203) -> dict:
    """Request server under seeded single MDPROP solves, N log-uniform in
    [nmin, nmax] over a pool of dense synthetic systems registered
    (device-resident, 2HQ(C) prepared) before the timed region.

    Two passes over fresh draws of `requests` solves: a saturated one (every
    request submitted at once) gives the capacity, then a Poisson stream at
    `rate` requests/s (None: half the measured capacity) gives the latency
    percentiles.  Beside them the plain one-solve-at-a-time GPU loop
    (mgpu_mdprop per request: plan, preparation and propagation each call) on
    the first `plain_sample` saturated requests, whose results must equal the
    served ones bit for bit."""
    import math
    import numpy as np
    from molscat_b200 import systems as S
    from molscat_b200.propagators import propagate
    from molscat_b200.serving import Server, latency_percentiles
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(nmin), math.log(nmax), nsys)).astype(int)
    pool = [S.synthetic_system(int(n), nstep, seed=1000 + k) for k, n in enumerate(ns)]
    srv = Server("LDMD", hbm_budget=48 << 30, streams=streams, max_batch=4096, max_systems=nsys)
    ids = [srv.add_system(c, seg) for (c, seg, _, _) in pool]
    for k in range(nsys):  # first use of every bucket's kernels
        srv.submit(ids[k], pool[k][2], pool[k][3]).wait()

    def stream(count, arrive):
        pick = rng.integers(0, nsys, count)
        de = rng.uniform(0.0, 10.0, count)
        t0 = time.perf_counter()
        reqs = []
        for i in range(count):
            if arrive is not None:
                while time.perf_counter() - t0 < arrive[i]:
                    pass
            k = int(pick[i])
            reqs.append(srv.submit(ids[k], pool[k][2] + de[i], pool[k][3]))
        for r in reqs:
            r.wait()
        wall = max(r.times()[2] for r in reqs) - min(r.times()[0] for r in reqs)
        work = float(sum(int(ns[int(k)]) ** 3 * nstep for k in pick))
        return reqs, pick, de, wall, work

    clocks = ClockSampler(0)
    clocks.start()
    sreqs, spick, sde, swall, swork = stream(requests, None)
    cap = requests / swall
    rate = rate or 0.5 * cap
    arrive = np.cumsum(rng.exponential(1.0 / rate, requests))
    preqs, _, _, pwall, pwork = stream(requests, arrive)
    clk = clocks.stop()
    lat = latency_percentiles(preqs, (50, 90, 99))
    lat_sat = latency_percentiles(sreqs, (50, 99))
    nplain = min(plain_sample, requests)
    same = True
    tp = time.perf_counter()
    for i in range(nplain):
        k = int(spick[i])
        c, seg, e, y0 = pool[k]
        y, nodes = propagate("LDMD", c, seg, e + sde[i], y0)
        same = same and bool(np.array_equal(y, sreqs[i].wait())) and nodes == sreqs[i].nodes
    tp = time.perf_counter() - tp
    work_plain = float(sum(int(ns[int(spick[i])]) ** 3 * nstep for i in range(nplain)))
    srv.close()
    return {
        "value": swork / swall, "unit": UNIT, "solves_per_s": cap,
        "latency_s": lat, "offered_rate_per_s": rate, "poisson_solves_per_s": requests / pwall,
        "poisson_value": pwork / pwall, "saturated_latency_s": lat_sat,
        "plain_loop": {"value": work_plain / tp, "unit": UNIT, "solves_per_s": nplain / tp,
                       "sample": f"first {nplain} saturated requests, mgpu_mdprop one at a time"},
        "served_over_plain": (swork / swall) / (work_plain / tp), "results_equal_plain": same,
        "config": {"workload": f"{requests} saturated then {requests} Poisson-arrival single MDPROP solves, "
                               f"N log-uniform {nmin}-{nmax} over {nsys} dense synthetic systems (NHAM 6), "
                               f"{nstep} steps each, energies jittered per request",
                   "streams": streams, "hbm_budget_gb": 48,
                   "registration": "systems registered and 2HQ(C) prepared before the timed region"},
        "clocks": clk,
    }


def run_serve(args):
    """--workload serve: the serving leg alone, with its own flags."""
    import torch
    from molscat_b200.build import build
    build()
    torch.cuda.set_device(0)
    from molscat_b200 import autotune
    tuned = autotune.apply(autotune.default_path("LDMD")) if os.path.exists(autotune.default_path("LDMD")) else 0
    out = serve_leg(args.requests, args.rate, args.nmin, args.nmax, args.serve_nstep, args.serve_systems,
                    args.streams, args.plain_sample)
    out["config"]["tuning"] = f"molscat_b200/tuning/ldmd.json ({tuned} N ranges off the default family)"
    line = {"metric": "channel^3*steps/s (served single MDPROP solves, mixed N)", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic", **out}
    print(json.dumps(line), flush=True)


def large_leg(ns, energies: int, nstep: int, reps: int, peak: float | None = None) -> dict:
    """Large dense N: one dense synthetic system per N (NHAM 6 Lennard-Jones
    terms, seeded), `energies` energies each, MDPROP over `nstep` steps; all
    systems in one plan (their buckets run concurrently), then each N alone.
    FP64 TFLOP/s of the propagation phase (CUDA events on the launching
    stream, 2HQ(C) prepared before) against the measured FP64 peak."""
    import numpy as np
    import torch
    from molscat_b200 import systems as S
    from molscat_b200.propagators import Plan
    sysd = [S.synthetic_system(n, nstep, seed=600 + n) for n in ns]

    def timed(idx):
        systems = [sysd[i][0] for i in idx]
        segs = [sysd[i][1] for i in idx]
        job_sys = np.repeat(np.arange(len(idx), dtype=np.int32), energies)
        job_e = np.concatenate([sysd[i][2] + np.linspace(0.0, 10.0, energies) for i in idx])
        plan = Plan("LDMD", systems, segs, job_sys, job_e)
        y0 = torch.from_numpy(plan.pack([sysd[i][3] for i in idx for _ in range(energies)])).cuda()
        y = torch.empty_like(y0)
        nd = torch.zeros(plan.njobs, dtype=torch.int32, device="cuda")
        st, kf = torch.zeros_like(nd), torch.zeros_like(nd)
        sp = torch.cuda.current_stream().cuda_stream
        y.copy_(y0)
        plan.run_device(y.data_ptr(), nd.data_ptr(), st.data_ptr(), kf.data_ptr(), sp, phases=3)
        torch.cuda.synchronize()
        if (st.cpu().numpy() != 0).any():
            raise RuntimeError("large-N propagation failed")
        ms = []
        for _ in range(max(1, reps)):
            y.copy_(y0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            plan.run_device(y.data_ptr(), nd.data_ptr(), st.data_ptr(), kf.data_ptr(), sp, phases=2)
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        t = statistics.mean(ms)
        out = {"ms": t, "tflops": plan.flops_prop / (t * 1e-3) / 1e12,
               "channel3_steps_per_s": sum(ns[i] ** 3 * nstep for i in idx) * energies / (t * 1e-3)}
        plan.close()
        del y0, y
        torch.cuda.empty_cache()
        return out

    clocks = ClockSampler(0)
    clocks.start()
    allr = timed(list(range(len(ns)))) if len(ns) > 1 else None
    alone = {str(ns[i]): timed([i]) for i in range(len(ns))}
    clk = clocks.stop()
    src = "given"
    if peak is None:
        dgemm, dfma = fp64_peaks(torch)
        peak = max(dgemm, dfma)
        src = "max(cuBLAS DGEMM 8192^3 %.1f, DFMA probe %.1f) TFLOP/s measured in this run (of measured)" % (
            dgemm / 1e12, dfma / 1e12)
    for r in ([allr] if allr else []) + list(alone.values()):
        r["frac"] = r["tflops"] * 1e12 / peak
    return {"value": (allr or alone[str(ns[0])])["tflops"], "unit": "TFLOP/s",
            "fp64_frac": (allr or alone[str(ns[0])])["frac"], "per_n": alone, "peak_tflops": peak / 1e12,
            "peak_source": src,
            "algorithmic": "2N^3 + 2 NHAM N(N+1) flops per propagation step (two Y inversions + W(B))",
            "config": {"workload": f"dense synthetic systems N={list(ns)} (NHAM 6), {energies} energies each, "
                                   f"{nstep} MDPROP steps; " + ("all N in one plan (buckets concurrent), then "
                                                               if len(ns) > 1 else "") +
                                   "each N alone; propagation phase timed (2HQ(C) prepared before)",
                       "reps": reps},
            "clocks": clk}


def field_leg(nfield: int, nout: int, nin: int, reps: int, peak: float | None = None) -> dict:
    """The BOUND/FIELD workload: the synthetic alkali pair (i = 3/2 on both
    atoms, N = 106) at E = 0 relative to its lowest threshold, counted at
    `nfield` fields in 0-1000 G.  Every field is a system; all share VL, P and
    the MDPROP U(C) preparation (the Zeeman term is a per-field EINT), so one
    plan runs 2 x nfield propagations (outward and inward) after two
    preparations.  The state count at a field is NODES_out + NODES_in + the
    non-positive eigenvalues of Y_out - Y_in; where it changes between
    neighbouring fields a bound state crosses threshold (a resonance field)."""
    import numpy as np
    import torch
    from molscat_b200.alkali import config4_sweep
    from molscat_b200.propagators import Plan
    t0 = time.perf_counter()
    sw = config4_sweep(nout=nout, nin=nin)
    fields = np.linspace(0.0, 1000.0, nfield)
    cs = [sw.coupling_at(float(f)) for f in fields]
    es = np.array([sw.ered_at(float(f)) for f in fields])
    m = nfield
    free0, total = torch.cuda.mem_get_info()
    plan = Plan("LDMD", cs + cs, [sw.seg_out] * m + [sw.seg_in] * m, np.arange(2 * m), np.concatenate([es, es]))
    free1, _ = torch.cuda.mem_get_info()

    def starts():
        # adiabatic WKB starts (yinit.f with ADIAMN), all fields in one batched eigh per end
        from molscat_b200.bound import w_matrix
        ys = []
        for seg, sgn in ((sw.seg_out, 1.0), (sw.seg_in, -1.0)):
            w = np.stack([w_matrix(c, float(seg.rtab[0]), seg.ptab[0], e) for c, e in zip(cs, es)])
            lam, vec = np.linalg.eigh(w)
            yl = np.where(lam > 0.0, sgn * np.sqrt(np.abs(lam)), 0.0)
            ys += list(np.einsum("fij,fj,fkj->fik", vec, yl, vec))
        return ys

    def counts_host(ybuf, nodes):
        yo = np.stack([plan.unpack(ybuf, k) for k in range(m)])
        yi = np.stack([plan.unpack(ybuf, m + k) for k in range(m)])
        ev = np.linalg.eigvalsh(yo - yi)
        return nodes[:m].astype(np.int64) + nodes[m:] + np.sum(ev <= 0.0, axis=1)

    pairs = np.stack([np.arange(m), np.arange(m, 2 * m)], axis=1)

    def counts_device(ybuf, nodes):
        mc = plan.match_counts(pairs).astype(np.int64)
        for k in np.nonzero(mc < 0)[0]:  # a zero pivot: count from the eigenvalues
            mc[k] = int(np.sum(np.linalg.eigvalsh(plan.unpack(ybuf, k) - plan.unpack(ybuf, m + k)) <= 0.0))
        return nodes[:m].astype(np.int64) + nodes[m:] + mc

    y0 = plan.pack(starts())
    t_setup = time.perf_counter() - t0
    dev = torch.device("cuda:0")
    y0d = torch.from_numpy(y0).to(dev)
    y = torch.empty_like(y0d)
    nd = torch.zeros(2 * m, dtype=torch.int32, device=dev)
    st, kf = torch.zeros_like(nd), torch.zeros_like(nd)
    sp = torch.cuda.current_stream().cuda_stream
    y.copy_(y0d)
    plan.run_device(y.data_ptr(), nd.data_ptr(), st.data_ptr(), kf.data_ptr(), sp, phases=3)
    torch.cuda.synchronize()
    if (st.cpu().numpy() != 0).any():
        raise RuntimeError("field-sweep propagation failed")
    clocks = ClockSampler(0)
    clocks.start()
    prep, prop = [], []
    for _ in range(max(1, reps)):
        y.copy_(y0d)
        a0, a1, a2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a0.record()
        plan.run_device(y.data_ptr(), nd.data_ptr(), st.data_ptr(), kf.data_ptr(), sp, phases=1)
        a1.record()
        plan.run_device(y.data_ptr(), nd.data_ptr(), st.data_ptr(), kf.data_ptr(), sp, phases=2)
        a2.record()
        a2.synchronize()
        prep.append(a0.elapsed_time(a1))
        prop.append(a1.elapsed_time(a2))
    clk = clocks.stop()
    # end to end through the C ABI with host buffers, then the matching on the host
    ta = time.perf_counter()
    ybuf, nodes, status, _ = plan.run_host(y0)
    tb = time.perf_counter()
    cnt = counts_device(ybuf, nodes)
    tc = time.perf_counter()
    if (status != 0).any():
        raise RuntimeError("field-sweep propagation failed")
    th = time.perf_counter()
    cnt_host = counts_host(ybuf, nodes)
    t_host_match = time.perf_counter() - th
    steps = [(f, int(cnt[k]), int(cnt[k + 1])) for k, f in enumerate(fields[:-1]) if cnt[k] != cnt[k + 1]]
    t_prep, t_prop = statistics.mean(prep), statistics.mean(prop)
    work = float(m) * sw.n ** 3 * (nout + nin)
    tfl = plan.flops_prop / (t_prop * 1e-3) / 1e12
    out = {"fields": m, "n": sw.n, "propagations": 2 * m, "shared_systems": plan.shared_systems,
           "device_gb": {"free_before_plan": free0 / 1e9, "plan": (free0 - free1) / 1e9, "total": total / 1e9},
           "prep_ms": t_prep, "prop_ms": t_prop, "fields_per_s": m / ((t_prep + t_prop) * 1e-3),
           "channel3_steps_per_s": work / ((t_prep + t_prop) * 1e-3), "prop_tflops": tfl,
           "prop_frac": (tfl * 1e12 / peak) if peak else None,
           "e2e": {"s": tc - ta, "run_host_s": tb - ta, "matching_s": tc - tb, "fields_per_s": m / (tc - ta),
                   "h2d_bytes": int(plan.y_elems * 8), "d2h_bytes": int(plan.y_elems * 8 + 3 * 4 * 2 * m),
                   "api": "mgpu_plan_run_host, then mgpu_plan_match_counts (LDL^T inertia of Y_out - Y_in on "
                          "the device)"},
           "matching_host_eigvalsh_s": t_host_match, "device_counts_equal_host": bool(np.array_equal(cnt, cnt_host)),
           "count_range": [int(cnt.min()), int(cnt.max())], "crossings": len(steps),
           "first_crossings_g": [round(float(f), 3) for f, _, _ in steps[:8]],
           "setup_s": t_setup, "clocks": clk,
           "config": {"workload": "alkali pair in the uncoupled basis (base9-alk_alk_ucpld form), s = 1/2, i = 3/2 "
                                  "on both atoms, hyperfine 1.0 / 0.8 GHz, L <= 4, MTOT = 2 (M_F), even L: N = %d; "
                                  "Morse singlet/triplet (De 3900/240 cm-1, Re 4.2/6.0 A) with damped -C6/R^6, "
                                  "C6 = 4700 Eh a0^6; E = 0 at the lowest threshold; %d fields 0-1000 G; MDPROP "
                                  "3 -> 12 A (%d steps) and 60 -> 12 A (%d steps)" % (sw.n, m, nout, nin)}}
    plan.close()
    del y0d, y
    torch.cuda.empty_cache()
    return out


def run_large(args):
    """--workload large: the large-N leg alone, with its own flags."""
    import torch
    from molscat_b200.build import build
    build()
    torch.cuda.set_device(0)
    ns = [int(x) for x in args.large_n.split(",")]
    out = large_leg(ns, args.large_energies, args.large_nstep, args.steps)
    line = {"metric": "FP64 TFLOP/s (batched large-N MDPROP propagation)", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic", **out}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return
    if args.workload == "large":
        run_large(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    # CPU baseline first (rank 0, N=1): before CUDA is initialised
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_serial(args.cpu_seconds)

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from molscat_b200.build import build
    if rank == 0:
        build()
    if dist:
        dist.barrier()
    from molscat_b200 import systems as S
    from molscat_b200 import autotune
    from molscat_b200.propagators import Plan
    tpath = autotune.default_path("LDMD")
    tuned = autotune.apply(tpath) if os.path.exists(tpath) else 0

    t_setup = time.perf_counter()
    if world > 1:
        # weak scaling through the sharding path: world x 512 energies, LPT units of one block and 512 energies
        wl = S.batched_workload_shard(rank, world, n_energies=args.energies, jmax=args.jmax)
    else:
        wl = S.batched_workload(n_energies=args.energies, jmax=args.jmax)
    plan = Plan("LDMD", wl.systems, wl.segments, wl.job_sys, wl.job_ered)
    y0_host = plan.pack(wl.job_y0)
    t_setup = time.perf_counter() - t_setup
    work = wl.channel3_steps()
    njobs = wl.njobs

    dev = torch.device("cuda", local)
    y0_dev = torch.from_numpy(y0_host).to(dev)
    y_dev = torch.empty_like(y0_dev)
    nodes = torch.zeros(njobs, dtype=torch.int32, device=dev)
    status = torch.zeros(njobs, dtype=torch.int32, device=dev)
    kfail = torch.zeros(njobs, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    ev = []

    def step(record=False):
        y_dev.copy_(y0_dev)
        if record:
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(stream)
            plan.run_device(y_dev.data_ptr(), nodes.data_ptr(), status.data_ptr(), kfail.data_ptr(), sp, phases=1)
            e[1].record(stream)
            plan.run_device(y_dev.data_ptr(), nodes.data_ptr(), status.data_ptr(), kfail.data_ptr(), sp, phases=2)
            e[2].record(stream)
            ev.append(e)
        else:
            plan.run_device(y_dev.data_ptr(), nodes.data_ptr(), status.data_ptr(), kfail.data_ptr(), sp)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    st = status.cpu().numpy()
    if (st != 0).any():
        raise RuntimeError(f"{int((st != 0).sum())} propagations failed (first status {int(st[st != 0][0])})")

    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        step(record=True)
    t1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms_local = t0.elapsed_time(t1) / args.steps
    prep_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in ev)
    prop_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in ev)
    ms = ms_local
    if dist:
        t = torch.tensor([ms_local], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        wt = torch.tensor([work, float(njobs)], dtype=torch.float64, device=dev)
        dist.all_reduce(wt)
        work_all, jobs_all = float(wt[0].item()), float(wt[1].item())
    else:
        work_all, jobs_all = work, float(njobs)

    # end to end through the C ABI with host buffers: initial Y in, the
    # propagation and Y -> K -> S on the device, S matrices, NODES, status out
    e2e = None
    if not args.no_e2e:
        k2 = args.e2e_steps or args.steps
        plan.run_host_smatrix(y0_host)  # warm
        times = []
        s_elems = 0
        for _ in range(k2):
            if dist:
                dist.barrier()
            ta = time.perf_counter()
            sr, si, nd, stt, kf = plan.run_host_smatrix(y0_host)
            times.append(time.perf_counter() - ta)
            s_elems = sr.size
            if (stt != 0).any():
                raise RuntimeError("e2e propagation failed")
        tm = statistics.mean(times)
        if dist:
            t = torch.tensor([tm], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tm = float(t.item())
        e2e = {"value": work_all / tm, "unit": UNIT, "h2d_bytes_per_step": int(plan.y_elems * 8),
               "d2h_bytes_per_step": int(2 * s_elems * 8 + 3 * 4 * njobs), "solves_per_s": jobs_all / tm,
               "api": "mgpu_plan_run_host_smatrix (C ABI, host buffers; S matrices computed on the device)"}

    # the dominant kernel alone: the N 33-40 bucket's step launch, timed with
    # CUDA events on the stream it is launched on (prep run once before)
    dom = None
    if rank == 0:
        ds, dg, dj, de, dy = dominant_bucket(wl)
        dplan = Plan("LDMD", ds, dg, dj, de)
        dy0 = torch.from_numpy(dplan.pack(dy)).to(dev)
        dyw = torch.empty_like(dy0)
        dn = torch.zeros(dplan.njobs, dtype=torch.int32, device=dev)
        dst, dkf = torch.zeros_like(dn), torch.zeros_like(dn)
        dyw.copy_(dy0)
        dplan.run_device(dyw.data_ptr(), dn.data_ptr(), dst.data_ptr(), dkf.data_ptr(), sp, phases=1)
        times = []
        for _ in range(3):
            dyw.copy_(dy0)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            dplan.run_device(dyw.data_ptr(), dn.data_ptr(), dst.data_ptr(), dkf.data_ptr(), sp, phases=2)
            a1.record(stream)
            a1.synchronize()
            times.append(a0.elapsed_time(a1))
        if (dst.cpu().numpy() != 0).any():
            raise RuntimeError("dominant-bucket propagation failed")
        dom = {"jobs": dplan.njobs, "ms": statistics.mean(times), "flops": dplan.flops_prop,
               "launches": dplan.launches}
        del dy0, dyw
        dplan.close()

    dgemm, dfma = (fp64_peaks(torch) if rank == 0 else (None, None))
    peak = max(dgemm or 0.0, dfma or 0.0) or None
    achieved = dom["flops"] / (dom["ms"] * 1e-3) if dom else None
    achieved_phase = plan.flops_prop / (prop_ms * 1e-3)
    traffic = load_traffic()
    if rank == 0:
        line = {
            "metric": METRIC, "value": work_all / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "rotor close-coupling (ITYPE=1 style) MDPROP: JTOT=0..%d x 2 parities x %d energies "
                                   "(1-500 cm-1), 4000 steps 2.5-40 A, N=5..36" % (args.jmax, args.energies),
                       "systems": len(wl.systems), "propagations_per_gpu": njobs,
                       "l2": "inputs larger than L2 (2HQ(C) and coupling-sum tables %.1f GB)" % (
                           2 * sum(512 * (((s.n + 7) // 8) * ((s.n + 7) // 8 + 1) // 2) * 4000 for s in wl.systems)
                           / 1e9),
                       "parallelism": ("LPT shards of (block, 512 energies) units over %d GPUs, no collective on the "
                                       "data path" % world) if world > 1 else "1 GPU",
                       "tuning": f"molscat_b200/tuning/ldmd.json ({tuned} N ranges off the default family)"},
            "solves_per_s": jobs_all / (ms * 1e-3),
            "flops_counted_per_s": plan.flops * world / (ms * 1e-3),
            "gpu_launches": plan.launches * args.steps,
            "clocks": clk,
            "roofline": {"bound": "fp64", "kernel": "ldmd_prop_frag_kernel<5> (one warp per matrix, N 33-40 bucket, "
                                                    "%d propagations x 4000 steps per launch)" % (dom["jobs"] if dom else 0),
                         "achieved": (achieved or 0) / 1e12,
                         "peak": (peak or 0) / 1e12, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if (peak and achieved) else None,
                         "traffic": (traffic or {}).get("bytes_per_launch"),
                         "launch_ms": dom["ms"] if dom else None,
                         "peak_source": "max(cuBLAS DGEMM 8192^3, DFMA probe) measured in this run: "
                                        "dgemm %.1f, dfma %.1f TFLOP/s (of measured)" % ((dgemm or 0) / 1e12, (dfma or 0) / 1e12),
                         "algorithmic": "2N^3 + 2 NHAM N(N+1) flops per propagation step (two Y inversions + W(B)); "
                                        "the energy-independent U(C) inversion is the prep kernel, timed apart",
                         "step_phase_all_buckets_tflops": achieved_phase / 1e12,
                         "prop_ms": prop_ms, "prep_ms": prep_ms},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "setup_s": t_setup,
        }
    plan.close()
    del y0_dev, y_dev
    torch.cuda.empty_cache()
    if rank == 0 and world == 1:
        # the rest of the metric: served mixed-N solves (capacity, p50/p99
        # latency, against the plain one-at-a-time loop) and large dense N
        if not args.no_serve:
            line["serving"] = serve_leg(args.leg_serve_requests, None, 16, 1024, args.leg_serve_nstep,
                                        args.leg_serve_systems, args.streams, args.leg_plain_sample)
        if not args.no_large:
            ns = [int(x) for x in args.leg_large_n.split(",")]
            line["large_n"] = large_leg(ns, args.leg_large_energies, args.leg_large_nstep, 2, peak=peak)
            line["large_n"]["peak_source"] = line["roofline"]["peak_source"]
        if not args.no_fields:
            try:
                line["field_sweep"] = field_leg(args.leg_fields, args.leg_field_nout, args.leg_field_nin, 2,
                                                peak=peak)
            except Exception as err:  # the headline line is still printed; the leg reports why it failed
                free, total = torch.cuda.mem_get_info()
                line["field_sweep"] = {"error": f"{type(err).__name__}: {err}",
                                       "device_free_gb": free / 1e9, "device_total_gb": total / 1e9}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
