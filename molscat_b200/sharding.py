"""Independent propagations spread over ranks (one process per GPU).

The units of a MOLSCAT run are independent: every (JTOT, parity block,
energy) propagation is its own MDPROP call (mol.driver.f:1181-1855 loops over
them).  They are grouped by coupled-channel block so that all energies of one
block stay on one rank and share the block's energy-independent 2HQ(C) table
(the energy reuse of mdprop.f:77-87).  Blocks go to ranks by the LPT rule
(longest first onto the least-loaded rank) with cost N^3 * NSTEP * energies.

There is no collective on the data path: each rank propagates its own blocks
and the per-job results (Y, NODES, status) are gathered once at the end.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable

import numpy as np

from .systems import Workload


def block_costs(wl: Workload) -> np.ndarray:
    """N^3 * NSTEP summed over the energies of each system (block)."""
    cost = np.zeros(len(wl.systems))
    for s in wl.job_sys:
        cost[s] += float(wl.systems[s].n) ** 3 * wl.segments[s].nstep
    return cost


def lpt_partition(costs, world: int) -> list:
    """Indices of `costs` per rank: longest processing time first, each unit
    onto the currently least-loaded rank (ties: lowest rank, then input order)."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = np.zeros(world)
    parts = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += costs[i]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


@dataclass
class Shard:
    workload: Workload   # this rank's systems and jobs (renumbered)
    jobs: np.ndarray     # global job index of each local job
    systems: np.ndarray  # global system index of each local system


def shard(wl: Workload, rank: int, world: int) -> Shard:
    """This rank's part of `wl`: whole blocks, jobs in their global order."""
    mine = lpt_partition(block_costs(wl), world)[rank]
    remap = {int(s): i for i, s in enumerate(mine)}
    jobs = np.array([j for j, s in enumerate(wl.job_sys) if int(s) in remap], dtype=np.int64)
    sub = Workload(name=f"{wl.name} [rank {rank}/{world}]",
                   systems=[wl.systems[s] for s in mine], segments=[wl.segments[s] for s in mine],
                   job_sys=np.array([remap[int(wl.job_sys[j])] for j in jobs], dtype=np.int32),
                   job_ered=np.array([wl.job_ered[j] for j in jobs]), job_y0=[wl.job_y0[j] for j in jobs],
                   labels=[wl.labels[s] for s in mine])
    return Shard(sub, jobs, np.asarray(mine, dtype=np.int64))


def run_sharded(wl: Workload, rank: int, world: int, run: Callable, group=None) -> dict:
    """Propagate this rank's shard with ``run(workload) -> (ys, nodes, status)``
    (per local job) and gather every rank's results.  Returns, on every rank,
    {global job index: (Y, NODES, status)}.  With world == 1 no process group
    is needed."""
    sh = shard(wl, rank, world)
    ys, nodes, status = run(sh.workload) if len(sh.jobs) else ([], [], [])
    local = {int(j): (np.asarray(ys[k]), int(nodes[k]), int(status[k])) for k, j in enumerate(sh.jobs)}
    if world == 1:
        return local
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    out = {}
    for p in parts:
        out.update(p)
    return out


def gpu_run(prop: str = "LDMD") -> Callable:
    """The per-rank `run` of run_sharded on this process's current GPU: all
    of the shard's systems and jobs in one batched plan (the energies of a
    block share its 2HQ(C) table), Y in and out through host buffers."""
    def run(wl: Workload):
        from .propagators import Plan
        plan = Plan(prop, wl.systems, wl.segments, wl.job_sys, wl.job_ered)
        try:
            ybuf, nodes, status, _ = plan.run_host(plan.pack(wl.job_y0))
            return [plan.unpack(ybuf, j).copy() for j in range(wl.njobs)], nodes, status
        finally:
            plan.close()
    return run


def rank_units(costs, rank: int, world: int) -> np.ndarray:
    """The units (by index into `costs`) this rank propagates under LPT."""
    return lpt_partition(costs, world)[rank]
