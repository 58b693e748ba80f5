"""Independent propagations spread over ranks: partition properties, and a
world_size-2 run over gloo on CPU whose gathered results equal a
single-process run exactly.

The propagation inside each rank is the CPU oracle here (test
infrastructure, run as the stand-in compute); with GPUs the same shards go
through the CUDA library, one process per GPU.
"""
import datetime
import os
import pickle
import socket

import numpy as np
import pytest

import cases
from molscat_b200 import sharding
from molscat_b200.systems import batched_workload


def small_workload():
    return batched_workload(n_energies=3, jtots=range(0, 6), nstep=150)


def oracle_run(wl):
    from oracle import oracle as O
    ys, nodes, status = [], [], []
    for j in range(wl.njobs):
        s = int(wl.job_sys[j])
        c, g = wl.systems[s], wl.segments[s]
        y, nd, st, _ = O.mdprop(cases.to_oracle(c), g.rtab, g.ptab, g.nstep, g.dr, float(wl.job_ered[j]),
                                wl.job_y0[j])
        ys.append(y)
        nodes.append(nd)
        status.append(st)
    return ys, nodes, status


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        wl = small_workload()
        res = sharding.run_sharded(wl, rank, world, oracle_run)
        mine = sharding.shard(wl, rank, world)
        with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump({"results": res, "my_jobs": mine.jobs.tolist()}, f)
    finally:
        dist.destroy_process_group()


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(3)
    costs = rng.uniform(1.0, 100.0, size=37) ** 3
    for world in (1, 2, 3, 8):
        parts = sharding.lpt_partition(costs, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(costs)))
        loads = [costs[p].sum() for p in parts]
        # LPT: no rank exceeds the least-loaded one by more than the largest unit
        assert max(loads) - min(loads) <= costs.max() + 1e-6
        again = sharding.lpt_partition(costs, world)  # deterministic
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))


def test_shard_keeps_blocks_whole():
    wl = small_workload()
    world = 2
    seen = []
    for r in range(world):
        sh = sharding.shard(wl, r, world)
        seen.extend(sh.jobs.tolist())
        for k, j in enumerate(sh.jobs):
            assert sh.systems[sh.workload.job_sys[k]] == wl.job_sys[j]
            assert sh.workload.job_ered[k] == wl.job_ered[j]
        # every energy of a block is on this rank
        for s in sh.systems:
            assert set(np.nonzero(wl.job_sys == s)[0]) <= set(sh.jobs.tolist())
    assert sorted(seen) == list(range(wl.njobs))


def test_two_ranks_gloo_equal_single_process(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    wl = small_workload()
    single = sharding.run_sharded(wl, 0, 1, oracle_run)
    outs = []
    for r in range(world):
        with open(tmp_path / f"rank{r}.pkl", "rb") as f:
            outs.append(pickle.load(f))
    assert set(outs[0]["my_jobs"]).isdisjoint(outs[1]["my_jobs"])
    assert outs[0]["my_jobs"] and outs[1]["my_jobs"]
    for o in outs:
        res = o["results"]
        assert sorted(res) == list(range(wl.njobs))
        for j, (y, nd, st) in res.items():
            ys, nds, sts = single[j]
            assert st == sts == 0
            assert nd == nds
            assert np.array_equal(y, ys)


def _gpu_worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)  # both ranks share the one GPU: their kernels never wait on each other
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300))
    try:
        wl = small_workload()
        res = sharding.run_sharded(wl, rank, world, sharding.gpu_run())
        with open(os.path.join(out_dir, f"gpu_rank{rank}.pkl"), "wb") as f:
            pickle.dump(res, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_cuda_path_equals_oracle_and_single_process(tmp_path):
    """The CUDA library as each rank's propagator: world size 1 against the
    oracle (NODES exact, Y within 5e-8), then two gloo ranks (one GPU, each
    its own process and plan) gathering results equal to world size 1's bit
    for bit."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    wl = small_workload()
    one = sharding.run_sharded(wl, 0, 1, sharding.gpu_run())
    ora = sharding.run_sharded(wl, 0, 1, oracle_run)
    assert sorted(one) == list(range(wl.njobs))
    for j, (y, nd, st) in one.items():
        yo, ndo, sto = ora[j]
        assert st == sto == 0 and nd == ndo
        assert cases.rel_err(y, yo) < 5e-8
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_gpu_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        with open(tmp_path / f"gpu_rank{r}.pkl", "rb") as f:
            res = pickle.load(f)
        assert sorted(res) == list(range(wl.njobs))
        for j, (y, nd, st) in res.items():
            assert st == one[j][2] and nd == one[j][1]
            assert np.array_equal(y, one[j][0])
