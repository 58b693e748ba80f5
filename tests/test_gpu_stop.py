"""Failure detection without a GPU fault: host-requested stops and the
bounded in-kernel wait running out.

* A plan cancelled before its run stops every job at step 1 with
  MGPU_ERR_CANCELLED (one-warp, one-CTA and 4x4-tile kernel families, both
  propagators); after the request is cleared the same plan runs to the same
  results as a fresh plan, so the context stays usable.
* A cancel from another host thread while the run is on the GPU stops every
  job at a poll step (1 + 128 m) strictly inside the run.
* A time limit shorter than the kernels' run stops the jobs with
  MGPU_ERR_DEADLINE at a poll step.
* With the one-warp kernels' per-step copy wait lowered to zero iterations
  (mgpu_set_step_wait_limit, a test hook) every job reports MGPU_ERR_TIMEOUT
  at step 1: the wait gives up, the copy in flight lands under the full
  drain limit, and the restored limit runs normally again.
No kernel traps, faults or spins without a bound here.
"""
import threading
import time

import numpy as np
import pytest

import cases
from molscat_b200 import _lib
from molscat_b200.propagators import Plan

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    _lib.load()


def _plan(prop, n, nstep, njobs, seed):
    c, seg, ered, y0 = cases.random_case(n, nstep, seed=seed)
    ereds = ered + np.linspace(0.0, 3.0, njobs)
    plan = Plan(prop, [c], [seg], np.zeros(njobs, dtype=np.int32), ereds)
    return plan, plan.pack([y0] * njobs)


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
@pytest.mark.parametrize("n, family", [(12, 0), (60, 0), (50, 1)], ids=["warp", "cta", "tile4"])
def test_cancel_before_run_then_clear(prop, n, family):
    old = _lib.set_kernel_family(family)
    try:
        plan, y0 = _plan(prop, n, 300, 3, seed=900 + n)
        fresh, _ = _plan(prop, n, 300, 3, seed=900 + n)
    finally:
        _lib.set_kernel_family(old)
    try:
        plan.cancel(True)
        _, nodes, st, kf = plan.run_host(y0)
        assert (st == _lib.MGPU_ERR_CANCELLED).all() and (kf == 1).all()
        plan.cancel(False)
        y, nodes, st, kf = plan.run_host(y0)
        yf, nf, sf, _ = fresh.run_host(y0)
        assert (st == 0).all() and (sf == 0).all()
        assert np.array_equal(nodes, nf) and np.array_equal(y, yf)
    finally:
        plan.close()
        fresh.close()


def test_cancel_from_another_thread_mid_run():
    nstep = 150000
    plan, y0 = _plan("LDMD", 36, nstep, 8, seed=77)
    out = {}

    def run():
        out["res"] = plan.run_host(y0)

    try:
        th = threading.Thread(target=run)
        th.start()
        time.sleep(0.4)
        plan.cancel(True)
        th.join(timeout=120)
        assert not th.is_alive()
        _, nodes, st, kf = out["res"]
        assert (st == _lib.MGPU_ERR_CANCELLED).all()
        assert ((kf > 1) & (kf < nstep) & ((kf - 1) % 128 == 0)).all(), kf
    finally:
        plan.close()


@pytest.mark.parametrize("n", [20, 60])
def test_time_limit_stops_jobs_with_deadline(n):
    plan, y0 = _plan("LDMD", n, 2000, 4, seed=600 + n)
    try:
        plan.set_time_limit(1e-9)
        _, nodes, st, kf = plan.run_host(y0)
        assert (st == _lib.MGPU_ERR_DEADLINE).all()
        assert ((kf >= 1) & ((kf - 1) % 128 == 0)).all(), kf
        plan.set_time_limit(0.0)
        _, nodes, st, kf = plan.run_host(y0)
        assert (st == 0).all()
    finally:
        plan.close()


def test_step_wait_running_out_reports_timeout():
    L = _lib.load()
    plan, y0 = _plan("LDMD", 30, 200, 4, seed=31)
    try:
        y_ok, n_ok, st_ok, _ = plan.run_host(y0)
        assert (st_ok == 0).all()
        assert L.mgpu_set_step_wait_limit(0) == 0
        try:
            _, nodes, st, kf = plan.run_host(y0)
        finally:
            assert L.mgpu_set_step_wait_limit(-1) == 0
        assert (st == _lib.MGPU_ERR_TIMEOUT).all() and (kf == 1).all()
        y2, n2, st2, _ = plan.run_host(y0)
        assert (st2 == 0).all() and np.array_equal(y2, y_ok) and np.array_equal(n2, n_ok)
    finally:
        plan.close()
