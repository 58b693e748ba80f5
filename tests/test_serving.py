"""Request server (mgpu_server_* / mgpu_submit / mgpu_poll / mgpu_wait):
every served result equals the same propagation run alone (bitwise: the
kernels propagate each job independently, so the batch a request lands in
cannot change it), requests that arrive while others run are admitted
without waiting for them, and admission respects the HBM budget."""
import time

import numpy as np
import pytest

import cases
from molscat_b200 import _lib
from molscat_b200.propagators import PropagatorError, propagate
from molscat_b200.serving import Server, latency_percentiles

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    _lib.load()


@pytest.mark.parametrize("prop", ["LDMD", "LDJ"])
def test_served_equals_alone(prop):
    sizes = (7, 24, 36, 45, 90, 260)  # one-warp, one-CTA and large-N buckets in one stream of requests
    items = [cases.random_case(n, 60, seed=900 + n) for n in sizes]
    with Server(prop, streams=3, max_batch=16) as srv:
        ids = [srv.add_system(c, seg) for (c, seg, _, _) in items]
        reqs = []
        for rnd in range(3):
            for k, (c, seg, ered, y0) in enumerate(items):
                e = ered + 3.0 * rnd
                reqs.append((k, e, srv.submit(ids[k], e, y0)))
        for k, e, r in reqs:
            c, seg, _, y0 = items[k]
            y = r.wait()
            ya, na = propagate(prop, c, seg, e, y0)
            assert np.array_equal(y, ya), (sizes[k], e)
            assert r.nodes == na
        p = latency_percentiles([r for _, _, r in reqs])
        assert 0.0 < p["p50"] <= p["p99"]


def test_arrivals_during_a_running_batch_are_admitted():
    big = cases.random_case(512, 40, seed=1)
    small = cases.random_case(20, 200, seed=2)
    with Server("LDMD", streams=4, max_batch=8) as srv:
        b = srv.add_system(big[0], big[1])
        s = srv.add_system(small[0], small[1])
        first = [srv.submit(b, big[2] + d, big[3]) for d in (0.0, 1.0, 2.0, 3.0)]
        t0 = time.time()
        while first[0].times()[1] == 0.0 and time.time() - t0 < 30:
            time.sleep(0.0005)
        assert first[0].times()[1] > 0.0  # the first batch is on the GPU
        later = [srv.submit(s, small[2] + d, small[3]) for d in np.linspace(0.0, 5.0, 8)]
        for r in later:
            r.wait()
        for r in first:
            r.wait()
        done_first = min(r.times()[2] for r in first)
        # admitted (launched) while the first batch was still running
        t0 = first[0].times()[0]
        info = [tuple(round(x - t0, 6) for x in r.times()) for r in first[:1] + later[:2]]
        assert all(r.times()[1] < done_first for r in later), info
        for r, d in zip(later, np.linspace(0.0, 5.0, 8)):
            ya, na = propagate("LDMD", small[0], small[1], small[2] + d, small[3])
            assert np.array_equal(r.wait(), ya) and r.nodes == na


def test_admission_respects_the_budget():
    c, seg, ered, y0 = cases.random_case(260, 20, seed=3)
    budget = 4 << 20
    with Server("LDMD", hbm_budget=budget, streams=4, max_batch=8) as srv:
        sid = srv.add_system(c, seg)
        reqs = [srv.submit(sid, ered + d, y0) for d in np.linspace(0.0, 4.0, 6)]
        peak = 0
        deadline = time.time() + 120
        while not all(r.done() for r in reqs) and time.time() < deadline:
            peak = max(peak, srv.in_flight()[2])
            time.sleep(0.0002)
        assert all(r.done() for r in reqs)
        assert peak <= budget
        ya, na = propagate("LDMD", c, seg, ered, y0)
        assert np.array_equal(reqs[0].wait(), ya)
        big = cases.random_case(1024, 2, seed=4)
        bid = srv.add_system(big[0], big[1])
        r = srv.submit(bid, big[2], big[3])
        with pytest.raises(PropagatorError) as e:
            r.wait()
        assert e.value.status == _lib.MGPU_ERR_NOMEM
