"""mgpu_mdprop_noalloc: the MDPROP entry point that allocates no device memory.

It is meant for callers that cannot allocate device memory (their device
memory comes from their own pool or a framework allocator, or they must not
call cudaMalloc/cudaFree inside a latency-critical loop).  Here the test plays
such a caller: it owns every input and output buffer on the device and calls
the entry point through the C ABI twice in a row, for two systems of
different size, checking each result against the plan entry point
(mgpu_plan_run_host) within the tolerance of the other GPU parity tests.
This file sorts last so a run that stops at the first failure has already
run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import cases
from molscat_b200 import _lib
from molscat_b200._lib import Coupling_C, Grid_C
from molscat_b200.propagators import Plan

pytestmark = pytest.mark.gpu

Y_TOL = 5e-8  # the tolerance of the other GPU parity tests


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    return torch


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _run_noalloc(torch, c, seg, ereds, y0s):
    """Call mgpu_mdprop_noalloc with caller-owned device buffers only."""
    L = _lib.load()
    n, nj = c.n, len(ereds)
    keep = []
    vl = _dev(torch, c.vl, np.float64)
    iv = _dev(torch, c.iv, np.int32)
    eint = _dev(torch, c.eint, np.float64)
    cent = _dev(torch, c.cent, np.float64)
    rtab = _dev(torch, seg.rtab, np.float64)
    ptab = _dev(torch, seg.ptab, np.float64)
    ered = _dev(torch, np.asarray(ereds), np.float64)
    y = _dev(torch, np.concatenate([np.asarray(m, dtype=np.float64).ravel(order="F") for m in y0s]), np.float64)
    nodes = torch.zeros(nj, dtype=torch.int32, device="cuda")
    status = torch.full((nj,), -1, dtype=torch.int32, device="cuda")
    kfail = torch.zeros(nj, dtype=torch.int32, device="cuda")
    keep += [vl, iv, eint, cent, rtab, ptab, ered, y, nodes, status, kfail]
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    cs = Coupling_C(n, c.nham, c.nvlblk, c.ivlfl, c.nconst, c.nrsq, float(c.conlen),
                    ctypes.cast(vl.data_ptr(), dp), ctypes.cast(iv.data_ptr(), ip),
                    ctypes.cast(eint.data_ptr(), dp), ctypes.cast(cent.data_ptr(), dp))
    gs = Grid_C(seg.nstep, float(seg.dr), ctypes.cast(rtab.data_ptr(), dp), ctypes.cast(ptab.data_ptr(), dp))
    stream = torch.cuda.current_stream().cuda_stream
    vp = ctypes.c_void_p
    rc = L.mgpu_mdprop_noalloc(ctypes.byref(cs), ctypes.byref(gs), nj, vp(ered.data_ptr()), vp(y.data_ptr()),
                               vp(nodes.data_ptr()), vp(status.data_ptr()), vp(kfail.data_ptr()), vp(stream))
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    yh = y.cpu().numpy()
    return ([yh[j * n * n:(j + 1) * n * n].reshape((n, n), order="F") for j in range(nj)],
            nodes.cpu().numpy(), status.cpu().numpy())


def _run_plan(c, seg, ereds, y0s):
    plan = Plan("LDMD", [c], [seg], np.zeros(len(ereds), dtype=np.int32), np.asarray(ereds))
    ybuf, nodes, status, _ = plan.run_host(plan.pack(y0s))
    ys = [plan.unpack(ybuf, j).copy() for j in range(len(ereds))]
    plan.close()
    return ys, nodes, status


def test_noalloc_matches_plan_on_two_calls_in_a_row(torch_cuda):
    # first call N=36 (five 8x8 tile rows), second call N=15: the second one
    # must not see anything the first left in the shared scratch array
    for jtot, block, nstep, energies in ((10, 2, 300, (120.0, 300.0, 480.0)), (4, 1, 200, (60.0, 250.0))):
        c, seg, jobs = cases.rotor_case(jtot, block, nstep=nstep, energies_cm=energies)
        ereds = [j[0] for j in jobs]
        y0s = [j[1] for j in jobs]
        ya, na, sa = _run_noalloc(torch_cuda, c, seg, ereds, y0s)
        yb, nb, sb = _run_plan(c, seg, ereds, y0s)
        assert (sa == 0).all() and (sb == 0).all()
        assert np.array_equal(na, nb)
        for u, v in zip(ya, yb):
            assert np.abs(u - v).max() / max(1.0, np.abs(v).max()) < Y_TOL


@pytest.mark.parametrize("n, ivlfl, nconst", [(100, 1, 1), (60, 0, 0)], ids=["cta-iv", "cta"])
def test_noalloc_cta_bucket_matches_plan_on_two_calls_in_a_row(torch_cuda, n, ivlfl, nconst):
    # one CTA per matrix (40 < N <= 200), with the IV indexing converted to
    # the tile layout on the device; two calls in a row with different
    # energies, each against the plan entry point
    c, seg, ered, y0 = cases.random_case(n, 120, seed=4100 + n, ivlfl=ivlfl, nconst=nconst)
    for ereds in ((ered, ered + 3.0), (ered + 7.5,)):
        y0s = [y0] * len(ereds)
        ya, na, sa = _run_noalloc(torch_cuda, c, seg, ereds, y0s)
        yb, nb, sb = _run_plan(c, seg, ereds, y0s)
        assert (sa == 0).all() and (sb == 0).all()
        assert np.array_equal(na, nb)
        for u, v in zip(ya, yb):
            assert np.abs(u - v).max() / max(1.0, np.abs(v).max()) < Y_TOL


def test_noalloc_bad_iv_reports_nonfinite(torch_cuda):
    # IV lives in device memory, so an index outside 1..NHAM is not checked
    # on the host: the device turns it into NaN couplings and every job
    # reports MGPU_ERR_NONFINITE at step 1
    c, seg, ered, y0 = cases.random_case(12, 20, seed=4200, ivlfl=1)
    c.iv = c.iv.copy()
    c.iv[0] = c.nham + 5
    _, _, st = _run_noalloc(torch_cuda, c, seg, [ered], [y0])
    assert (st == _lib.MGPU_ERR_NONFINITE).all()


def test_noalloc_rejects_requests_beyond_the_scratch_limit(torch_cuda):
    L = _lib.load()
    c, seg, _ = cases.rotor_case(10, 2, nstep=10)
    cs = Coupling_C(c.n, c.nham, c.nvlblk, 0, 0, 0, 0.0, ctypes.cast(1 << 20, ctypes.POINTER(ctypes.c_double)),
                    ctypes.cast(1 << 20, ctypes.POINTER(ctypes.c_int)),
                    ctypes.cast(1 << 20, ctypes.POINTER(ctypes.c_double)),
                    ctypes.cast(1 << 20, ctypes.POINTER(ctypes.c_double)))
    # N=36 (five 8x8 tile rows) needs 512*15 = 7680 bytes of 2HQ(C) per
    # step: 20000 steps exceed 64 MiB
    gs = Grid_C(20000, 0.001, ctypes.cast(1 << 20, ctypes.POINTER(ctypes.c_double)),
                ctypes.cast(1 << 20, ctypes.POINTER(ctypes.c_double)))
    vp = ctypes.c_void_p
    rc = L.mgpu_mdprop_noalloc(ctypes.byref(cs), ctypes.byref(gs), 1, vp(1 << 20), vp(1 << 20), vp(1 << 20),
                               vp(1 << 20), vp(1 << 20), vp(0))
    assert rc == _lib.MGPU_ERR_UNSUPPORTED
    assert "64 MiB" in _lib.last_error()
