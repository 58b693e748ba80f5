"""The device matching count (kernels_match.cuh): negative eigenvalues of
Y_a - Y_b from the inertia of an unpivoted LDL^T, against the host's
eigenvalue count (bdctrl.f:221-257 counts DIAGVL's eigenvalues <= 0).

* random symmetric pairs, N = 1..240, well and badly conditioned: equal to
  numpy's eigvalsh count;
* an exactly zero pivot reports -1 (the caller counts from eigenvalues);
* N above 240 is refused as unsupported;
* a field sweep counted on the device equals the host count at every field.
"""
import ctypes

import numpy as np
import pytest

import cases
from molscat_b200 import _lib
from molscat_b200.propagators import Plan

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    return torch


def _plan_for(ns):
    """A plan whose jobs 2k and 2k+1 have N = ns[k] (the systems only set the
    Y layout; nothing is propagated)."""
    systems, segs = [], []
    for n in ns:
        c, seg, _, _ = cases.random_case(n, 4, seed=n)
        systems.append(c)
        segs.append(seg)
    job_sys = np.repeat(np.arange(len(ns)), 2)
    return Plan("LDMD", systems, segs, job_sys, np.full(job_sys.size, 10.0))


def _device_counts(torch, plan, mats):
    L = _lib.load()
    y = np.zeros(plan.y_elems)
    for j, a in enumerate(mats):
        n = a.shape[0]
        y[plan.offsets[j]:plan.offsets[j] + n * n] = a.ravel(order="F")
    yd = torch.from_numpy(y).cuda()
    npairs = len(mats) // 2
    pairs = torch.tensor(np.arange(2 * npairs, dtype=np.int32)).cuda()
    counts = torch.full((npairs,), -7, dtype=torch.int32).cuda()
    st = torch.cuda.current_stream().cuda_stream
    rc = L.mgpu_plan_match_counts_device(plan._handle, ctypes.c_void_p(yd.data_ptr()), npairs,
                                         ctypes.c_void_p(pairs.data_ptr()), ctypes.c_void_p(counts.data_ptr()),
                                         ctypes.c_void_p(st))
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    return counts.cpu().numpy()


def _sym(rng, n, spread):
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    lam = rng.normal(size=n) * np.exp(rng.uniform(-spread, spread, n))
    return (q * lam) @ q.T


def test_device_counts_equal_eigenvalue_counts(torch_cuda):
    rng = np.random.default_rng(11)
    ns = [1, 2, 5, 17, 36, 64, 106, 150, 200, 240]
    plan = _plan_for(ns)
    mats = []
    for n in ns:
        b = _sym(rng, n, 1.0)
        d = _sym(rng, n, 6.0)  # eigenvalues over ~5 decades
        mats += [b + d, b]
    got = _device_counts(torch_cuda, plan, mats)
    want = [int(np.sum(np.linalg.eigvalsh(mats[2 * k] - mats[2 * k + 1]) < 0.0)) for k in range(len(ns))]
    assert list(got) == want
    plan.close()


def test_zero_pivot_reports_minus_one(torch_cuda):
    rng = np.random.default_rng(5)
    plan = _plan_for([12])
    b = _sym(rng, 12, 1.0)
    d = _sym(rng, 12, 1.0)
    d[0, :] = 0.0
    d[:, 0] = 0.0
    got = _device_counts(torch_cuda, plan, [b + d, b])
    assert list(got) == [-1]
    plan.close()


def test_large_n_is_unsupported(torch_cuda):
    torch = torch_cuda
    L = _lib.load()
    plan = _plan_for([256])
    yd = torch.zeros(plan.y_elems, dtype=torch.float64).cuda()
    pairs = torch.tensor([0, 1], dtype=torch.int32).cuda()
    counts = torch.zeros(1, dtype=torch.int32).cuda()
    rc = L.mgpu_plan_match_counts_device(plan._handle, ctypes.c_void_p(yd.data_ptr()), 1,
                                         ctypes.c_void_p(pairs.data_ptr()), ctypes.c_void_p(counts.data_ptr()),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.MGPU_ERR_UNSUPPORTED
    plan.close()


def test_field_sweep_counts_on_device_equal_host(torch_cuda):
    from molscat_b200.alkali import config4_sweep
    from molscat_b200.field import FieldProblem, field_node_counts
    sw = config4_sweep(mtot=8, block=1, nout=600, nin=800)
    fp = FieldProblem(sw.coupling_at, sw.seg_out, sw.seg_in, ered_at=sw.ered_at, prop="LDMD")
    fields = np.linspace(0.0, 1000.0, 40)
    host = field_node_counts(fp, fields, eig=True)
    dev = field_node_counts(fp, fields, eig=False)
    assert np.array_equal(host[3], dev[3])
    assert np.array_equal(host[0], dev[0])
