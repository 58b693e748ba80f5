"""The pivot reciprocal every inversion uses (tiles.cuh, pivot_reciprocal):
the hardware seed rcp.approx.ftz.f64 refined by one third-order Newton step
(e = 1 - d r, r <- r + r (e + e^2); J.-M. Muller et al., Handbook of
Floating-Point Arithmetic, ch. 5), with exact power-of-two scaling of
magnitudes outside [2^-1000, 2^1000].  Claim: within one ulp of the
correctly rounded 1/x for every x whose reciprocal is a normal number.
Checked against CUDA's own 1.0/x (IEEE division on the device) and numpy's,
over random magnitudes spanning the exponent range and the scaling edges."""
import ctypes

import numpy as np
import pytest

from molscat_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.build import build
    build()
    return torch


def _inputs():
    rng = np.random.default_rng(31)
    mags = np.ldexp(rng.uniform(1.0, 2.0, 200_000), rng.integers(-1021, 1022, 200_000))
    edges = []
    for e in (-1022, -1021, -1001, -1000, -999, -512, -1, 0, 1, 511, 999, 1000, 1001, 1021):
        b = np.ldexp(1.0, e)
        edges += [b, np.nextafter(b, 0.0), np.nextafter(b, np.inf), 1.5 * b]
    x = np.concatenate([mags, np.array(edges), rng.uniform(-3.0, 3.0, 50_000)])
    x = x[(x != 0.0) & np.isfinite(x)]
    sgn = np.where(rng.random(x.size) < 0.5, -1.0, 1.0)
    x = x * sgn
    # keep x whose reciprocal is a normal double
    return x[np.abs(1.0 / x) >= np.finfo(np.float64).tiny]


def _ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    assert (np.sign(a) == np.sign(b)).all()
    return np.abs(ia - ib)


def test_pivot_reciprocal_within_one_ulp_of_division(torch_cuda):
    torch = torch_cuda
    L = _lib.load()
    x = _inputs()
    xd = torch.from_numpy(x).cuda()
    rd = torch.empty_like(xd)
    st = torch.cuda.current_stream().cuda_stream
    rc = L.mgpu_probe_pivot_reciprocal(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(rd.data_ptr()), x.size,
                                       ctypes.c_void_p(st))
    assert rc == 0, _lib.last_error()
    cuda_div = (1.0 / xd).cpu().numpy()  # CUDA's IEEE double division
    got = rd.cpu().numpy()
    assert np.array_equal(cuda_div, 1.0 / x)
    u = _ulps(got, cuda_div)
    assert u.max() <= 1, f"max {u.max()} ulp at x = {x[np.argmax(u)]!r}"
    # nearly always the correctly rounded value
    assert (u == 0).mean() > 0.99
