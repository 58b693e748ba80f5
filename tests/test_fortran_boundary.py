"""The Fortran calling convention at the boundary.

The replacement MDPROP/LDPROP/MGPROP (molscat_b200/fortran/mdprop_gpu.f)
binds mgpu_mdprop_f / mgpu_ldprop_f / mgpu_mgprop_f (and mgpu_ldmg_radii for
MGPROP's stage radii) with plain BIND(C) interface blocks, every argument
by reference except the radii helper's scalars.  No Fortran compiler exists in this image, so a C
host (tests/host/fortran_convention_host.c) makes the same calls: each
scalar as the address of a variable, each array column-major.

* CPU: the host compiles and links against libmolscat_gpu.so and gets
  MGPU_ERR_ARG back for a bad step (no GPU needed for argument checks); the
  shim source declares the two entry points the header declares.
* GPU: the host's results equal the Python path's (the C ABI through
  ctypes) bit for bit, MDPROP and LDPROP with IV indexing, MGPROP (CS4 and
  MA5) on the one-warp and one-CTA kernels.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import cases
from molscat_b200 import _lib
from molscat_b200.build import LIB, PKG, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    build()
    exe = tmp_path_factory.mktemp("host") / "fortran_convention_host"
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "host", "fortran_convention_host.c"), "-o", str(exe),
                           "-L", PKG, "-lmolscat_gpu", "-Wl,-rpath," + PKG])
    return exe


def _write_input(path, iprop, c, seg, ered, y0):
    n = c.n
    with open(path, "wb") as f:
        np.array([iprop, n, c.nham, c.nvlblk, c.ivlfl, c.nconst, c.nrsq, seg.nstep], dtype=np.int32).tofile(f)
        np.array([c.conlen, seg.dr, ered], dtype=np.float64).tofile(f)
        npair = n * (n + 1) // 2
        np.ascontiguousarray(c.vl[:c.nvlblk * npair], dtype=np.float64).tofile(f)
        iv = c.iv if c.ivlfl > 0 else np.ones(c.nvlblk * npair, dtype=np.int32)
        np.ascontiguousarray(iv[:c.nvlblk * npair], dtype=np.int32).tofile(f)
        np.ascontiguousarray(c.eint[:n], dtype=np.float64).tofile(f)
        np.ascontiguousarray(c.cent[:n], dtype=np.float64).tofile(f)
        np.ascontiguousarray(seg.rtab, dtype=np.float64).tofile(f)
        np.ascontiguousarray(seg.ptab[:, :c.nham], dtype=np.float64).tofile(f)
        np.asfortranarray(y0, dtype=np.float64).ravel(order="F").tofile(f)


def _run(host, tmp_path, iprop, c, seg, ered, y0):
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    _write_input(inp, iprop, c, seg, ered, y0)
    subprocess.check_call([str(host), str(inp), str(out)])
    raw = np.fromfile(out, dtype=np.uint8)
    istat, nodes, kfail = (int(x) for x in raw[:12].view(np.int32))
    y = raw[12:].view(np.float64).reshape((c.n, c.n), order="F")
    return istat, nodes, kfail, y


def test_shim_binds_the_declared_entry_points():
    with open(os.path.join(ROOT, "molscat_b200", "fortran", "mdprop_gpu.f")) as f:
        src = f.read()
    names = set(re.findall(r"NAME='(mgpu_[a-z_]+)'", src))
    assert names == {"mgpu_mdprop_f", "mgpu_ldprop_f", "mgpu_mgprop_f", "mgpu_ldmg_radii"}
    assert names <= set(_lib.EXPORTS)
    for ln in src.splitlines():  # fixed form: statements end by column 72
        assert ln[:1] in "Cc" or len(ln) <= 72, ln


def test_host_gets_argument_errors_without_a_gpu(host, tmp_path):
    c, seg, ered, y0 = cases.random_case(5, 10, seed=5)
    seg.dr = 0.0
    istat, nodes, kfail, _ = _run(host, tmp_path, _lib.MGPU_PROP_LDMD, c, seg, ered, y0)
    assert istat == _lib.MGPU_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("iprop", [6, 5], ids=["MDPROP", "LDPROP"])
@pytest.mark.parametrize("n, kw", [(12, {}), (36, dict(ivlfl=1)), (70, dict(nconst=1, nrsq=1))],
                         ids=["n12", "n36-iv", "n70-const-rsq"])
def test_host_matches_python_path(host, tmp_path, iprop, n, kw):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.propagators import propagate
    c, seg, ered, y0 = cases.random_case(n, 80, seed=300 + n, **kw)
    istat, nodes, kfail, y = _run(host, tmp_path, iprop, c, seg, ered, y0)
    assert istat == 0 and kfail == 0
    yp, np_ = propagate("LDMD" if iprop == 6 else "LDJ", c, seg, ered, y0)
    assert nodes == np_
    assert np.array_equal(y, yp)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["LDMG4", "LDMG5"])
@pytest.mark.parametrize("n", [12, 36, 70])
def test_host_matches_python_path_mgprop(host, tmp_path, kind, n):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from molscat_b200.propagators import PROPS, propagate
    c, seg, ered, y0 = cases.random_case(n, 60, seed=400 + n, kind=kind)
    istat, nodes, kfail, y = _run(host, tmp_path, PROPS[kind], c, seg, ered, y0)
    assert istat == 0 and kfail == 0
    yp, np_ = propagate(kind, c, seg, ered, y0)
    assert nodes == np_
    assert np.array_equal(y, yp)
