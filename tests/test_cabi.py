"""The C-ABI library loads and exports every symbol include/molscat_gpu.h
declares; argument validation works without a GPU (no compute calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

from molscat_b200 import _lib
from molscat_b200.build import LIB, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build()
    return _lib.load()


def header_functions():
    with open(os.path.join(ROOT, "include", "molscat_gpu.h")) as f:
        txt = f.read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mgpu_[a-z_0-9]+)\s*\(", txt)))


def test_header_symbols_exported(lib):
    names = header_functions()
    assert len(names) >= 13
    raw = ctypes.CDLL(LIB)
    for n in names:
        assert hasattr(raw, n), n
    assert set(_lib.EXPORTS) == set(names)


def test_library_is_sm100a_cuda(lib):
    # the shared object links the CUDA runtime and carries an sm_100a image
    with open(LIB, "rb") as f:
        blob = f.read()
    assert b"sm_100a" in blob


def test_argument_validation_without_gpu(lib):
    from molscat_b200.propagators import Coupling, Segment, PropagatorError, Plan
    assert lib.mgpu_max_n() >= 1024
    n = lib.mgpu_max_n() + 1
    c = Coupling(n=n, nham=1, vl=np.zeros(n * (n + 1) // 2), eint=np.zeros(n), cent=np.zeros(n))
    seg = Segment(1, 0.1, np.array([1.0, 1.05, 1.1]), np.zeros((3, 1)))
    with pytest.raises(PropagatorError) as e:
        Plan("LDMD", [c], [seg], np.array([0]), np.array([1.0]))
    assert e.value.status == _lib.MGPU_ERR_UNSUPPORTED
    c2 = Coupling(n=2, nham=1, vl=np.zeros(3), eint=np.zeros(2), cent=np.zeros(2))
    with pytest.raises(PropagatorError) as e:
        Plan("LDMD", [c2], [seg], np.array([3]), np.array([1.0]))  # bad system index
    assert e.value.status == _lib.MGPU_ERR_ARG
    bad = Segment(1, 0.0, np.array([1.0, 1.0, 1.0]), np.zeros((3, 1)))
    with pytest.raises(PropagatorError) as e:
        Plan("LDJ", [c2], [bad], np.array([0]), np.array([1.0]))  # DR = 0
    assert e.value.status == _lib.MGPU_ERR_ARG
    assert _lib.status_string(_lib.MGPU_ERR_INVERSION).startswith("matrix inversion")


def test_segment_radii_accumulate_like_the_reference():
    from molscat_b200.propagators import radial_grid
    r = radial_grid(0.5, 0.1, 3)
    x = 0.5
    for k in range(1, 7):
        x = x + 0.05
        assert r[k] == x
