"""ctypes binding of libmolscat_gpu.so (C ABI: include/molscat_gpu.h).

The CUDA library is the only implementation: if it is missing this module
raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

from .build import LIB

MGPU_OK = 0
MGPU_ERR_INVERSION = 1
MGPU_ERR_NONFINITE = 2
MGPU_ERR_ARG = 3
MGPU_ERR_CUDA = 4
MGPU_ERR_UNSUPPORTED = 5
MGPU_ERR_NOMEM = 6
MGPU_ERR_TIMEOUT = 7
MGPU_ERR_CANCELLED = 8
MGPU_ERR_DEADLINE = 9

MGPU_PROP_LDJ = 5
MGPU_PROP_LDMD = 6
MGPU_PROP_LDMG4 = 84  # MGPROP, IMGSEL = 4 (CS4)
MGPU_PROP_LDMG5 = 85  # MGPROP, IMGSEL = 5 (MA5)

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class Coupling_C(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("nham", ctypes.c_int), ("nvlblk", ctypes.c_int), ("ivlfl", ctypes.c_int),
        ("nconst", ctypes.c_int), ("nrsq", ctypes.c_int), ("conlen", ctypes.c_double),
        ("vl", _dp), ("iv", _ip), ("eint", _dp), ("cent", _dp),
    ]


class Grid_C(ctypes.Structure):
    _fields_ = [("nstep", ctypes.c_int), ("dr", ctypes.c_double), ("rtab", _dp), ("ptab", _dp)]


# every symbol include/molscat_gpu.h declares
EXPORTS = (
    "mgpu_mdprop", "mgpu_ldprop",
    "mgpu_plan_create", "mgpu_plan_destroy", "mgpu_plan_y_elems", "mgpu_plan_y_offset",
    "mgpu_plan_flops", "mgpu_plan_shared_systems", "mgpu_plan_match_counts", "mgpu_plan_match_counts_device",
    "mgpu_plan_run_host", "mgpu_plan_run_device", "mgpu_plan_launches",
    "mgpu_plan_run_device_phases", "mgpu_plan_flops_phase", "mgpu_probe_fp64_fma",
    "mgpu_status_string", "mgpu_last_error", "mgpu_max_n", "mgpu_mdprop_noalloc", "mgpu_set_kernel_family",
    "mgpu_server_create", "mgpu_server_destroy", "mgpu_server_add_system", "mgpu_submit", "mgpu_poll",
    "mgpu_wait", "mgpu_request_times", "mgpu_release", "mgpu_server_in_flight", "mgpu_set_family_for_n",
    "mgpu_plan_s_elems", "mgpu_plan_s_offset", "mgpu_plan_nopen", "mgpu_plan_smatrix_device",
    "mgpu_plan_run_host_smatrix", "mgpu_plan_set_asymptote", "mgpu_plan_smatrix_host",
    "mgpu_probe_pivot_reciprocal", "mgpu_mdprop_f", "mgpu_ldprop_f",
    "mgpu_plan_cancel", "mgpu_plan_set_time_limit", "mgpu_set_step_wait_limit", "mgpu_ldmg_radii",
    "mgpu_mgprop", "mgpu_mgprop_f", "mgpu_ldma_create", "mgpu_ldma_run_host", "mgpu_ldma_destroy",
    "mgpu_airy_create", "mgpu_airy_run_host", "mgpu_airy_destroy",
)

_lib = None


def load(path: str | None = None):
    """Load the CUDA library (no compute call is made): `path`, else
    $MOLSCAT_GPU_LIB, else the in-tree build."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("MOLSCAT_GPU_LIB") or LIB
    if not os.path.exists(p):
        raise ImportError(f"{p} is missing: build it with `python -m molscat_b200.build` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(p)
    pc = ctypes.POINTER(Coupling_C)
    pg = ctypes.POINTER(Grid_C)
    vp = ctypes.c_void_p
    L.mgpu_mdprop.argtypes = [pc, pg, ctypes.c_double, _dp, _ip, _ip]
    L.mgpu_ldprop.argtypes = [pc, pg, ctypes.c_double, _dp, _ip, _ip]
    L.mgpu_mgprop.argtypes = [ctypes.c_int, pc, pg, ctypes.c_double, _dp, _ip, _ip]
    L.mgpu_ldma_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   _dp, _dp, _dp, _dp, _dp]
    L.mgpu_ldma_run_host.argtypes = [vp, ctypes.c_int, _dp, _dp, _ip, _ip]
    L.mgpu_ldma_destroy.argtypes = [vp]
    L.mgpu_airy_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
    L.mgpu_airy_run_host.argtypes = [vp, ctypes.c_int, _dp, _dp, _ip, _ip]
    L.mgpu_airy_destroy.argtypes = [vp]
    L.mgpu_plan_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, pc, pg, ctypes.c_int, _ip, _dp]
    L.mgpu_plan_destroy.argtypes = [vp]
    L.mgpu_plan_destroy.restype = None
    L.mgpu_plan_y_elems.argtypes = [vp]
    L.mgpu_plan_y_elems.restype = ctypes.c_size_t
    L.mgpu_plan_y_offset.argtypes = [vp, ctypes.c_int]
    L.mgpu_plan_y_offset.restype = ctypes.c_size_t
    L.mgpu_plan_flops.argtypes = [vp]
    L.mgpu_plan_flops.restype = ctypes.c_double
    L.mgpu_plan_shared_systems.argtypes = [vp]
    L.mgpu_plan_match_counts.argtypes = [vp, ctypes.c_int, _ip, _ip]
    L.mgpu_plan_match_counts_device.argtypes = [vp, vp, ctypes.c_int, vp, vp, vp]
    L.mgpu_plan_run_host.argtypes = [vp, _dp, _ip, _ip, _ip]
    L.mgpu_plan_run_device.argtypes = [vp, vp, vp, vp, vp, vp]
    L.mgpu_plan_launches.argtypes = [vp]
    L.mgpu_plan_run_device_phases.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_int]
    L.mgpu_plan_flops_phase.argtypes = [vp, ctypes.c_int]
    L.mgpu_plan_flops_phase.restype = ctypes.c_double
    L.mgpu_probe_fp64_fma.argtypes = [vp, ctypes.c_int, vp, _dp]
    L.mgpu_probe_pivot_reciprocal.argtypes = [vp, vp, ctypes.c_int, vp]
    L.mgpu_plan_cancel.argtypes = [vp, ctypes.c_int]
    L.mgpu_plan_set_time_limit.argtypes = [vp, ctypes.c_double]
    L.mgpu_set_step_wait_limit.argtypes = [ctypes.c_int]
    L.mgpu_mdprop_noalloc.argtypes = [pc, pg, ctypes.c_int, vp, vp, vp, vp, vp, vp]
    L.mgpu_status_string.argtypes = [ctypes.c_int]
    L.mgpu_status_string.restype = ctypes.c_char_p
    L.mgpu_last_error.argtypes = []
    L.mgpu_last_error.restype = ctypes.c_char_p
    L.mgpu_max_n.argtypes = []
    L.mgpu_set_kernel_family.argtypes = [ctypes.c_int]
    L.mgpu_set_family_for_n.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.mgpu_plan_s_elems.argtypes = [vp]
    L.mgpu_plan_s_elems.restype = ctypes.c_size_t
    L.mgpu_plan_s_offset.argtypes = [vp, ctypes.c_int]
    L.mgpu_plan_s_offset.restype = ctypes.c_size_t
    L.mgpu_plan_nopen.argtypes = [vp, ctypes.c_int]
    L.mgpu_plan_smatrix_device.argtypes = [vp, vp, vp, vp, vp, vp]
    L.mgpu_plan_run_host_smatrix.argtypes = [vp, _dp, _dp, _dp, _ip, _ip, _ip]
    L.mgpu_plan_set_asymptote.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double]
    L.mgpu_plan_smatrix_host.argtypes = [vp, _dp, _dp, _dp, _ip]
    L.mgpu_ldmg_radii.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp]
    ll = ctypes.c_longlong
    L.mgpu_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int]
    L.mgpu_server_destroy.argtypes = [vp]
    L.mgpu_server_destroy.restype = None
    L.mgpu_server_add_system.argtypes = [vp, pc, pg, _ip]
    L.mgpu_submit.argtypes = [vp, ctypes.c_int, ctypes.c_double, _dp, _dp, _ip, _ip, _ip, ctypes.POINTER(ll)]
    L.mgpu_poll.argtypes = [vp, ll]
    L.mgpu_wait.argtypes = [vp, ll]
    L.mgpu_request_times.argtypes = [vp, ll, _dp]
    L.mgpu_release.argtypes = [vp, ll]
    L.mgpu_server_in_flight.argtypes = [vp, _ip, _ip, ctypes.POINTER(ctypes.c_size_t)]
    if path is None:
        _lib = L
    return L


FAMILY_DMMA = 0
FAMILY_TILE4 = 1
FAMILY_BIG = 2


def set_family_for_n(n_lo: int, n_hi: int, family: int, prop: str | None = None) -> None:
    """Per-N kernel family for plans created afterwards, for one propagator
    ("LDMD" / "LDJ") or both (None); family < 0 clears."""
    iprop = 0 if prop is None else (MGPU_PROP_LDMD if prop == "LDMD" else MGPU_PROP_LDJ)
    rc = load().mgpu_set_family_for_n(iprop, int(n_lo), int(n_hi), int(family))
    if rc != 0:
        raise ValueError(last_error())


def set_kernel_family(family: int) -> int:
    """Kernel family for N <= 64 (FAMILY_DMMA default, FAMILY_TILE4); returns the old one."""
    return int(load().mgpu_set_kernel_family(int(family)))


def last_error() -> str:
    return load().mgpu_last_error().decode()


def status_string(code: int) -> str:
    return load().mgpu_status_string(int(code)).decode()
