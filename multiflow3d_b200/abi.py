"""ctypes mirror of include/mf3d.h and the loader of the native library.

The native library ``libmf3d.so`` (CUDA sm_100a kernels + C++ host driver)
is built in-tree by ``multiflow3d_b200.build``.  Loading fails loudly when it
is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmf3d.so")

MF3D_OK = 0
MF3D_NOT_CONVERGED = 1
MF3D_DIVERGED = 2
MF3D_PENDING = 3
MF3D_E_INVALID = -1
MF3D_E_CUDA = -2
MF3D_E_OOM = -3
MF3D_E_TIMEOUT = -4
MF3D_E_NONFINITE = -5
MF3D_E_UNSUPPORTED = -6

MF3D_BC_PERIODIC = 5
MF3D_PREC_FP64 = 0
MF3D_PREC_FP32 = 1
MF3D_PREC_BF16 = 2

_dp = C.POINTER(C.c_double)


class BlockDesc(C.Structure):
    """``mf3d_block_desc`` - one block (reference ``type multidom``)."""

    _fields_ = [
        ("id", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("xsl", C.c_double), ("xel", C.c_double),
        ("ysl", C.c_double), ("yel", C.c_double),
        ("zsl", C.c_double), ("zel", C.c_double),
        ("iprev", C.c_int), ("inext", C.c_int),
        ("jprev", C.c_int), ("jnext", C.c_int),
        ("kprev", C.c_int), ("knext", C.c_int),
        ("corprev", C.c_int * 4), ("cornext", C.c_int * 4),
        ("edgprev", C.c_int * 6), ("edgnext", C.c_int * 6),
        ("per_ip", C.c_int), ("per_in", C.c_int),
        ("per_jp", C.c_int), ("per_jn", C.c_int),
        ("per_kp", C.c_int), ("per_kn", C.c_int),
        ("bc_west", C.c_int), ("bc_east", C.c_int),
        ("bc_south", C.c_int), ("bc_north", C.c_int),
        ("bc_bottom", C.c_int), ("bc_top", C.c_int),
        ("hx", _dp), ("hy", _dp), ("hz", _dp),
    ]


class DomainDesc(C.Structure):
    """``mf3d_domain_desc`` - one independent single-block domain of a batch."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("bc", C.c_int * 3),
        ("ngrid", C.c_int),
        ("hx", _dp), ("hy", _dp), ("hz", _dp),
    ]


class Params(C.Structure):
    """``mf3d_params`` - the control.cin fields the projection reads."""

    _fields_ = [
        ("ngrid", C.c_int),
        ("mg_itrsch", C.c_int),
        ("irestr", C.c_int),
        ("iproln", C.c_int),
        ("maxcy", C.c_int),
        ("eps", C.c_double),
        ("eps_relative", C.c_int),
        ("pl", C.c_int),
        ("differencing", C.c_int),
        ("precision", C.c_int),
        ("device", C.c_int),
        ("pl_ex", C.c_int),
        ("lsm", C.c_int),
        ("bounds", C.c_int),
        ("solver", C.c_int),
        ("nswp", C.c_int),
        ("alfabc", C.c_int),
        ("ubulk", C.c_double),
    ]


class Fields(C.Structure):
    """``mf3d_fields`` - per-block field pointers (ttc layout)."""

    _fields_ = [
        ("ustar", _dp), ("vstar", _dp), ("wstar", _dp),
        ("u", _dp), ("v", _dp), ("w", _dp),
        ("p", _dp), ("su", _dp), ("dens", _dp),
    ]


class RkFields(C.Structure):
    """``mf3d_rk_fields`` - the predictor's start-of-step velocities and viscosity."""

    _fields_ = [("uoo", _dp), ("voo", _dp), ("woo", _dp), ("vis", _dp)]


class TecbinInfo(C.Structure):
    """``mf3d_tecbin_info`` - the header of a restart file."""

    _fields_ = [
        ("toti", C.c_int), ("totj", C.c_int), ("totk", C.c_int),
        ("pl", C.c_int),
        ("inind", C.c_int), ("jnind", C.c_int), ("knind", C.c_int),
        ("records", C.c_longlong),
        ("data_offset", C.c_longlong),
    ]


class SolveInfo(C.Structure):
    """``mf3d_solve_info``."""

    _fields_ = [
        ("rmax", C.c_double),
        ("rmax0", C.c_double),
        ("iter", C.c_int),
        ("status", C.c_int),
        ("ms_device", C.c_double),
    ]


class RequestInfo(C.Structure):
    """mf3d_request_info: a served request's result and timeline (seconds)."""
    _fields_ = [("info", SolveInfo), ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


# Every symbol include/mf3d.h declares (checked by the tests).
EXPORTED_SYMBOLS = (
    "mf3d_build_topology",
    "mf3d_create",
    "mf3d_destroy",
    "mf3d_newsolv_mg",
    "mf3d_newsolv_mg_device",
    "mf3d_mgkcyc_device",
    "mf3d_last_error",
    "mf3d_status_string",
    "mf3d_abi_version",
    "mf3d_last_launch_count",
    "mf3d_halo_map",
    "mf3d_halo_refresh_host",
    "mf3d_profile",
    "mf3d_profile_read",
    "mf3d_max_levels",
    "mf3d_batch_create",
    "mf3d_batch_solve_device",
    "mf3d_selftest_divide",
    "mf3d_mgkcyc_device_noalloc",
    "mf3d_server_create",
    "mf3d_server_submit",
    "mf3d_server_poll",
    "mf3d_server_stats",
    "mf3d_server_clock",
    "mf3d_server_profile",
    "mf3d_server_destroy",
    "mf3d_tecbin_info_of",
    "mf3d_tecbin_size",
    "mf3d_tecbin_decode_device",
    "mf3d_tecbin_encode_device",
    "mf3d_rungek_2nd_device",
    "mf3d_calvel_device",
    "mf3d_field_exchange_map",
    "mf3d_tuning",
    "mf3d_set_inlet",
    "mf3d_bind_old_velocity",
    "mf3d_set_wall_model",
    "mf3d_bounds_device",
    "mf3d_test_fail_alloc",
    "mf3d_test_stall_copy",
)

MF3D_NOALLOC_MAX_BLOCKS = 512

MF3D_PROF_OFF = 0
MF3D_PROF_SMOOTH_L1 = 1
MF3D_PROF_CALMAS = 2
MF3D_PROF_RESTRICT_L1 = 3
MF3D_PROF_PROLONG_L1 = 4

_lib = None


def _declare(lib):
    vp = C.c_void_p
    lib.mf3d_build_topology.argtypes = [C.c_int, _dp, C.POINTER(C.c_int), C.c_double,
                                        C.c_double, C.c_double, C.POINTER(BlockDesc)]
    lib.mf3d_create.argtypes = [C.POINTER(BlockDesc), C.c_int, C.POINTER(Params), C.POINTER(vp)]
    lib.mf3d_destroy.argtypes = [vp]
    lib.mf3d_newsolv_mg.argtypes = [vp, C.POINTER(Fields), C.c_double, C.c_double,
                                    C.POINTER(SolveInfo), _dp, C.c_int]
    lib.mf3d_newsolv_mg_device.argtypes = lib.mf3d_newsolv_mg.argtypes
    lib.mf3d_mgkcyc_device.argtypes = [vp, C.POINTER(_dp), C.POINTER(_dp)]
    lib.mf3d_mgkcyc_device_noalloc.argtypes = [vp, C.POINTER(_dp), C.POINTER(_dp)]
    lib.mf3d_last_error.restype = C.c_char_p
    lib.mf3d_status_string.restype = C.c_char_p
    lib.mf3d_status_string.argtypes = [C.c_int]
    lib.mf3d_last_launch_count.restype = C.c_longlong
    lib.mf3d_last_launch_count.argtypes = [vp]
    lib.mf3d_halo_map.restype = C.c_longlong
    lib.mf3d_halo_map.argtypes = [C.POINTER(BlockDesc), C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    lib.mf3d_halo_refresh_host.argtypes = [C.POINTER(BlockDesc), C.c_int, C.c_int, C.c_int, C.POINTER(_dp)]
    lib.mf3d_max_levels.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.mf3d_batch_create.argtypes = [C.POINTER(DomainDesc), C.c_int, C.POINTER(Params), C.POINTER(vp)]
    lib.mf3d_batch_solve_device.argtypes = [vp, C.POINTER(Fields), _dp, _dp, C.POINTER(SolveInfo), _dp, C.c_int]
    lib.mf3d_profile.argtypes = [vp, C.c_int]
    lib.mf3d_selftest_divide.argtypes = [_dp, _dp, C.c_longlong, _dp, _dp, C.c_int]
    lib.mf3d_server_create.argtypes = [C.POINTER(Params), C.c_double, C.c_int, C.POINTER(vp)]
    lib.mf3d_server_submit.argtypes = [vp, C.POINTER(DomainDesc), C.POINTER(Fields), C.c_double, C.c_double,
                                       C.POINTER(C.c_longlong)]
    lib.mf3d_server_poll.argtypes = [vp, C.c_longlong, C.POINTER(RequestInfo), C.c_int]
    lib.mf3d_server_stats.argtypes = [vp] + [C.POINTER(C.c_longlong)] * 4 + [C.POINTER(C.c_double),
                                                                          C.POINTER(C.c_longlong)]
    lib.mf3d_server_profile.argtypes = [vp] + [C.POINTER(C.c_double)] * 4 + [C.POINTER(C.c_longlong)] * 2
    lib.mf3d_server_clock.restype = C.c_double
    lib.mf3d_server_clock.argtypes = []
    lib.mf3d_server_destroy.argtypes = [vp]
    lib.mf3d_tecbin_info_of.argtypes = [vp, C.c_size_t, C.POINTER(TecbinInfo)]
    lib.mf3d_tecbin_size.restype = C.c_longlong
    lib.mf3d_tecbin_size.argtypes = [C.c_int] * 3
    lib.mf3d_tecbin_decode_device.argtypes = [vp, C.POINTER(TecbinInfo), C.POINTER(vp), C.c_int]
    lib.mf3d_tecbin_encode_device.argtypes = [C.c_int] * 7 + [vp] * 3 + [C.POINTER(vp), vp, C.c_int]
    lib.mf3d_profile_read.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                      C.POINTER(C.c_double)]
    lib.mf3d_rungek_2nd_device.argtypes = [vp, C.POINTER(Fields), C.POINTER(RkFields), C.c_double, C.c_double,
                                           C.c_int, C.c_int, C.c_double]
    lib.mf3d_calvel_device.argtypes = [vp, C.POINTER(Fields), C.c_double, C.c_double]
    lib.mf3d_field_exchange_map.restype = C.c_longlong
    lib.mf3d_field_exchange_map.argtypes = [C.POINTER(BlockDesc), C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    lib.mf3d_tuning.argtypes = [vp, C.c_int] + [C.POINTER(C.c_int)] * 4
    lib.mf3d_set_inlet.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_longlong]
    lib.mf3d_bind_old_velocity.argtypes = [vp, vp]
    lib.mf3d_set_wall_model.argtypes = [vp, C.c_double, C.c_double]
    lib.mf3d_bounds_device.argtypes = [vp, C.POINTER(Fields), C.c_double, C.c_double, C.c_int]
    lib.mf3d_test_fail_alloc.argtypes = [C.c_longlong]
    lib.mf3d_test_stall_copy.argtypes = [C.c_int, C.c_int]
    return lib


def load(path: str | None = None):
    """Load ``libmf3d.so``; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"native library {p} is missing: run `python -c 'import __graft_entry__ as g; g.build()'`"
            " (there is no CPU fallback)")
    lib = _declare(C.CDLL(p))
    if path is None:
        _lib = lib
    return lib


def last_error(lib) -> str:
    return lib.mf3d_last_error().decode()


def check(lib, status: int, what: str = "") -> int:
    """Raise on a negative status (the solve did not run)."""
    if status < 0:
        raise RuntimeError(f"{what}: {lib.mf3d_status_string(status).decode()} ({status}): {last_error(lib)}")
    return status
