"""Test-side ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use this module; the oracle is the checker, never the thing shipped.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from multiflow3d_b200.abi import BlockDesc, Params, Fields, SolveInfo, RkFields

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

_dp = C.POINTER(C.c_double)
_lib = None


def build_oracle() -> str:
    src = os.path.join(ORACLE_DIR, "mf3d_oracle.cpp")
    if (not os.path.exists(ORACLE_SO)) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return ORACLE_SO


def load():
    global _lib
    if _lib is None:
        lib = C.CDLL(build_oracle())
        lib.orc_newsolv_mg.argtypes = [C.POINTER(BlockDesc), C.c_int, C.POINTER(Params),
                                       C.POINTER(Fields), C.c_double, C.c_double,
                                       C.POINTER(SolveInfo), _dp, C.c_int]
        lib.orc_mgkcyc.argtypes = [C.POINTER(BlockDesc), C.c_int, C.POINTER(Params),
                                   C.POINTER(_dp), C.POINTER(_dp)]
        lib.orc_exchangepp.argtypes = [C.POINTER(BlockDesc), C.c_int, C.c_int, C.c_int, C.POINTER(_dp)]
        lib.orc_apply_operator.argtypes = [C.POINTER(BlockDesc), C.c_int, C.c_int, C.c_int,
                                           C.POINTER(_dp), C.POINTER(_dp)]
        lib.orc_build_topology.argtypes = [C.c_int, _dp, C.POINTER(C.c_int), C.c_double,
                                           C.c_double, C.c_double, C.POINTER(BlockDesc)]
        lib.orc_rungek_2nd.argtypes = [C.POINTER(BlockDesc), C.c_int, C.POINTER(Params), C.POINTER(Fields),
                                       C.POINTER(RkFields), C.c_double, C.c_double, C.c_int, C.c_int, C.c_double]
        lib.orc_calvel.argtypes = [C.POINTER(BlockDesc), C.c_int, C.POINTER(Params), C.POINTER(Fields),
                                   C.c_double, C.c_double]
        lib.orc_exchange.argtypes = [C.POINTER(BlockDesc), C.c_int, C.POINTER(Params), C.POINTER(Fields), C.c_int]
        lib.orc_set_inlet.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_longlong]
        lib.orc_bind_old_velocity.argtypes = [C.c_int, C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp)]
        lib.orc_set_wall_model.argtypes = [C.c_double, C.c_double]
        lib.orc_bounds.argtypes = [C.POINTER(BlockDesc), C.c_int, C.POINTER(Params), C.POINTER(Fields), C.c_double,
                                   C.c_double, C.c_int]
        lib.orc_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def ptr_array(arrays):
    arr = (_dp * len(arrays))()
    for i, a in enumerate(arrays):
        arr[i] = a.ctypes.data_as(_dp)
    return arr
