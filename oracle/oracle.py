"""ctypes binding of the CPU oracle (oracle/build/libq2d_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, never by the q2d_b200 package. The oracle exports the q2d_gpu_* entry
points under the q2d_oracle_* prefix, so q2d_b200.solver.Q2DSolver drives it unchanged.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "build" / "libq2d_oracle.so"

_LIB = None


def build(force: bool = False) -> Path:
    srcs = [HERE / "q2d_oracle.cpp", HERE / "q2d_oracle.h", HERE / "Makefile",
            HERE.parent / "include" / "q2d_gpu.h"]
    if force or not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB_PATH


def load():
    global _LIB
    if _LIB is None:
        from q2d_b200 import _abi
        build()
        lib = C.CDLL(str(LIB_PATH))
        _abi._declare(lib, "q2d_oracle", C.c_void_p)
        lib.q2d_oracle_set_threads.restype = C.c_int
        lib.q2d_oracle_set_threads.argtypes = [C.c_int]
        lib.q2d_oracle_limiter.restype = C.c_double
        lib.q2d_oracle_limiter.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.q2d_oracle_riemann.restype = None
        lib.q2d_oracle_riemann.argtypes = [C.c_int, C.POINTER(_abi.Options),
                                           C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.c_double, C.c_double, C.POINTER(C.c_double)]
        lib.q2d_oracle_thermo_tab.restype = C.c_int
        lib.q2d_oracle_thermo_tab.argtypes = [C.c_int, C.POINTER(_abi.Options), C.c_int] + \
            [C.POINTER(C.c_double)] * 4 + [C.c_double, C.c_double, C.POINTER(C.c_double)]
        lib.q2d_oracle_riemann_sd.restype = None
        lib.q2d_oracle_riemann_sd.argtypes = [C.c_int, C.POINTER(_abi.Options),
                                              C.POINTER(C.c_double), C.POINTER(C.c_double),
                                              C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]
        lib.q2d_oracle_sd_tramel.restype = C.c_double
        lib.q2d_oracle_sd_tramel.argtypes = [C.c_double] * 5
        lib.q2d_oracle_shock_sensor.restype = C.c_int
        lib.q2d_oracle_shock_sensor.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        lib.q2d_oracle_get_geometry.restype = C.c_int
        lib.q2d_oracle_get_geometry.argtypes = [C.c_void_p, C.c_int] + [C.POINTER(C.c_double)] * 4
        _LIB = lib
    return _LIB


def solver(options, cases, **kw):
    """A Q2DSolver over the oracle library (keywords as Q2DSolver's, e.g. thermo_table)."""
    from q2d_b200.solver import Q2DSolver
    return Q2DSolver(options, cases, lib=load(), prefix="q2d_oracle", **kw)


def set_threads(n: int) -> int:
    return load().q2d_oracle_set_threads(n)
