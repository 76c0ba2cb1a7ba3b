"""ctypes mirror of include/q2d_gpu.h (structs, constants) and the loader of the CUDA library.

The structures follow the C header field by field; see the header for the reference
(Q2D Fortran) interface each entry point replaces.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
REPO = ROOT.parent
LIB_DIR = ROOT / "lib"
LIB_PATH = LIB_DIR / "libq2d_gpu.so"

# status codes
OK, ERR_BADARG, ERR_OOM, ERR_CUDA, ERR_NONPHYSICAL, ERR_NAN, ERR_TIMEOUT, ERR_UNSUPPORTED, \
    ERR_CAPACITY = range(9)

LIM = {"iord": 0, "none": 0, "first-order": 0, "minmod": 1, "vanleer": 2, "vanalbada": 3,
       "mc": 4, "superbee": 5, "LIMO3": 6}
RIEMANN = {"HLLC": 0, "HLLE": 1, "LLF": 2, "Rusanov": 2, "SLAU": 3, "SLAU2": 4, "HLLC+": 5, "HLLE++": 6,
           "HLLEM": 7, "HLLC Rotated": 8, "PLLF": 9, "exact": 10, "Exact": 10, "Hanel": 11, "AUSM+": 12,
           "AUSM+-up": 13, "AUSM+-up2": 14}
SRC = {"none": 0, "axisymmetric": 1, "area_variation": 2}
PREC_FP64, PREC_FP32_FLUX = 0, 1
TODO_CONTINUE, TODO_IO, TODO_END = 1, 2, 3
NORMAL_DIR = sys.float_info.max  # 'normal' keyword sentinel of the flow angle


class Options(C.Structure):
    _fields_ = [
        ("limiter", C.c_int), ("riemann", C.c_int), ("n_rk", C.c_int),
        ("time_accurate", C.c_int), ("source", C.c_int), ("precision", C.c_int),
        ("rampa_iter", C.c_int), ("res_diter", C.c_int), ("sol_diter", C.c_int),
        ("res_relative", C.c_int),
        ("itermax", C.c_longlong),
        ("cfl", C.c_double), ("res_threshold", C.c_double), ("time_threshold", C.c_double),
        ("sol_dtime", C.c_double), ("gas_R", C.c_double), ("gas_gamma", C.c_double),
        ("irs_beta", C.c_double), ("shock_detector", C.c_int), ("riemann_minf", C.c_double),
    ]


class BCRec(C.Structure):
    _fields_ = [
        ("b", C.c_int), ("i", C.c_int), ("j", C.c_int), ("f", C.c_int), ("type", C.c_int),
        ("bs", C.c_int), ("is_", C.c_int), ("js", C.c_int), ("fs", C.c_int),
        ("d11", C.c_int), ("d12", C.c_int), ("d21", C.c_int), ("d22", C.c_int),
        ("T0", C.c_double), ("p0", C.c_double), ("pamb", C.c_double), ("mach", C.c_double),
        ("alpha", C.c_double), ("rel_fac", C.c_double),
    ]


class StepInfo(C.Structure):
    _fields_ = [
        ("dtglobal", C.c_double), ("time", C.c_double), ("iter", C.c_longlong),
        ("residual", C.c_double * 4), ("residual0", C.c_double),
        ("todo", C.c_int), ("err", C.c_int),
        ("err_b", C.c_int), ("err_i", C.c_int), ("err_j", C.c_int), ("err_stage", C.c_int),
    ]

    def as_dict(self) -> dict:
        return {"dtglobal": self.dtglobal, "time": self.time, "iter": self.iter,
                "residual": list(self.residual), "residual0": self.residual0,
                "todo": self.todo, "err": self.err,
                "err_at": (self.err_b, self.err_i, self.err_j, self.err_stage)}


def default_options(**kw) -> Options:
    """Reference defaults (Register_Numerics.f90:31-76, Register_Sim_Param.f90:26-29,
    Register_IO.f90:26-35) with the keyword overrides given."""
    o = Options()
    o.limiter = 0
    o.riemann = 0
    o.n_rk = 1
    o.time_accurate = 0
    o.source = 0
    o.precision = PREC_FP64
    o.rampa_iter = 0
    o.res_diter = 1
    o.sol_diter = 1000000000
    o.res_relative = 0
    o.itermax = 1000000000
    o.cfl = 0.5
    o.res_threshold = 1e-10
    o.time_threshold = 1e30
    o.sol_dtime = 1e30
    o.gas_R = 287.0
    o.gas_gamma = 1.4
    o.irs_beta = 0.0
    o.shock_detector = 0
    o.riemann_minf = 0.0
    for k, v in kw.items():
        if isinstance(v, str):
            v = {"limiter": LIM, "riemann": RIEMANN, "source": SRC}[k][v]
        setattr(o, k, v)
    return o


def options_copy(o: Options, **kw) -> Options:
    n = Options()
    C.memmove(C.byref(n), C.byref(o), C.sizeof(Options))
    for k, v in kw.items():
        setattr(n, k, v)
    return n


def bc_array(recs) -> "C.Array":
    arr = (BCRec * max(len(recs), 1))()
    for k, r in enumerate(recs):
        for name, val in r.items():
            setattr(arr[k], "is_" if name == "is" else name, val)
    return arr


def _declare(lib: C.CDLL, prefix: str, ctx_t) -> None:
    P = C.POINTER
    sig = {
        "create": (C.c_int, [P(ctx_t), P(Options)]),
        "add_case": (C.c_int, [ctx_t, P(C.c_int)]),
        "add_block": (C.c_int, [ctx_t, C.c_int, C.c_int, C.c_int, P(C.c_double), P(C.c_double),
                                P(C.c_int)]),
        "set_bcs": (C.c_int, [ctx_t, C.c_int, P(BCRec), C.c_int]),
        "upload_prim": (C.c_int, [ctx_t, C.c_int, P(C.c_double)]),
        "set_case_time": (C.c_int, [ctx_t, C.c_int, C.c_double]),
        "set_case_end": (C.c_int, [ctx_t, C.c_int, C.c_longlong]),
        "set_thermo_table": (C.c_int, [ctx_t, C.c_int, P(C.c_double), P(C.c_double)]),
        "commit": (C.c_int, [ctx_t]),
        "step": (C.c_int, [ctx_t, C.c_int, P(StepInfo)]),
        "case_info": (C.c_int, [ctx_t, C.c_int, P(StepInfo)]),
        "download_prim": (C.c_int, [ctx_t, C.c_int, P(C.c_double)]),
        "destroy": (None, [ctx_t]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, f"{prefix}_{name}")
        fn.restype = res
        fn.argtypes = args


def build_library(force: bool = False) -> Path:
    """Compiles the CUDA library in-tree for sm_100a (make in q2d_b200/csrc)."""
    csrc = ROOT / "csrc"
    if force or not LIB_PATH.exists() or _stale(LIB_PATH, csrc):
        subprocess.run(["make", "-C", str(csrc), "-j8"], check=True)
    return LIB_PATH


def _stale(target: Path, src_dir: Path) -> bool:
    t = target.stat().st_mtime
    files = list(src_dir.glob("*.cu")) + list(src_dir.glob("*.cuh")) + list(src_dir.glob("*.h")) \
        + list(src_dir.glob("*.cpp")) + list((ROOT / "host").glob("*.cpp")) \
        + [REPO / "include" / "q2d_gpu.h", src_dir / "Makefile"]
    return any(f.exists() and f.stat().st_mtime > t for f in files)


_LIB = None


def load_library() -> C.CDLL:
    """Loads libq2d_gpu.so (building it first when it is missing). There is no fallback:
    without the CUDA library the package cannot run."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        build_library()
    lib = C.CDLL(str(LIB_PATH))
    _declare(lib, "q2d_gpu", C.c_void_p)
    lib.q2d_gpu_errstr.restype = C.c_char_p
    lib.q2d_gpu_errstr.argtypes = [C.c_int]
    lib.q2d_gpu_last_error.restype = C.c_char_p
    lib.q2d_gpu_last_error.argtypes = [C.c_void_p]
    lib.q2d_gpu_num_cases.restype = C.c_int
    lib.q2d_gpu_num_cases.argtypes = [C.c_void_p]
    lib.q2d_gpu_num_cells.restype = C.c_longlong
    lib.q2d_gpu_num_cells.argtypes = [C.c_void_p]
    lib.q2d_gpu_launch_count.restype = C.c_longlong
    lib.q2d_gpu_launch_count.argtypes = [C.c_void_p]
    lib.q2d_gpu_step_async.restype = C.c_int
    lib.q2d_gpu_step_async.argtypes = [C.c_void_p, C.c_int]
    lib.q2d_gpu_wait.restype = C.c_int
    lib.q2d_gpu_wait.argtypes = [C.c_void_p, C.POINTER(StepInfo)]
    lib.q2d_gpu_autotune.restype = C.c_int
    lib.q2d_gpu_autotune.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float)]
    lib.q2d_gpu_residual_norm_noalloc.restype = C.c_int
    lib.q2d_gpu_residual_norm_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_longlong,
                                                  C.c_void_p, C.c_void_p]
    lib.q2d_gpu_prepare.restype = C.c_int
    lib.q2d_gpu_prepare.argtypes = [C.c_void_p, C.c_int]
    lib.q2d_gpu_stream.restype = C.c_void_p
    lib.q2d_gpu_stream.argtypes = [C.c_void_p]
    lib.q2d_gpu_set_schedule.restype = C.c_int
    lib.q2d_gpu_set_schedule.argtypes = [C.c_void_p, C.c_int]
    lib.q2d_gpu_get_schedule.restype = C.c_int
    lib.q2d_gpu_get_schedule.argtypes = [C.c_void_p]
    lib.q2d_options_default.restype = None
    lib.q2d_options_default.argtypes = [C.POINTER(Options)]
    PD = C.POINTER(C.POINTER(C.c_double))
    for name in ("upload_prim_many", "download_prim_many"):
        fn = getattr(lib, f"q2d_gpu_{name}")
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), PD]
    lib.q2d_serve_create.restype = C.c_int
    lib.q2d_serve_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Options), C.c_ulonglong, C.c_int]
    lib.q2d_serve_admit.restype = C.c_int
    lib.q2d_serve_admit.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), PD, PD, PD,
                                    C.POINTER(BCRec), C.c_int, C.POINTER(C.c_int)]
    lib.q2d_serve_retire.restype = C.c_int
    lib.q2d_serve_retire.argtypes = [C.c_void_p, C.c_int]
    lib.q2d_serve_block_id.restype = C.c_int
    lib.q2d_serve_block_id.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]
    lib.q2d_serve_free_cells.restype = C.c_longlong
    lib.q2d_serve_free_cells.argtypes = [C.c_void_p]
    _LIB = lib
    return lib


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))
