"""The C-ABI libraries load on a CPU-only machine and export every entry point that
include/q2d_gpu.h declares (no compute call is made here)."""
import ctypes as C
import re
from pathlib import Path

from q2d_b200 import _abi

HDR = Path(__file__).resolve().parents[1] / "include" / "q2d_gpu.h"


def declared_functions():
    txt = HDR.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(q2d_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("q2d_gpu_create", "q2d_gpu_add_block", "q2d_gpu_set_bcs", "q2d_gpu_upload_prim",
                     "q2d_gpu_step", "q2d_gpu_download_prim", "q2d_gpu_errstr", "q2d_gpu_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_abi.build_library()))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_errstr_and_defaults_without_gpu():
    lib = _abi.load_library()
    assert lib.q2d_gpu_errstr(0) == b"ok"
    assert b"NaN" in lib.q2d_gpu_errstr(5)
    o = _abi.Options()
    lib.q2d_options_default(C.byref(o))
    assert o.riemann == 0 and o.n_rk == 1 and o.cfl == 0.5 and o.res_threshold == 1e-10
    assert o.itermax == 1000000000 and o.gas_gamma == 1.4


def test_oracle_mirrors_the_boundary():
    from oracle import oracle
    lib = oracle.load()
    for n in declared_functions():
        if n.startswith("q2d_gpu_") and n[8:] in ("create", "add_case", "add_block", "set_bcs",
                                                   "upload_prim", "set_case_time", "set_case_end",
                                                   "commit", "step", "case_info",
                                                   "download_prim", "destroy"):
            assert hasattr(lib, "q2d_oracle_" + n[8:])


def test_oracle_case_end():
    """A case's own fixed end (set_case_end): the case stops at that iteration, inside a
    multi-step call, while the case next to it runs on; a finished case stays finished."""
    from oracle import oracle
    from q2d_b200 import cases, make_options
    batch = [cases.ramp(16, 6, seed=2), cases.ramp(12, 6, seed=4)]
    s = oracle.solver(make_options(batch[0], itermax=100), batch)
    try:
        s.set_case_end(0, 4)
        assert [i["iter"] for i in s.step(6)] == [4, 6]
        assert [i["todo"] for i in s.step(3)] == [_abi.TODO_END, _abi.TODO_CONTINUE]
        assert s.info(0)["iter"] == 4
    finally:
        s.close()
