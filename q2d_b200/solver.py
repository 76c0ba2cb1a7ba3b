"""Host-side driver over the C ABI: the Python mirror of Q2D's Wrap_Setup / Wrap_Solve.

`Q2DSolver` performs the setup sequence of Q2D_setup (src/lib/driver/Wrap_Setup.f90:10-167:
options -> blocks + nodes + Cross_Section -> initial state -> bc records -> metrics) through
the q2d_gpu_* entry points, and `solve()` repeats Q2D_solve (Wrap_Solve.f90:10-34) while the
TODO flag asks for more steps, like the main loop of src/app/main.f90:47-50.
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional

import numpy as np

from . import _abi
from .cases import CaseSpec


class Q2DError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: status {status} {detail}".strip())


def make_options(case_or_opts, **overrides) -> _abi.Options:
    base = dict(case_or_opts.options) if isinstance(case_or_opts, CaseSpec) else dict(case_or_opts)
    base.update(overrides)
    return _abi.default_options(**base)


class Q2DSolver:
    """A set of cases advanced together through one library context.

    lib/prefix select the implementation behind the C ABI: the CUDA library
    (`q2d_gpu`, default) or another library exporting the same entry points. thermo_table =
    (h, cp), arrays on 1-K knots from 0 K, selects the thermally perfect gas
    (q2d_gpu_set_thermo_table)."""

    def __init__(self, options: _abi.Options, cases: Iterable[CaseSpec], lib=None,
                 prefix: str = "q2d_gpu", thermo_table=None):
        self.lib = lib if lib is not None else _abi.load_library()
        self.prefix = prefix
        self.options = options
        self.cases = list(cases)
        self.ctx = C.c_void_p()
        self._call("create", C.byref(self.ctx), C.byref(options))
        self.block_ids = []
        try:
            if thermo_table is not None:
                h, cp = (np.ascontiguousarray(t, dtype=np.float64) for t in thermo_table)
                if h.shape != cp.shape or h.ndim != 1:
                    raise ValueError("thermo_table: h and cp must be 1-D arrays of one length")
                self._call("set_thermo_table", self.ctx, len(h), _abi.dptr(h), _abi.dptr(cp))
            for cs in self.cases:
                cid = C.c_int()
                self._call("add_case", self.ctx, C.byref(cid))
                ids = []
                for b in cs.blocks:
                    nodes = np.ascontiguousarray(b.nodes, dtype=np.float64)
                    area = None if b.area is None else np.ascontiguousarray(b.area, dtype=np.float64)
                    bid = C.c_int()
                    self._call("add_block", self.ctx, cid.value, b.ni, b.nj, _abi.dptr(nodes),
                               None if area is None else _abi.dptr(area), C.byref(bid))
                    P = b.prim_ghost()
                    self._call("upload_prim", self.ctx, bid.value, _abi.dptr(P))
                    ids.append(bid.value)
                self.block_ids.append(ids)
                if cs.meta.get("restart_time") is not None:   # resume a time-accurate case
                    self._call("set_case_time", self.ctx, cid.value, float(cs.meta["restart_time"]))
                if cs.meta.get("iter_end"):   # the case's own fixed end
                    self._call("set_case_end", self.ctx, cid.value, int(cs.meta["iter_end"]))
                recs = _abi.bc_array(cs.bcs)
                self._call("set_bcs", self.ctx, cid.value, recs, len(cs.bcs))
            self._call("commit", self.ctx)
        except Exception:
            self.close()
            raise

    # -- plumbing -------------------------------------------------------------------------
    def _fn(self, name):
        return getattr(self.lib, f"{self.prefix}_{name}")

    def _call(self, name, *args):
        st = self._fn(name)(*args)
        if st != _abi.OK:
            detail = ""
            if self.prefix == "q2d_gpu" and self.ctx:
                msg = self.lib.q2d_gpu_last_error(self.ctx)
                detail = msg.decode() if msg else ""
            raise Q2DError(st, f"{self.prefix}_{name}", detail)
        return st

    # -- API ------------------------------------------------------------------------------
    def step(self, nsteps: int = 1, check: bool = True) -> list:
        infos = (_abi.StepInfo * max(len(self.cases), 1))()
        st = self._fn("step")(self.ctx, nsteps, infos)
        out = [infos[c].as_dict() for c in range(len(self.cases))]
        if check and st != _abi.OK:
            raise Q2DError(st, f"{self.prefix}_step", str([o["err_at"] for o in out if o["err"]]))
        return out

    SCHEDULES = ["tile 32x10", "tile 32x8", "tile 64x4",
                 "fp32-flux tile 32x10", "fp32-flux tile 32x8", "fp32-flux tile 64x4",
                 "fp32-flux tile 32x16", "fp32-flux tile 64x8", "fp32-flux difference tile 32x8"]

    def set_schedule(self, schedule) -> None:
        """Pins a schedule (index or name from SCHEDULES) without tuning (q2d_gpu_set_schedule)."""
        idx = self.SCHEDULES.index(schedule) if isinstance(schedule, str) else int(schedule)
        self._call("set_schedule", self.ctx, idx)

    @property
    def schedule(self) -> str:
        k = self.lib.q2d_gpu_get_schedule(self.ctx)
        return self.SCHEDULES[k] if k >= 0 else "unknown"

    def autotune(self, steps: int = 2) -> dict:
        """Times every stage-kernel schedule on this workload and keeps the fastest
        (q2d_gpu_autotune); the state is left unchanged."""
        idx = C.c_int()
        ms = C.c_float()
        self._call("autotune", self.ctx, steps, C.byref(idx), C.byref(ms))
        return {"schedule": self.SCHEDULES[idx.value], "ms_per_step": ms.value}

    def set_case_end(self, case: int, iter_end: int) -> None:
        """Gives a case its own fixed end: TODO = END once its iteration count reaches iter_end
        (0 clears it), besides the options' limits (q2d_gpu_set_case_end)."""
        self._call("set_case_end", self.ctx, case, int(iter_end))

    def info(self, case: int = 0) -> dict:
        s = _abi.StepInfo()
        self._call("case_info", self.ctx, case, C.byref(s))
        return s.as_dict()

    def prim(self, case: int = 0, block: int = 0) -> np.ndarray:
        b = self.cases[case].blocks[block]
        P = np.zeros((b.nj + 4, b.ni + 4, 4))
        self._call("download_prim", self.ctx, self.block_ids[case][block], _abi.dptr(P))
        return P[2:b.nj + 2, 2:b.ni + 2, :].copy()

    def prims(self) -> list:
        """Interior states of every block of every case, [case][block] -> (nj, ni, 4), read
        by one many-block transfer (q2d_gpu_download_prim_many)."""
        arrs, ids = [], []
        for c, cs in enumerate(self.cases):
            for k, b in enumerate(cs.blocks):
                arrs.append(np.zeros((b.nj + 4, b.ni + 4, 4)))
                ids.append(self.block_ids[c][k])
        ptrs = (C.POINTER(C.c_double) * max(len(arrs), 1))(*[_abi.dptr(a) for a in arrs])
        idv = (C.c_int * max(len(ids), 1))(*ids)
        self._call("download_prim_many", self.ctx, len(ids), idv, ptrs)
        out, k = [], 0
        for cs in self.cases:
            row = []
            for b in cs.blocks:
                row.append(arrs[k][2:b.nj + 2, 2:b.ni + 2, :].copy())
                k += 1
            out.append(row)
        return out

    def solve(self, max_calls: int = 10 ** 9, steps_per_call: int = 1) -> dict:
        """Runs until every case reports TODO = END (or an error)."""
        for _ in range(max_calls):
            infos = self.step(steps_per_call)
            if all(i["todo"] == _abi.TODO_END or i["err"] for i in infos):
                break
        return self.info(0)

    def close(self):
        if self.ctx:
            self._fn("destroy")(self.ctx)
            self.ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
