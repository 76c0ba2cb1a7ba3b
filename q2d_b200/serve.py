"""Serving: continuous batching of independent solves on one GPU.

The reference solves one domain per process, from input files to TODO = END
(src/app/main.f90:20-50, Wrap_Solve.f90:10-34). Here a request loop keeps many such solves
resident in one serving context (q2d_serve_* in include/q2d_gpu.h): requests that arrive
while others run are admitted as case slots and device memory free up (FIFO, memory-budget
admission), every resident case advances in the same captured step graphs, and a case is
retired when its residual has dropped by the requested factor or it reaches its fixed end (the
context's iteration cap, or a per-request budget of cell-updates), after its state has been read
back when the caller keeps results.

Admission does its host work (validation, metrics) while the GPU runs the previous steps; its
device writes are applied at the next step call.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _abi
from .cases import BASE_SEED, CaseSpec, request_case
from .solver import Q2DError


def wire(case: CaseSpec) -> dict:
    """The request as the C ABI takes it (the layout a client would send: node coordinates,
    the state in the reference's ghosted P array, the cross-sections and the bc.txt records as
    q2d_bc_rec), built once per case and kept with it."""
    w = getattr(case, "_wire", None)
    if w is not None:
        return w
    nb = len(case.blocks)
    PD = C.POINTER(C.c_double)
    w = {"nb": nb, "ni": (C.c_int * nb)(*[b.ni for b in case.blocks]),
         "nj": (C.c_int * nb)(*[b.nj for b in case.blocks]),
         "nodes": (PD * nb)(), "areas": (PD * nb)(), "prims": (PD * nb)(), "keep": []}
    for k, b in enumerate(case.blocks):
        nd = np.ascontiguousarray(b.nodes, dtype=np.float64)
        P = b.prim_ghost(ghosts=None)
        w["keep"] += [nd, P]
        w["nodes"][k] = _abi.dptr(nd)
        w["prims"][k] = _abi.dptr(P)
        if b.area is not None:
            a = np.ascontiguousarray(b.area, dtype=np.float64)
            w["keep"].append(a)
            w["areas"][k] = _abi.dptr(a)
    w["recs"] = _abi.bc_array(case.bcs)
    case._wire = w
    return w


class ServeContext:
    """A serving context: case slots over device pools sized from a byte budget."""

    def __init__(self, options: _abi.Options, device_bytes: int, max_cases: int, lib=None):
        self.lib = lib if lib is not None else _abi.load_library()
        self.options = options
        self.max_cases = max_cases
        self.ctx = C.c_void_p()
        st = self.lib.q2d_serve_create(C.byref(self.ctx), C.byref(options), int(device_bytes), int(max_cases))
        if st != _abi.OK:
            raise Q2DError(st, "q2d_serve_create", self.lib.q2d_gpu_errstr(st).decode())
        self.cases: dict[int, CaseSpec] = {}
        self._infos = (_abi.StepInfo * max_cases)()

    def _check(self, st, where):
        if st != _abi.OK:
            raise Q2DError(st, where, self.lib.q2d_gpu_last_error(self.ctx).decode())

    def admit(self, case: CaseSpec) -> Optional[int]:
        """Admits a case; returns its slot, or None when slots or memory are exhausted."""
        w = wire(case)
        cid = C.c_int(-1)
        st = self.lib.q2d_serve_admit(self.ctx, w["nb"], w["ni"], w["nj"], w["nodes"], w["areas"], w["prims"],
                                      w["recs"], len(case.bcs), C.byref(cid))
        if st == _abi.ERR_CAPACITY:
            return None
        self._check(st, "q2d_serve_admit")
        self.cases[cid.value] = case
        return cid.value

    def set_end(self, cid: int, iter_end: int) -> None:
        """The case's own fixed end: it reports TODO = END at iteration iter_end, inside a
        multi-step call (q2d_gpu_set_case_end)."""
        self._check(self.lib.q2d_gpu_set_case_end(self.ctx, cid, int(iter_end)), "q2d_gpu_set_case_end")

    def retire(self, cid: int) -> None:
        self._check(self.lib.q2d_serve_retire(self.ctx, cid), "q2d_serve_retire")
        self.cases.pop(cid, None)

    def step_async(self, nsteps: int) -> None:
        self._check(self.lib.q2d_gpu_step_async(self.ctx, nsteps), "q2d_gpu_step_async")

    def wait(self) -> list:
        """Per-slot step info (the returned status of individual cases is in 'err')."""
        st = self.lib.q2d_gpu_wait(self.ctx, self._infos)
        if st == _abi.ERR_CUDA:
            self._check(st, "q2d_gpu_wait")
        return [self._infos[c] for c in range(self.max_cases)]

    def prim(self, cid: int, block: int = 0) -> np.ndarray:
        b = self.cases[cid].blocks[block]
        bid = C.c_int()
        self._check(self.lib.q2d_serve_block_id(self.ctx, cid, block + 1, C.byref(bid)), "q2d_serve_block_id")
        P = np.zeros((b.nj + 4, b.ni + 4, 4))
        self._check(self.lib.q2d_gpu_download_prim(self.ctx, bid.value, _abi.dptr(P)), "q2d_gpu_download_prim")
        return P[2:b.nj + 2, 2:b.ni + 2, :].copy()

    def prims_many(self, cids: list, buffer: Optional[np.ndarray] = None) -> list:
        """Interior states of several resident cases, [case][block] -> (nj, ni, 4), read back by
        one many-block transfer (q2d_gpu_download_prim_many). With `buffer` (a float64 array,
        best in page-locked memory) the ghosted arrays of the transfer are carved out of it while
        it has room, so that the returned views stay valid until the buffer is reused."""
        arrs, ids = [], []
        used = 0
        for cid in cids:
            for k, b in enumerate(self.cases[cid].blocks):
                bid = C.c_int()
                self._check(self.lib.q2d_serve_block_id(self.ctx, cid, k + 1, C.byref(bid)), "q2d_serve_block_id")
                n = (b.nj + 4) * (b.ni + 4) * 4
                if buffer is not None and used + n <= buffer.size:
                    arrs.append(buffer[used:used + n].reshape(b.nj + 4, b.ni + 4, 4))
                    used += n
                else:
                    arrs.append(np.empty((b.nj + 4, b.ni + 4, 4)))
                ids.append(bid.value)
        if ids:
            ptrs = (C.POINTER(C.c_double) * len(arrs))(*[_abi.dptr(a) for a in arrs])
            idv = (C.c_int * len(ids))(*ids)
            self._check(self.lib.q2d_gpu_download_prim_many(self.ctx, len(ids), idv, ptrs),
                        "q2d_gpu_download_prim_many")
        out, k = [], 0
        for cid in cids:
            row = []
            for b in self.cases[cid].blocks:
                row.append(arrs[k][2:b.nj + 2, 2:b.ni + 2, :])
                k += 1
            out.append(row)
        return out

    def free_cells(self) -> int:
        return int(self.lib.q2d_serve_free_cells(self.ctx))

    def launches(self) -> int:
        return int(self.lib.q2d_gpu_launch_count(self.ctx))

    def close(self) -> None:
        if self.ctx:
            self.lib.q2d_gpu_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ------------------------------------------------------------------------------------------
# request stream
# ------------------------------------------------------------------------------------------
@dataclass
class Request:
    rid: int
    arrival: float               # seconds from the start of the stream
    kind: str                    # "ramp" or "nozzle"
    cells: int                   # requested cells (the generated grid is close to it)
    seed: int
    case: Optional[CaseSpec] = None
    admitted: float = math.nan
    done: float = math.nan
    iters: int = 0
    residual_drop: float = math.nan
    err: int = 0
    rule: str = ""               # why it retired: "drop", "end" or "error"
    rejected: bool = False
    result: Optional[list] = None
    meta: dict = field(default_factory=dict)

    def build(self) -> CaseSpec:
        """The request's payload: the case and its C-ABI layout (client side)."""
        if self.case is None:
            self.case = request_case(self.kind, self.cells, np.random.default_rng(self.seed))
            wire(self.case)
        return self.case

    @property
    def latency(self) -> float:
        return self.done - self.arrival

    @property
    def queueing(self) -> float:
        return self.admitted - self.arrival

    @property
    def service(self) -> float:
        return self.done - self.admitted


def request_stream(rate: float, duration: float, seed: int = BASE_SEED + 5, cells_lo: float = 4e3,
                   cells_hi: float = 2e6, max_requests: Optional[int] = None,
                   distinct: Optional[int] = None) -> list:
    """Poisson arrivals at `rate` per second over `duration` seconds. Each request is a planar
    ramp or a quasi-2D nozzle (equal odds) with a log-normal cell count whose +-3 sigma range
    is [cells_lo, cells_hi], clipped to it. With `distinct`, request k carries the payload
    (kind, cells, seed) of request k mod distinct: a long stream replays that many distinct
    seeded cases, so that their payloads can be held in host memory."""
    rng = np.random.default_rng(seed)
    mu = 0.5 * (math.log(cells_lo) + math.log(cells_hi))
    sigma = (math.log(cells_hi) - math.log(cells_lo)) / 6.0
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration or (max_requests is not None and len(out) >= max_requests):
            break
        cells = int(np.clip(rng.lognormal(mu, sigma), cells_lo, cells_hi))
        kind = "ramp" if rng.random() < 0.5 else "nozzle"
        out.append(Request(len(out), t, kind, cells, int(rng.integers(1 << 31))))
    if distinct:
        for r in out[distinct:]:
            src = out[r.rid % distinct]
            r.kind, r.cells, r.seed = src.kind, src.cells, src.seed
    return out


def serve_options(precision: int = _abi.PREC_FP32_FLUX, itermax: int = 2000, drop: float = 1e-8,
                  **kw) -> _abi.Options:
    """Options shared by every served case: MUSCL van Leer + HLLC, SSP-RK3, CFL 0.5, local
    time stepping, area-variation sources (zero for cases without a cross-section), retire on
    a relative residual drop of `drop` or at `itermax` iterations."""
    base = dict(limiter="vanleer", riemann="HLLC", n_rk=3, cfl=0.5, source="area_variation",
                precision=precision, res_relative=1, res_threshold=drop, itermax=itermax,
                res_diter=1, sol_diter=10 ** 9)
    base.update(kw)
    return _abi.default_options(**base)


def serve(requests: list, options: _abi.Options, device_bytes: int, max_cases: int = 1024,
          steps_per_call: int = 10, keep_results: bool = False, lib=None, clock=time.perf_counter,
          realtime: bool = True, end_cell_updates: Optional[float] = None,
          result_sink=None, readback_buffer: Optional[np.ndarray] = None) -> dict:
    """Runs the request loop until every request is retired (or rejected as larger than the
    whole budget). With realtime=False arrivals are taken as already due (a replay of a
    backlog), which makes the admission order independent of host timing.

    A request retires on the residual drop of the options, on an error, or at its fixed end:
    the options' iteration cap or, with end_cell_updates, the iteration at which its cells
    times its iterations first reach that budget (set on the device at admission, so that the
    case stops there inside a multi-step call). With
    keep_results the states of the cases retiring after a step call are read back in one
    many-block transfer before they are retired; that read-back is inside their latency. The
    states are kept in Request.result, or handed to result_sink(request, states) when given
    (a client that takes the result away); with readback_buffer the states handed to the sink
    are views into it, valid until the sink returns."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    pending = deque(reqs)
    queue: deque = deque()
    active: dict = {}
    cell_updates = 0
    steps_calls = 0
    readback_bytes = 0
    with ServeContext(options, device_bytes, max_cases, lib=lib) as sc:
        budget_cells = sc.free_cells()
        t0 = clock()
        busy = 0.0
        t_admit = t_readback = t_retire = t_launch = 0.0

        def now():
            return clock() - t0 if realtime else math.inf

        def admit_due():
            t = now()
            while pending and pending[0].arrival <= t:
                queue.append(pending.popleft())
            while queue:
                r = queue[0]
                case = r.build()
                if case.cells > budget_cells:
                    r.rejected = True
                    queue.popleft()
                    continue
                cid = sc.admit(case)
                if cid is None:
                    break
                r.admitted = clock() - t0
                if end_cell_updates is not None:
                    r.meta["end_iter"] = max(1, math.ceil(end_cell_updates / case.cells))
                    sc.set_end(cid, r.meta["end_iter"])
                active[cid] = r
                queue.popleft()

        admit_due()
        while pending or queue or active:
            if not active:
                if pending and realtime:
                    time.sleep(max(0.0, pending[0].arrival - (clock() - t0)))
                admit_due()
                continue
            tb = clock()
            sc.step_async(steps_per_call)   # applies admissions and retirements, then launches
            t_launch += clock() - tb
            on_device = set(active.keys())   # cases admitted from here on join the next call
            steps_calls += 1
            ta = clock()
            admit_due()              # host work overlaps the steps in flight
            t_admit += clock() - ta
            infos = sc.wait()
            busy += clock() - tb
            leaving = []
            for cid in sorted(on_device):
                inf = infos[cid]
                r = active[cid]
                end_iter = r.meta.get("end_iter")
                if inf.err:
                    r.rule = "error"
                elif inf.todo == _abi.TODO_END:
                    fixed = inf.iter >= options.itermax or (end_iter is not None and inf.iter >= end_iter)
                    r.rule = "end" if fixed else "drop"
                else:
                    continue
                r.iters = int(inf.iter)
                r.err = int(inf.err)
                r.residual_drop = inf.residual[0] / inf.residual0 if inf.residual0 > 0 else math.nan
                leaving.append(cid)
            if leaving:
                tr = clock()
                if keep_results:
                    buf = readback_buffer if result_sink is not None else None
                    for cid, res in zip(leaving, sc.prims_many(leaving, buf)):
                        readback_bytes += sum(x.nbytes for x in res)
                        if result_sink is not None:
                            result_sink(active[cid], res)
                        else:
                            active[cid].result = res
                t_readback += clock() - tr
                tr = clock()
                for cid in leaving:
                    r = active.pop(cid)
                    sc.retire(cid)
                    r.done = clock() - t0
                    cell_updates += r.case.cells * r.iters
                    r.case = None if not keep_results or result_sink is not None else r.case
                t_retire += clock() - tr
        makespan = clock() - t0
        launches = sc.launches()
    done = [r for r in reqs if not r.rejected]

    def pct(xs, q):
        return float(np.percentile(np.array(xs), q)) if xs else math.nan
    lat = [r.latency for r in done]
    que = [r.queueing for r in done]
    ser = [r.service for r in done]
    rules = {k: sum(1 for r in done if r.rule == k) / max(1, len(done)) for k in ("drop", "end", "error")}
    drops = [r.residual_drop for r in done if math.isfinite(r.residual_drop)]
    return {
        "requests": len(reqs), "served": len(done), "rejected": sum(r.rejected for r in reqs),
        "errors": sum(1 for r in done if r.err),
        "cell_updates": int(cell_updates), "makespan_s": makespan, "busy_s": busy,
        "cell_updates_per_s": cell_updates / makespan if makespan > 0 else math.nan,
        "p50_latency_s": pct(lat, 50), "p99_latency_s": pct(lat, 99),
        "mean_latency_s": float(np.mean(lat)) if lat else math.nan,
        "p50_queueing_s": pct(que, 50), "p99_queueing_s": pct(que, 99),
        "p50_service_s": pct(ser, 50), "p99_service_s": pct(ser, 99),
        "retired_by": rules, "median_residual_drop": pct(drops, 50),
        "readback_bytes": int(readback_bytes),
        "host_s": {"apply_and_launch": t_launch, "admission_during_steps": t_admit, "readback": t_readback,
                   "retire": t_retire},
        "step_calls": steps_calls, "gpu_launches": launches,
        "budget_cells": int(budget_cells),
    }
