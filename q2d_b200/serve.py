"""Serving: continuous batching of independent solves on one GPU.

The reference solves one domain per process, from input files to TODO = END
(src/app/main.f90:20-50, Wrap_Solve.f90:10-34). Here a request loop keeps many such solves
resident in one serving context (q2d_serve_* in include/q2d_gpu.h): requests that arrive
while others run are admitted as case slots and device memory free up (FIFO, memory-budget
admission), every resident case advances in the same captured step graphs, and a case is
retired when its residual has dropped by the requested factor or it reaches its iteration
cap (the fixed end), after its state has been read back.

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


def request_stream(rate: float, duration: float, seed: int = BASE_SEED + 5, cells_lo: float = 4e3,
                   cells_hi: float = 2e6, max_requests: Optional[int] = None) -> list:
    """Poisson arrivals at `rate` per second over `duration` seconds. Each request is a planar
    ramp or a quasi-2D nozzle (equal odds) with a log-normal cell count whose +-3 sigma range
    is [cells_lo, cells_hi], clipped to it."""
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
          realtime: bool = True) -> dict:
    """Runs the request loop until every request is retired (or rejected as larger than the
    whole budget). With realtime=False arrivals are taken as already due (a replay of a
    backlog), which makes the admission order independent of host timing."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    pending = deque(reqs)
    queue: deque = deque()
    active: dict = {}
    cell_updates = 0
    steps_calls = 0
    with ServeContext(options, device_bytes, max_cases, lib=lib) as sc:
        budget_cells = sc.free_cells()
        t0 = clock()
        busy = 0.0

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
            sc.step_async(steps_per_call)
            on_device = set(active.keys())   # cases admitted from here on join the next call
            steps_calls += 1
            admit_due()              # host work overlaps the steps in flight
            infos = sc.wait()
            busy += clock() - tb
            for cid in sorted(on_device):
                inf = infos[cid]
                if inf.todo == _abi.TODO_END or inf.err:
                    r = active.pop(cid)
                    r.iters = int(inf.iter)
                    r.err = int(inf.err)
                    r.residual_drop = inf.residual[0] / inf.residual0 if inf.residual0 > 0 else math.nan
                    if keep_results:
                        r.result = [sc.prim(cid, b) for b in range(len(r.case.blocks))]
                    sc.retire(cid)
                    r.done = clock() - t0
                    cell_updates += r.case.cells * r.iters
                    r.case = None if not keep_results else r.case
        makespan = clock() - t0
        launches = sc.launches()
    done = [r for r in reqs if not r.rejected]
    lat = np.array([r.latency for r in done]) if done else np.array([math.nan])
    return {
        "requests": len(reqs), "served": len(done), "rejected": sum(r.rejected for r in reqs),
        "errors": sum(1 for r in done if r.err),
        "cell_updates": int(cell_updates), "makespan_s": makespan, "busy_s": busy,
        "cell_updates_per_s": cell_updates / makespan if makespan > 0 else math.nan,
        "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
        "mean_latency_s": float(lat.mean()), "step_calls": steps_calls, "gpu_launches": launches,
        "budget_cells": int(budget_cells),
    }
