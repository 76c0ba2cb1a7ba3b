#!/usr/bin/env python
"""Benchmark of the Q2D explicit residual/update path on B200.

Workload (one "step" = one explicit SSP-RK3 time step — 3 fused stage kernels including the
ghost fill, MUSCL + HLLC fluxes, boundary fluxes, area-variation sources, the RK update, the
local time step and the residual norm — over every case of the batch):
  the batched quasi-2D area-variation nozzles: 4096 independent cases, Nx ~ lognormal clipped
  to [64, 1024], Ny ~ U{8..64}, A(x) = A_t (1 + k (x - x_t)^2), p0 ~ U[2, 10] bar,
  T0 ~ U[300, 800] K, van Leer + HLLC, local time stepping; synthetic seeded inputs with the
  layout of the reference's planar-nozzle case. Computed in the FP32-flux / FP64-state form;
  the plain FP64 form of the same batch is timed beside it.

Output: one JSON line (rank 0). `--impl reference` times the CPU oracle (the C++ restatement
of the reference's OpenMP loops, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "cell-updates/s batched+served vs plain FP64 on 1 B200; p50/p99 solve latency"
UNIT = "cell-updates/s"
# Algorithmic bytes per cell-update (one SSP-RK3 step): per stage read state 32 + U^n 32 +
# write 32 + dt 8 + node geometry 16 = 120, plus the dt pass 56, plus 16 per stage for the
# area-variation geometry (Gx, Gy): 3 * (120 + 16) + 56 = 464.
B_ALG = 464.0
STAGES = 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cases", type=int, default=4096)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--schedule", type=int, default=None,
                    help="pin the stage-kernel schedule of the headline leg instead of autotuning")
    ap.add_argument("--form", default="fp32-flux", choices=["fp32-flux", "fp64"],
                    help="precision form of the headline leg (profiling of the plain FP64 kernel)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="Poisson arrivals per second")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="length of the arrival window")
    ap.add_argument("--serve-end", type=float, default=1.0e7,
                    help="fixed end of a request: its cells x iterations budget (cell-updates)")
    ap.add_argument("--serve-gb", type=float, default=24.0, help="device-memory budget of the pools")
    ap.add_argument("--serve-seq", type=int, default=64, help="requests solved one after another in FP64")
    ap.add_argument("--serve-distinct", type=int, default=512, help="distinct seeded payloads of the stream")
    ap.add_argument("--serve-readback-gb", type=float, default=2.0,
                    help="page-locked host buffer the results of each step call are read back into")
    return ap.parse_args()


from q2d_b200.replicas import dist_env  # noqa: E402  (one process per GPU, replicas)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        try:
            rows = [r.split(",") for r in Path(self.out.name).read_text().strip().splitlines()]
        except Exception:
            rows = []
        rows = [[x.strip() for x in r] for r in rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def read_traffic(schedule):
    """DRAM bytes (read + write) per stage launch of the full batch, from the ncu summary of
    the stage kernel under profiles/ (a smaller batch captured and scaled by cells), when that
    summary holds a capture taken with the same schedule (lines "- schedule: S" followed by
    "- dram_bytes_per_launch_full_batch: B"); otherwise None."""
    name = ("stage32d_kernel_batched_nozzles.md" if "difference" in schedule else
            "stage32_kernel_batched_nozzles.md" if schedule.startswith("fp32-flux") else
            "stage_kernel_fp64_batched_nozzles.md")
    f = REPO / "profiles" / name
    try:
        cur = None
        for line in f.read_text().splitlines():
            if line.startswith("- schedule:"):
                cur = line.split(":", 1)[1].strip()
            elif line.startswith("- dram_bytes_per_launch_full_batch:") and cur == schedule:
                return float(line.split(":", 1)[1])
        return None
    except Exception:
        return None


def batch_cases(n, rank):
    from q2d_b200 import cases
    from q2d_b200.replicas import rank_seed
    return cases.area_nozzle_batch(n=n, seed=rank_seed(cases.BASE_SEED + 3, rank))


def time_device(lib, solver, K):
    """K steps in one captured graph, CUDA events on the library's stream."""
    import torch
    stream = torch.cuda.ExternalStream(lib.q2d_gpu_stream(solver.ctx))
    assert lib.q2d_gpu_prepare(solver.ctx, K) == 0
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    n0 = lib.q2d_gpu_launch_count(solver.ctx)
    ev0.record(stream)
    st = lib.q2d_gpu_step_async(solver.ctx, K)
    ev1.record(stream)
    lib.q2d_gpu_wait(solver.ctx, None)
    torch.cuda.synchronize()
    assert st == 0, st
    return ev0.elapsed_time(ev1), lib.q2d_gpu_launch_count(solver.ctx) - n0


def cpu_baseline(batch, budget_s=12.0):
    """The CPU oracle (all host threads) on a bounded sample of the workload."""
    from oracle import oracle
    from q2d_b200 import make_options
    threads = oracle.set_threads(os.cpu_count() or 1)
    sample = batch[:256]
    cells = sum(c.cells for c in sample)
    s = oracle.solver(make_options(sample[0]), sample)
    try:
        s.step(1)   # first step (setup, dt)
        t0 = time.perf_counter()
        n = 0
        while time.perf_counter() - t0 < budget_s and n < 200:
            s.step(1)
            n += 1
        dt = time.perf_counter() - t0
    finally:
        s.close()
    return {"value": cells * n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(sample)} of the batch's cases ({cells} cells) x {n} steps, "
                      f"{dt:.1f} s, C++ oracle -O3 OpenMP"}


def serving_leg(args, lib, fp64_batched=None):
    """The served request stream: Poisson arrivals (args.serve_rate per second over
    args.serve_seconds) of planar ramps and quasi-2D nozzles with log-normal sizes in [4e3, 2e6]
    cells, admitted by memory budget into one serving context (FP32-flux / FP64-state). A request
    retires on a 1e-8 relative residual drop or at its fixed end, the iteration at which its
    cells x iterations reach args.serve_end cell-updates; its state is read back to the host
    before it is retired, inside its latency. Beside it, the first args.serve_seq requests of the
    same stream solved one after another through the plain FP64 path with the same retirement
    rule and read-back (one context per request, wall clock including setup). The payloads of
    both come from the clients and are built before the timed region; admission (validation,
    metrics, upload) is timed."""
    from q2d_b200 import _abi
    from q2d_b200.serve import request_stream, serve, serve_options
    from q2d_b200.solver import Q2DSolver
    reqs = request_stream(args.serve_rate, args.serve_seconds, distinct=args.serve_distinct)
    # the request payloads (grid, initial state, boundary records) come from clients: built before
    # the timed region, one per distinct seeded case
    for r in reqs[:args.serve_distinct]:
        r.build()
    for r in reqs[args.serve_distinct:]:
        r.case = reqs[r.rid % args.serve_distinct].case
    bad = []

    def sink(r, states):   # the client takes the result away (a spot check of each block)
        if not all(np.isfinite(x[2:-2:7, 2:-2:7]).all() for x in states):
            bad.append(r.rid)
    import torch
    rb = torch.empty(int(args.serve_readback_gb * (1 << 30)) // 8, dtype=torch.float64, pin_memory=True).numpy()
    opts = serve_options(itermax=10 ** 9, drop=1e-8)
    st = serve(reqs, opts, device_bytes=int(args.serve_gb * (1 << 30)), max_cases=4096, steps_per_call=10,
               keep_results=True, end_cell_updates=args.serve_end, result_sink=sink, readback_buffer=rb)
    del rb
    st["nonfinite_results"] = len(bad)
    st["distinct_payloads"] = args.serve_distinct
    for r in reqs:
        r.case = None
    # sequential plain FP64 on the first requests of the same stream, same rule and read-back
    seq = request_stream(args.serve_rate, args.serve_seconds, distinct=args.serve_distinct)[:args.serve_seq]
    for r in seq:
        r.build()
    opts64 = serve_options(precision=_abi.PREC_FP64, itermax=10 ** 9, drop=1e-8)
    t0 = time.perf_counter()
    cu = 0
    for r in seq:
        case = r.case
        s = Q2DSolver(opts64, [case])
        try:
            end_iter = max(1, -(-int(args.serve_end) // case.cells))
            info = s.step(end_iter)[0]
            _ = [s.prim(0, b) for b in range(len(case.blocks))]
            cu += case.cells * info["iter"]
        finally:
            s.close()
    tseq = time.perf_counter() - t0
    seq_v = cu / tseq
    st.update({"arrival_rate_per_s": args.serve_rate, "arrival_window_s": args.serve_seconds,
               "end_cell_updates_per_request": args.serve_end, "residual_drop": 1e-8,
               "budget_gb": args.serve_gb, "dtype": "fp32-flux/fp64-state", "readback": True,
               "sequential_plain_fp64": {"value": seq_v, "unit": UNIT, "requests": len(seq),
                                         "cell_updates": cu, "seconds": tseq, "readback": True},
               "ratio_served_over_sequential_fp64": st["cell_updates_per_s"] / seq_v})
    if fp64_batched:
        st["ratio_served_over_batched_fp64"] = st["cell_updates_per_s"] / fp64_batched
    return st


def _rel_l1(a, b, gamma=1.4):
    """Relative L1 error per conserved variable, sum |U(a) - U(b)| / sum |U(b)| (both momenta
    against sum |rho V|), and the same per primitive variable over its scale (max |b|)."""
    def cons(p):
        r, u, v, q = (p[..., k] for k in range(4))
        return np.stack([r, r * u, r * v, q / (gamma - 1) + 0.5 * r * (u * u + v * v)], axis=-1).reshape(-1, 4)
    Ua, Ub = cons(a), cons(b)
    den = np.abs(Ub).sum(axis=0)
    den[1] = den[2] = max(np.hypot(Ub[:, 1], Ub[:, 2]).sum(), 1e-300)
    std = np.abs(Ua - Ub).sum(axis=0) / den
    bb = b.reshape(-1, 4)
    snd = np.sqrt(gamma * np.abs(bb[:, 3]) / np.abs(bb[:, 0]))
    vs = max(np.abs(bb[:, 1]).max(), np.abs(bb[:, 2]).max(), snd.max())
    sc = np.array([np.abs(bb[:, 0]).max(), vs, vs, np.abs(bb[:, 3]).max()])
    d = np.abs(a.reshape(-1, 4) - bb) / sc
    return float(std.max()), float(d.mean(axis=0).max()), float(d.max())


def accuracy_leg(batch, n=512, steps=2000):
    """The batched workload's FP32-flux error against the plain FP64 GPU path after the
    configuration's 2000 steps, on the first n cases: relative L1 per conserved variable (the
    north star's metric), the max-scaled relative L1 and L-inf of the primitive variables,
    worst case of the sample."""
    from q2d_b200 import make_options
    from q2d_b200.solver import Q2DSolver
    sample = batch[:n]
    out = []
    for prec in (1, 0):
        s = Q2DSolver(make_options(sample[0], precision=prec), sample)
        try:
            for _ in range(steps // 500):
                s.step(500)
            if steps % 500:
                s.step(steps % 500)
            out.append([p[0] for p in s.prims()])
        finally:
            s.close()
    errs = [_rel_l1(a, b) for a, b in zip(out[0], out[1])]
    return {"vs": "plain FP64 GPU path", "cases": len(sample), "steps": steps,
            "rel_l1_cons_max": max(e[0] for e in errs), "rel_l1_max": max(e[1] for e in errs),
            "rel_linf_max": max(e[2] for e in errs)}


def configs_leg(lib):
    """Configurations 1-3 at their stated sizes: each solved in the plain FP64 form and in the
    FP32-flux form, device time per step (CUDA events), cell-updates/s and the FP32-flux error
    against FP64 at the end."""
    from q2d_b200 import cases, make_options
    from q2d_b200.solver import Q2DSolver

    def solve(cs, prec, steps, chunk, **ov):
        s = Q2DSolver(make_options(cs, precision=prec, **ov), [cs])
        try:
            s.step(1)
            ms, _ = time_device(lib, s, 1)
            info = s.info(0)
            t0 = time.perf_counter()
            done = 2
            while done < steps and info["todo"] != 3:
                info = s.step(min(chunk, steps - done))[0]
                done = info["iter"]
            wall = time.perf_counter() - t0
            return [s.prim(0, b) for b in range(len(cs.blocks))], info, ms, wall
        finally:
            s.close()

    out = {}
    specs = [("1", cases.riemann_1d(), 10 ** 6, 1000, {},
              "1-D Riemann 1024x4, minmod + HLLC, SSP-RK3, CFL 0.5, time accurate to t = 0.15"),
             ("2", cases.ramp(), 4000, 500, {},
              "compression ramp 1536x512, van Leer + HLLC, SSP-RK3, local dt, 4000 steps"),
             ("3", cases.nozzle_axi(), 20000, 2000, {"cfl": 0.2, "res_relative": 1},
              "axisymmetric nozzle 4 x 512x128, minmod + HLLC, SSP-RK3, local dt at CFL 0.2, 20000 "
              "iterations (the residual stalls near 1e-3 of its peak: no 1e-10 drop)")]
    for key, cs, steps, chunk, ov, what in specs:
        res = {"workload": what, "cells": cs.cells}
        states = {}
        for name, prec in (("fp64", 0), ("fp32_flux", 1)):
            P, info, ms, wall = solve(cs, prec, steps, chunk, **ov)
            states[name] = P
            res[name] = {"iterations": int(info["iter"]), "time": info["time"], "err": info["err"],
                         "ms_per_step": ms, "cell_updates_per_s": cs.cells / (ms / 1e3),
                         "residual_drop": info["residual"][0] / info["residual0"] if info["residual0"] > 0 else None,
                         "wall_s": wall}
        e = [_rel_l1(a, b) for a, b in zip(states["fp32_flux"], states["fp64"])]
        res["fp32_flux_vs_fp64"] = {"rel_l1_cons_max": max(x[0] for x in e), "rel_l1_max": max(x[1] for x in e),
                                    "rel_linf_max": max(x[2] for x in e)}
        out[key] = res
    return out


WORKLOAD = ("batched area-variation nozzles (4096 independent cases per GPU, Nx~lognormal[64,1024], "
            "Ny~U{8..64}), van Leer + HLLC, SSP-RK3, local dt")


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    batch = batch_cases(args.cases, 0)
    cb = cpu_baseline(batch, budget_s=max(5.0, min(60.0, 0.5 * (args.steps + args.warmup))))
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cases_per_gpu": len(batch),
                       "cells_per_gpu": int(sum(cs.cells for cs in batch)), "parallelism": "host threads",
                       "measured_on": "a bounded sample of the cases (cpu_baseline.sample)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    from q2d_b200 import make_options, _abi
    from q2d_b200.solver import Q2DSolver
    from q2d_b200 import replicas
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        replicas.init("nccl", timeout_s=300)
    lib = _abi.load_library()
    K, W = args.steps, max(3, args.warmup)
    batch = batch_cases(args.cases, rank)
    cells = sum(c.cells for c in batch)
    cells_all = replicas.sum_over_ranks(cells, "cuda")   # whole-job cells (replicas, weak scaling)
    barrier = replicas.barrier

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, "cuda")

    # ---- FP32-flux / FP64-state batched form (the headline) ----------------------------
    prec = 1 if args.form == "fp32-flux" else 0
    s = Q2DSolver(make_options(batch[0], precision=prec), batch)
    if args.schedule is None:
        tuned = s.autotune(2)
        tuned["schedule"] += " (autotuned)"
    else:
        s.set_schedule(args.schedule)
        tuned = {"schedule": s.schedule + " (pinned)"}
    s.step(W)
    barrier()
    with ClockSampler(local) as clk:
        ms, launches = time_device(lib, s, K)
    ms = max_over_ranks(ms)
    value = cells_all * K / (ms / 1e3)
    infos = s.step(0)
    errs = sum(1 for i in infos if i["err"])
    t_launch = ms / 1e3 / (K * STAGES)
    achieved = (B_ALG / STAGES) * cells / t_launch / 1e9
    peaks = {}
    try:
        peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic = read_traffic(s.schedule)
    # ---- e2e through the C ABI with host buffers ----------------------------------------
    e2e = None
    if not args.no_e2e:
        P_host = []
        for cs in batch:
            a = torch.empty((cs.blocks[0].nj + 4, cs.blocks[0].ni + 4, 4), dtype=torch.float64,
                            pin_memory=True).numpy()
            a[...] = cs.blocks[0].prim_ghost()
            P_host.append(a)
        outs = [torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy() for a in P_host]
        infos_t = (_abi.StepInfo * len(batch))()
        Ke = max(3, K // 2)
        assert lib.q2d_gpu_prepare(s.ctx, 1) == 0
        torch.cuda.synchronize()
        barrier()
        nb = len(batch)
        ids = (C.c_int * nb)(*[s.block_ids[b][0] for b in range(nb)])
        p_in = (C.POINTER(C.c_double) * nb)(*[_abi.dptr(a) for a in P_host])
        p_out = (C.POINTER(C.c_double) * nb)(*[_abi.dptr(o) for o in outs])
        t0 = time.perf_counter()
        st = lib.q2d_gpu_upload_prim_many(s.ctx, nb, ids, p_in)
        for _ in range(Ke):
            st = st or lib.q2d_gpu_step(s.ctx, 1, infos_t)
        st = st or lib.q2d_gpu_download_prim_many(s.ctx, nb, ids, p_out)
        te = max_over_ranks(time.perf_counter() - t0)
        assert st == 0, lib.q2d_gpu_last_error(s.ctx)
        bytes_state = sum(a.nbytes for a in P_host)   # upload: each whole ghosted array
        bytes_interior = sum(32 * cs.blocks[0].ni * cs.blocks[0].nj for cs in batch)   # download: interior rows
        e2e = {"value": cells_all * Ke / te, "unit": UNIT,
               "h2d_bytes_per_step": int(bytes_state / Ke),
               "d2h_bytes_per_step": int(bytes_interior / Ke + C.sizeof(_abi.StepInfo) * len(batch)),
               "steps": Ke, "seconds": te,
               "path": "q2d_gpu_upload_prim_many (every block) + q2d_gpu_step(1) x steps (per-step "
                       "case info to host) + q2d_gpu_download_prim_many (every block)"}
    s.close()
    # ---- plain FP64 form of the same batch -------------------------------------------------
    fp64 = None
    if not args.no_fp64:
        s64 = Q2DSolver(make_options(batch[0], precision=0), batch)
        tuned64 = s64.autotune(1)
        s64.step(W)
        K64 = max(5, K // 4)
        ms64, _ = time_device(lib, s64, K64)
        ms64 = max_over_ranks(ms64)
        v64 = cells_all * K64 / (ms64 / 1e3)
        fp64 = {"value": v64, "unit": UNIT, "steps": K64, "ms_per_step": ms64 / K64,
                "schedule": tuned64["schedule"] + " (autotuned)",
                "ratio_fp32flux_over_fp64": value / v64}
        s64.close()
    # ---- the same batch with implicit residual smoothing (irs-beta 0.5), FP32-flux form ----------
    irs = None
    if not args.no_fp64:
        sir = Q2DSolver(make_options(batch[0], precision=prec, irs_beta=0.5), batch)
        sir.autotune(1)   # the smoothing passes run on the tile kernels
        sir.step(W)
        Ki = max(5, K // 4)
        msi, li = time_device(lib, sir, Ki)
        msi = max_over_ranks(msi)
        irs = {"value": cells_all * Ki / (msi / 1e3), "unit": UNIT, "steps": Ki, "ms_per_step": msi / Ki,
               "irs_beta": 0.5, "gpu_launches": li, "schedule": sir.schedule,
               "note": "each stage: scaled-residual pass, smoothing along i and j, update pass"}
        sir.close()
    served = None
    if not args.no_serve:
        served = serving_leg(args, lib, fp64["value"] if fp64 else None)
    accuracy = accuracy_leg(batch) if not args.no_fp64 else None
    configs = configs_leg(lib) if not args.no_fp64 else None
    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(batch)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32-flux/fp64-state" if prec == 1 else "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cases_per_gpu": len(batch), "cells_per_gpu": cells,
                   "schedule": tuned["schedule"],
                   "parallelism": f"replicas x{world} (independent cases per GPU)",
                   "l2": "inputs larger than L2 (state %.2f GB per buffer)" % (cells * 32 / 1e9)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650",
                     "bytes_per_cell_update": B_ALG, "launch_ms": t_launch * 1e3},
        "gpu_launches": launches, "errors": errs,
        "clocks": clk.summary(),
        "e2e": e2e, "plain_fp64": fp64, "irs": irs, "served": served, "accuracy_fp32flux": accuracy,
        "configs": configs,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
