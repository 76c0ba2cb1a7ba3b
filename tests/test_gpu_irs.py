"""Implicit residual smoothing (irs-beta > 0; Lib_IRS.f90:17-177, Lib_Newstate.f90:36-66) on the
GPU: the scaled residual of each stage is smoothed by two Jacobi sweeps along i, then along j,
before the update.

* FP64 form against the CPU oracle, which restates the reference's smoothing loop by loop:
  <= 1e-12 relative L-infinity after one step, <= 1e-10 after several, on every boundary type
  (connections between blocks included), the axisymmetric and area-variation sources, a 1-D
  time-accurate case (one direction only) and each RK scheme.
* FP32-flux form against the FP64 form with the same smoothing: <= 1e-6 relative L1.
* Smoothing changes the trajectory (the same case without it differs).
"""
import numpy as np
import pytest

from q2d_b200 import cases, make_options
from q2d_b200.solver import Q2DSolver
from tests.conftest import rel_l1, rel_linf
from tests.helpers import run_pair

pytestmark = pytest.mark.gpu


def check(gs, os_, tol, what):
    for c, (gb, ob) in enumerate(zip(gs, os_)):
        for b, (g, o) in enumerate(zip(gb, ob)):
            assert np.all(np.isfinite(g)), f"{what}: non-finite state case {c} block {b}"
            err = rel_linf(g, o)
            assert err.max() <= tol, f"{what}: case {c} block {b} rel Linf {err} > {tol}"


@pytest.mark.parametrize("n_rk", [1, 2, 3])
def test_irs_ramp_vs_oracle(n_rk):
    cs = cases.ramp(64, 24, seed=3)
    gs, os_, gi, oi = run_pair([cs], 1, n_rk=n_rk, irs_beta=0.5)
    check(gs, os_, 1e-12, f"ramp irs rk{n_rk} 1 step")
    gs, os_, gi, oi = run_pair([cs], 12, chunks=3, n_rk=n_rk, irs_beta=0.5)
    check(gs, os_, 1e-10, f"ramp irs rk{n_rk} 12 steps")
    assert gi[0]["iter"] == oi[0]["iter"] == 12
    assert gi[0]["residual"][0] == pytest.approx(oi[0]["residual"][0], rel=1e-9)


def test_irs_connected_blocks_vs_oracle():
    cs = cases.nozzle_axi(ni=40, nj=12, nblocks=3, seed=9)
    gs, os_, gi, oi = run_pair([cs], 1, irs_beta=0.5)
    check(gs, os_, 1e-12, "nozzle_axi irs 1 step")
    gs, os_, gi, oi = run_pair([cs], 10, chunks=2, irs_beta=0.5)
    check(gs, os_, 1e-10, "nozzle_axi irs 10 steps")


def test_irs_area_batch_and_1d_vs_oracle():
    batch = cases.area_nozzle_batch(n=4, seed=11, nx_range=(24, 60), ny_range=(4, 10))
    gs, os_, gi, oi = run_pair(batch, 6, chunks=2, irs_beta=0.3)
    check(gs, os_, 1e-10, "area batch irs")
    cs = cases.riemann_1d(ni=96, nj=1, seed=7)
    gs, os_, gi, oi = run_pair([cs], 8, chunks=2, irs_beta=0.5)
    check(gs, os_, 1e-10, "riemann1d irs (ndir 1, time-accurate)")


def test_irs_changes_the_trajectory():
    cs = cases.ramp(48, 16, seed=4)
    a, _, _, _ = run_pair([cs], 5, irs_beta=0.5)
    b, _, _, _ = run_pair([cs], 5)
    assert not np.array_equal(a[0][0], b[0][0])


@pytest.mark.parametrize("schedule", ["fp32-flux tile 32x8", "fp32-flux tile 32x10", "tile 32x10"])
def test_irs_fp32flux_vs_fp64(schedule):
    batch = [cases.nozzle_axi(ni=40, nj=12, nblocks=2, seed=5),
             cases.area_nozzle_batch(n=2, seed=13, nx_range=(40, 80), ny_range=(8, 12))[0]]
    out = []
    for prec, sched in ((1, schedule), (0, None)):
        s = Q2DSolver(make_options(batch[0], precision=prec, irs_beta=0.5), batch)
        try:
            if sched is not None:
                s.set_schedule(sched)
            infos = s.step(20, check=False)
            assert all(i["err"] == 0 for i in infos)
            out.append([[s.prim(c, b) for b in range(len(cs.blocks))] for c, cs in enumerate(batch)])
        finally:
            s.close()
    for ca, cb in zip(*out):
        for xa, xb in zip(ca, cb):
            assert rel_l1(xa, xb).max() <= 1e-6


def test_planar_nozzle_reference_case_through_host(tmp_path):
    """The reference's planar-nozzle case written in its own formats and run by q2d_host on the
    GPU (FP64 form, IRS beta 0.5): the density residual follows the reference binary's printed
    history within 5 %, res-threshold 1e-10 is met within 5 iterations of the binary (3172),
    and the field it writes passes the case's area-law acceptance gates."""
    from pathlib import Path
    from q2d_b200 import refio
    from tests.helpers import planar_nozzle_gates
    from tests.test_host_harness import host
    hist = np.loadtxt(Path(__file__).resolve().parent / "golden" / "planar_nozzle_residuals.txt")
    cs = cases.planar_nozzle()
    refio.write_case(cs, tmp_path)
    gamma = make_options(cs).gas_gamma
    host(tmp_path, "--gamma", repr(gamma), "--steps-per-call", 500, "--quiet")
    res = np.loadtxt(tmp_path / "OUTPUT" / "residuals.dat")
    by_iter = {int(r[0]): r[3] for r in res}
    for it, ref in hist[:-1]:
        assert abs(by_iter[int(it)] / ref - 1.0) < 0.05, (it, by_iter[int(it)], ref)
    assert abs(res[-1, 0] - hist[-1, 0]) <= 5 and res[-1, 3] <= 1e-10
    prim = refio.read_field(tmp_path / "OUTPUT" / "field.tec")[0].prim
    planar_nozzle_gates(prim, cs.meta["xc"], gamma)


def test_planar_nozzle_fp32flux_passes_the_area_law():
    """The same case in the FP32-flux form: its residual stalls at the FP32 level of the fluxes
    (far above the FP64 threshold), so it runs 4000 iterations; the state then passes the same
    acceptance gates and differs from the FP64 form's by less than the form's bound."""
    from tests.helpers import planar_nozzle_gates
    cs = cases.planar_nozzle()
    out = []
    for prec in (1, 0):
        s = Q2DSolver(make_options(cs, precision=prec, itermax=4000, res_threshold=0.0), [cs])
        try:
            infos = s.step(4000, check=False)
            assert infos[0]["err"] == 0 and infos[0]["iter"] == 4000
            out.append(s.prim(0, 0))
        finally:
            s.close()
    planar_nozzle_gates(out[0], cs.meta["xc"], make_options(cs).gas_gamma)
    assert rel_l1(out[0], out[1]).max() <= 1e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_chang_nozzle_reference_case(precision):
    """The reference's chang-nozzle case (axisymmetric source, IRS beta 0.5, MC + HLLC, CFL 0.8)
    on the GPU: the FP64 form converges to the oracle's iteration count and state, the FP32-flux
    form runs the case's 5000 iterations; both pass the case's gates against Chang's data along
    the wall and the axis."""
    from tests.helpers import chang_nozzle_case, chang_nozzle_gates
    cs = chang_nozzle_case()
    s = Q2DSolver(make_options(cs, precision=precision), [cs])
    try:
        info = s.solve(steps_per_call=500)
        assert info["err"] == 0
        prim = s.prim(0, 0)
    finally:
        s.close()
    chang_nozzle_gates(cs, prim)
    if precision == 0:
        from oracle import oracle
        o = oracle.solver(make_options(cs), [cs])
        try:
            oi = o.solve(steps_per_call=500)
            ref = o.prim()
        finally:
            o.close()
        assert info["iter"] == oi["iter"] and info["residual"][0] <= 1e-10
        assert rel_linf(prim, ref).max() <= 1e-8


def test_chang_nozzle_reference_case_through_host(tmp_path):
    """The chang-nozzle case written in the reference's formats (axisymmetric source, IRS) and
    run by q2d_host: it stops at the case's res-threshold within its 5000 iterations, the
    residual history is the reference's format, and the field passes the case's Mach gates."""
    from q2d_b200 import refio
    from tests.helpers import chang_nozzle_case, chang_nozzle_gates
    from tests.test_host_harness import host
    cs = chang_nozzle_case()
    refio.write_case(cs, tmp_path, res_threshold=1e-10, res_diter=100)
    host(tmp_path, "--gamma", repr(cs.options["gas_gamma"]), "--steps-per-call", 500, "--quiet")
    lines = (tmp_path / "OUTPUT" / "residual-history.dat").read_text().splitlines()
    assert lines and all(len(ln) == 108 for ln in lines)
    res = np.loadtxt(tmp_path / "OUTPUT" / "residuals.dat")
    assert res[-1, 0] < 5000 and res[-1, 3] <= 1e-10
    chang_nozzle_gates(cs, refio.read_field(tmp_path / "OUTPUT" / "field.tec")[0].prim)
